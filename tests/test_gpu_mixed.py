"""Mixed-precision path (FP32 contact forces on FP64 pair offsets; FP64 history, sums and
integration) against the FP64 path on the same inputs.  The bar is 1e-5 relative force error,
and each physical observable of the reference's validation cases (peak normal force, contact
duration, coefficient of restitution, rebound spin, energy drift) is stated as an error."""
import numpy as np
import pytest

from cabanadem_b200 import api, scenarios as S
from cabanadem_b200._lib import DEM_FP64, DEM_MIXED

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5


def _force_pass(sc, precision):
    s = api.from_scenario(sc, rebuild_every_step=True, precision=precision)
    s.build_neighbors()
    s.compute_force()
    st = s.particles.download()
    s.close()
    return st


@pytest.mark.parametrize("quirks", [S.REF_COMPAT, 0x00], ids=["ref_compat", "fixed"])
def test_mixed_force_error_dense_pack(quirks):
    """One force pass from an identical dense state (thousands of contacts, friction,
    walls): max |F_mixed - F_fp64| / max |F_fp64| <= 1e-5, same for torque."""
    sc = S.random_box(n=4096, quirks=quirks)
    c = sc.state.x.mean(axis=0)
    sc.state.x[:] = c + (sc.state.x - c) * 0.97
    # give tangential history something to act on: one step of motion first
    warm = api.from_scenario(sc, rebuild_every_step=True)
    warm.run_steps(20)
    sc.state = warm.particles.download()
    warm.close()
    a = _force_pass(sc, DEM_FP64)
    b = _force_pass(sc, DEM_MIXED)
    assert a.tng_count.sum() > 50
    for f in ("force", "torque"):
        ref = getattr(a, f)
        scale = np.abs(ref).max()
        if scale == 0:
            continue
        err = np.abs(getattr(b, f) - ref).max() / scale
        assert err <= FORCE_TOL, (f, err)
    assert np.array_equal(a.tng_count, b.tng_count)


def _trajectory(sc, precision, every=1):
    s = api.from_scenario(sc, rebuild_every_step=True, precision=precision)
    out = []
    for _ in range(0, sc.nsteps, every):
        s.run_steps(every)
        st = s.particles.download()
        out.append((st.force.copy(), st.u.copy(), st.omega.copy(), st.x.copy()))
    s.close()
    return out


def test_mixed_observables_head_on(example_inputs):
    sc = S.example01(example_inputs["01_elastic_normal_impact_of_two_identical_particles"])
    res = {}
    for prec in (DEM_FP64, DEM_MIXED):
        tr = _trajectory(sc, prec, every=1)
        f = np.array([t[0][1, 0] for t in tr])
        on = np.nonzero(f)[0]
        res[prec] = dict(peak=f.max(), dur=len(on), v_out=tr[-1][1][1, 0])
    assert abs(res[DEM_MIXED]["peak"] / res[DEM_FP64]["peak"] - 1) < FORCE_TOL
    assert res[DEM_MIXED]["dur"] == res[DEM_FP64]["dur"]
    assert abs(res[DEM_MIXED]["v_out"] / res[DEM_FP64]["v_out"] - 1) < FORCE_TOL


@pytest.mark.parametrize("cor", [0.2, 0.6, 0.9])
def test_mixed_restitution(example_inputs, cor):
    sc = S.example03(example_inputs["03_normal_particle_wall_different_cor"], cor)
    out = {}
    for prec in (DEM_FP64, DEM_MIXED):
        s = api.from_scenario(sc, rebuild_every_step=True, precision=prec)
        s.run_steps(sc.nsteps)
        out[prec] = s.particles.get("u")[0, 1]
        s.close()
    assert abs(out[DEM_MIXED] - out[DEM_FP64]) <= FORCE_TOL * abs(out[DEM_FP64])


@pytest.mark.parametrize("angle", [10.0, 30.0, 60.0])
def test_mixed_rebound_spin(example_inputs, angle):
    sc = S.example04(example_inputs["04_oblique_particle_wall_different_angles"], angle)
    out = {}
    for prec in (DEM_FP64, DEM_MIXED):
        s = api.from_scenario(sc, rebuild_every_step=True, precision=prec)
        s.run_steps(sc.nsteps)
        out[prec] = s.particles.get("omega")[0, 2]
        s.close()
    assert abs(out[DEM_MIXED] - out[DEM_FP64]) <= 1e-4 * abs(out[DEM_FP64])


def test_mixed_energy_drift_elastic(example_inputs):
    """e = 1, mu = 0 head-on impact: kinetic energy after the rebound equals the energy
    before within the FP64 path's own drift."""
    sc = S.example01(example_inputs["01_elastic_normal_impact_of_two_identical_particles"])
    ke0 = 0.5 * (sc.state.m * (sc.state.u ** 2).sum(axis=1)).sum()
    drift = {}
    for prec in (DEM_FP64, DEM_MIXED):
        s = api.from_scenario(sc, rebuild_every_step=True, precision=prec)
        s.run_steps(sc.nsteps)
        e = s.energy()
        drift[prec] = abs(e[0] + e[1] - ke0) / ke0
        s.close()
    assert drift[DEM_FP64] < 1e-3
    assert abs(drift[DEM_MIXED] - drift[DEM_FP64]) < 1e-5


def test_mixed_contact_kernels_agree():
    """Mixed precision through the per-thread and the cooperative contact kernel, the
    one-kernel dense step and the pair-parallel dense step: the same per-contact function and
    summation order, so the same state after 300 dense steps."""
    sc = S.random_box(n=4096, nsteps=300)
    c = sc.state.x.mean(axis=0)
    sc.state.x[:] = c + (sc.state.x - c) * 0.6
    got = []
    # 0: the one-kernel dense step once the box is found dense; (0, 2): the pair-parallel form
    for lanes, form in ((1, 0), (8, 0), (0, 0), (0, 2)):
        s = api.from_scenario(sc, precision=DEM_MIXED, contact_lanes=lanes, dense_form=form)
        s.run_steps(300)
        got.append(s.particles.download())
    for other in got[1:]:
        for f in ("x", "u", "omega", "force", "torque", "tng_count"):
            assert np.array_equal(getattr(got[0], f), getattr(other, f)), f
