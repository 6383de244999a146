"""GPU parity on the configurations as they are stated, through the C ABI, against the oracle.

- C1: 4,096 non-overlapping r = 1 mm spheres in a walled 5 cm cube, gravity, mu 0.3, e 0.8,
  dt 1e-7 s, Verlet skin 0.1 r, the reference's quirks, 10,000 steps, unmodified
  (`scenarios.random_box()`): every field bit-identical to the oracle with x^1.5 = x*sqrt(x),
  tangential slot layout, slot history and wall history included; against the oracle's libm
  pow (the reference's literal arithmetic) within 1e-10 relative.
- C2: the 2,000,000-sphere lattice, 64 steps with a neighbour rebuild (Morton re-sort and
  history remap) forced in the middle: every field, slot and wall history included.
- Hertz elastic energy totals of dem_energy against the oracle's brute-force restatement.
- Mixed precision on the C2 lattice compressed by 3 % (about 10^5 contacts) after a warm-up
  that builds tangential history: one force pass from the same state, force and torque
  within 1e-5 of FP64.
"""
import numpy as np
import pytest

from cabanadem_b200 import api, scenarios as S
from cabanadem_b200._lib import DEM_FP64, DEM_MIXED
from oracle import oracle as O

pytestmark = pytest.mark.gpu

STATE_F = ("x", "u", "omega", "force", "torque")
HIST_F = ("tng_idx", "tng_ss_x", "tng_ss_y", "tng_ss_z", "tng_count")
WALL_F = ("tng_sw_x", "tng_sw_y", "tng_sw_z")
ALL_F = STATE_F + HIST_F + WALL_F
FORCE_TOL = 1e-5     # mixed precision: max |F_mixed - F_fp64| / max |F_fp64|
LIBM_TOL = 1e-10     # FP64 against the oracle's libm pow, relative to the field's largest value



def _assert_bitwise(got, ref, fields=ALL_F, where=""):
    for f in fields:
        a, b = getattr(got, f), getattr(ref, f)
        if f.startswith("tng_sw"):
            a, b = a[:, : b.shape[1]], b[:, : a.shape[1]]
        if f in ("tng_idx", "tng_ss_x", "tng_ss_y", "tng_ss_z"):
            # the live slots: those below the particle's contact count
            mask = np.arange(a.shape[1])[None, :] < ref.tng_count[:, None]
            a, b = np.where(mask, a, 0), np.where(mask, b, 0)
        if not np.array_equal(a, b):
            d = np.abs(np.asarray(a, float) - np.asarray(b, float))
            raise AssertionError("%s %s differs: max |d| = %g at %s" % (where, f, d.max(),
                                                                        np.unravel_index(d.argmax(), d.shape)))


def _oracle(sc, nsteps, pow_mode=O.POW_SQRT, state=None):
    ref = (state if state is not None else sc.state).copy()
    st = O.run(ref, sc.walls.copy(), sc.params, sc.dt, nsteps, delta=sc.delta, skin=sc.skin, gravity=sc.gravity,
               pow_mode=pow_mode)
    return ref, st


def test_c1_as_configured_10000_steps_bitwise():
    """C1 unmodified: 10,000 fused steps in three runs, every field bit-identical to the
    oracle; then the same run against the libm-pow oracle within 1e-10 over all 10,000 steps
    (at this packing, a gas with a few contacts at a time, the two arithmetics stay within
    5e-16 of each other throughout)."""
    sc = S.random_box()
    assert sc.state.n == 4096 and sc.nsteps == 10_000 and sc.delta == 0.0
    ref, st = _oracle(sc, sc.nsteps)
    assert st == 0
    s = api.from_scenario(sc)
    for n in (3333, 3333, 3334):
        s.run_steps(n)
    got = s.particles.download()
    _assert_bitwise(got, ref, where="C1")
    assert ref.tng_count.sum() > 0      # pair contacts live at the end
    assert s.stats()["rebuilds"] >= 2
    lib, _ = _oracle(sc, sc.nsteps, pow_mode=O.POW_LIBM)
    for f in STATE_F:
        a, b = getattr(got, f), getattr(lib, f)
        err = np.abs(a - b).max() / np.abs(b).max()
        assert err <= LIBM_TOL, (f, err)


def test_c2_64_steps_with_a_forced_rebuild_bitwise():
    """C2, 2,000,000 spheres: 30 steps, a full rebuild (re-sort along the Morton curve with
    contact-partner and history remap), 34 more steps; every field against the oracle's 64
    steps, slot and wall history included."""
    sc = S.hcp_box()
    ref, st = _oracle(sc, 64)
    assert st == 0
    s = api.from_scenario(sc)
    s.run_steps(30)
    r0 = s.stats()["rebuilds"]
    s.rebuild()
    assert s.stats()["rebuilds"] == r0 + 1
    s.run_steps(34)
    _assert_bitwise(s.particles.download(), ref, where="C2")
    assert ref.tng_count.sum() > 0


def test_elastic_energy_totals_match_the_oracle():
    """dem_energy out[2] (pairs) and out[3] (walls): the Hertz elastic energy 2/5 kn d^2.5 of
    every overlap, against the oracle's brute-force sum over all pairs (a different summation
    order: 1e-12 relative); out[0] + out[1] against the oracle's kinetic energy."""
    sc = S.random_box(n=4096, nsteps=200)
    c = sc.state.x.mean(axis=0)
    sc.state.x[:] = c + (sc.state.x - c) * 0.6
    sc.state.x[:, 2] -= sc.state.x[:, 2].min() - 0.9 * sc.state.rad[0]   # the lowest layer presses into the floor
    s = api.from_scenario(sc)
    s.run_steps(200)
    got = s.particles.download()
    e = s.energy()
    ep, ew = O.elastic_energy(got, sc.walls)
    assert ep > 0 and ew > 0
    assert abs(e[2] - ep) <= 1e-12 * ep, (e[2], ep)
    assert abs(e[3] - ew) <= 1e-12 * ew, (e[3], ew)
    ke = O.kinetic_energy(got)
    assert abs(e[0] + e[1] - ke) <= 1e-12 * ke
    assert np.array_equal(e, s.energy())


def _force_pass(sc, state, precision):
    s = api.from_scenario(sc, precision=precision)
    s.particles.upload(state)
    s.build_neighbors()
    s.compute_force()
    out = s.particles.download()
    s.close()
    s.particles.close()
    return out


@pytest.mark.parametrize("quirks", [S.REF_COMPAT, 0x00], ids=["ref_compat", "fixed"])
def test_mixed_force_error_on_the_c2_lattice(quirks):
    """One force pass from the same warmed-up state in both precisions.  With the reference's
    quirks the pair contacts add no torque (src/CabanaDEM_Force.hpp:324-326) and the lattice
    touches no wall, so the torque is zero in both; with every quirk clear it is not."""
    sc = S.hcp_box(quirks=quirks)
    c = sc.state.x.mean(axis=0)
    sc.state.x[:] = c + (sc.state.x - c) * 0.97
    warm = api.from_scenario(sc)
    warm.run_steps(40)
    state = warm.particles.download()
    warm.close()
    warm.particles.close()
    assert state.tng_count.sum() > 50_000
    a = _force_pass(sc, state, DEM_FP64)
    b = _force_pass(sc, state, DEM_MIXED)
    g = np.asarray(sc.gravity)[None, :] * state.m[:, None]
    for f in ("force", "torque"):
        ref, mix = getattr(a, f), getattr(b, f)
        contact = ref - g if f == "force" else ref
        scale = np.abs(contact).max()
        if f == "torque" and quirks & 0x04:
            assert scale == 0.0 and np.abs(mix).max() == 0.0
            continue
        assert scale > 0.0, f
        err = np.abs(mix - ref).max() / scale
        assert err <= FORCE_TOL, (f, err)
    assert np.array_equal(a.tng_count, b.tng_count)
