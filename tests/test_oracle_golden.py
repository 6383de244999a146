"""Pin the CPU oracle to the reference's golden data (examples/validation_data/*.csv and the
COR identity line), with the observables automate.py reads (automate.py:134-135, :315, :447).
The CSVs are digitised curves, so tolerances are a few percent of the peak."""
import numpy as np
import pytest

from cabanadem_b200 import scenarios as S
from oracle import oracle as O

T1 = "01_elastic_normal_impact_of_two_identical_particles"
T4_LETHE = "04_oblique_particle_wall_different_angles_omega_vs_incident_angle_Lethe_DEM_data"
T4_EXP = "04_oblique_particle_wall_different_angles_omega_vs_incident_angle_Kharaz_Gorham_Salman_experimental_data"


def _run_test1(example_inputs):
    sc = S.example01(example_inputs[T1])
    st = sc.state
    t, f, ov = [], [], []
    for step in range(sc.nsteps):
        O.run(st, sc.walls, sc.params, sc.dt, 1, delta=sc.delta)
        t.append(step * sc.dt)
        f.append(st.force[1, 0])      # automate.py:134: forces[1][0]
        ov.append(st.rad[0] + st.rad[1] - (st.x[1, 0] - st.x[0, 0]))
    return sc, np.array(t), np.array(f), np.array(ov)


def test_example01_force_vs_time(example_inputs, validation_data):
    sc, t, f, _ = _run_test1(example_inputs)
    ref = validation_data[T1 + "_time_vs_fn_analytical_data"]
    on = np.nonzero(f)[0]
    t0 = t[on[0]]
    sim = np.interp(ref[:, 0] * 1e-6 + t0, t, f / 1e3)
    peak = ref[:, 1].max()
    assert np.max(np.abs(sim - ref[:, 1])) < 0.03 * peak
    # contact duration within one digitised sample of the analytical 40.4 us
    dur = (on[-1] - on[0] + 1) * sc.dt * 1e6
    assert abs(dur - ref[-1, 0]) < 1.0
    assert abs(f.max() / 1e3 - peak) < 0.01 * peak


def test_example01_force_vs_overlap(example_inputs, validation_data):
    _, _, f, ov = _run_test1(example_inputs)
    ref = validation_data[T1 + "_overlap_vs_fn_analytical_data"]
    load = slice(0, int(np.argmax(ov)) + 1)
    order = np.argsort(ov[load])
    sim = np.interp(ref[:, 0] * 1e-6, ov[load][order], (f[load] / 1e3)[order], left=0.0)
    assert np.max(np.abs(sim - ref[:, 1])) < 0.03 * ref[:, 1].max()


@pytest.mark.parametrize("cor", [0.01, 0.2, 0.4, 0.6, 0.8, 1.0])
def test_example03_restitution_identity(example_inputs, cor):
    sc = S.example03(example_inputs["03_normal_particle_wall_different_cor"], cor)
    O.run(sc.state, sc.walls, sc.params, sc.dt, sc.nsteps, delta=sc.delta)
    out = sc.state.u[0, 1] / float(example_inputs["03_normal_particle_wall_different_cor"]["velocity_p"])
    assert abs(out - cor) < 0.02


def test_example04_rebound_spin_vs_angle(example_inputs, validation_data):
    angles = [2., 5., 10., 15., 20., 25., 30., 35., 40., 50., 55., 60., 65., 70.]  # automate.py:359-414
    om = []
    for a in angles:
        sc = S.example04(example_inputs["04_oblique_particle_wall_different_angles"], a)
        O.run(sc.state, sc.walls, sc.params, sc.dt, sc.nsteps, delta=sc.delta)
        om.append(sc.state.omega[0, 2])    # automate.py:447: omega[0][2]
    om = np.array(om)
    lethe = validation_data[T4_LETHE]
    exp = validation_data[T4_EXP]
    peak = lethe[:, 1].max()
    assert abs(om.max() - peak) < 0.05 * peak
    assert 25.0 <= angles[int(np.argmax(om))] <= 35.0
    sel = np.array(angles) >= 20.0
    lethe_at = np.interp(np.array(angles)[sel], lethe[:, 0], lethe[:, 1])
    assert np.max(np.abs(om[sel] - lethe_at)) < 0.10 * peak
    exp_sel = exp[:, 0] >= 20.0
    sim_at_exp = np.interp(exp[exp_sel, 0], angles, om)
    assert np.max(np.abs(sim_at_exp - exp[exp_sel, 1])) < 0.10 * exp[:, 1].max()


def test_tst03_contact_slots(example_inputs):
    """tst_03: sphere 0 strikes the offset pair 1, 2 (automate.py:531 reads the tracked
    contact counts).  Both partners are tracked at once, then released."""
    sc = S.tst03(example_inputs["tst_03_multiple_particles_contacts"])
    st = sc.state
    counts = []
    for _ in range(0, sc.nsteps, 10):
        O.run(st, sc.walls, sc.params, sc.dt, 10, delta=sc.delta)
        counts.append(st.tng_count.copy())
    counts = np.array(counts)
    assert counts[:, 0].max() == 2
    assert counts[-1].sum() == 0
    assert np.all(np.isfinite(st.x))
