"""GPU bonded DEM (bond build, fused bond force + integration, breakage) against the CPU
oracle's restatement of setupBonds / computeBondedForce on the same inputs.  FP64 results are
bit-identical (the oracle's pow(b,2.)/pow(b,4.) evaluated as products, the device arithmetic);
broken-bond counts are exact."""
import numpy as np
import pytest

from cabanadem_b200 import api, scenarios as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu

HIST = ("ft_x", "ft_y", "ft_z", "mn_x", "mn_y", "mn_z", "mt_x", "mt_y", "mt_z")


def _oracle(case, nsteps):
    st, b = case["state"].copy(), case["bonds"].copy()
    O.setup_bonds(b, st, case["bond_factor"], case["search_cutoff"])
    status = O.bonded_run(st, b, case["bparams"], case["dt"], nsteps, ext_force=case["ext_force"],
                          fix_flags=case["fix_flags"], pow_mode=O.POW_SQRT)
    return st, b, status


def _compare(bonds, st, b, where):
    p = bonds.solver.particles
    for f in ("x", "u", "omega", "force", "torque"):
        a, r = p.get(f), getattr(st, f)
        assert np.array_equal(a, r), (where, f, np.abs(a - r).max())
    assert np.array_equal(bonds.get("count"), b.count)
    assert np.array_equal(bonds.get("idx"), b.idx)
    assert np.array_equal(bonds.get("init_len"), b.init_len)
    assert np.array_equal(bonds.get("broken"), b.broken)
    for k in HIST:
        assert np.array_equal(bonds.get(k), b.hist[k]), (where, k)


def test_two_bonded_particles_reference_case():
    """tst_01_BDEM: two spheres pulled apart by +-1e3 N with the reference's own quirks
    (partner-indexed history, stiffness from E/G, vel_j from u_i)."""
    case = S.bdem_two_particles()
    n = 4001
    st, b, status = _oracle(case, n)
    bonds = api.bonded_from_case(case, steps_per_launch=64)
    bonds.run_steps(n)
    _compare(bonds, st, b, "tst01")
    assert b.count.tolist() == [1, 1]


def test_bonded_bar_breakage_bitwise():
    """A small bar pulled fast enough that bonds break inside the test window."""
    case = S.bonded_bar(nx=32, ny=8, nz=4, pull=5.0, nsteps=2000)
    st, b, status = _oracle(case, 2000)
    assert int(b.broken.sum()) > 0
    bonds = api.bonded_from_case(case)
    bonds.run_steps(2000)
    _compare(bonds, st, b, "bar")
    assert bonds.broken() == int(b.broken.sum())


def test_bonded_bar_full_size_bitwise():
    """Full 256x64x8 bar (131,072 spheres, ~390k bond ends... 6 per interior sphere): 30 steps."""
    case = S.bonded_bar()
    st, b, status = _oracle(case, 30)
    bonds = api.bonded_from_case(case)
    assert int(bonds.get("count").sum()) == int(b.count.sum())
    bonds.run_steps(30)
    _compare(bonds, st, b, "bar_full")


def test_bonded_mixed_precision_against_fp64():
    """FP32 bond force/moment history with FP64 strain: the broken-bond set is exact and the
    stress-strain record (axial force through the mid-plane, sampled along the pull) stays
    within 1e-4 of the FP64 path."""
    from cabanadem_b200._lib import DEM_MIXED

    def record(precision):
        case = S.bonded_bar(nx=32, ny=8, nz=4, pull=5.0, nsteps=2000)
        b = api.bonded_from_case(case, precision=precision)
        mid = case["state"].x[:, 0] < np.median(case["state"].x[:, 0])
        curve = []
        for _ in range(10):
            b.run_steps(200)
            f = b.solver.particles.get("force")
            curve.append(float(f[mid, 0].sum()))
        return np.asarray(curve), b.get("broken").copy(), b.solver.particles.get("x")

    c64, br64, x64 = record(0)
    c32, br32, x32 = record(DEM_MIXED)
    assert br64.sum() > 0
    assert np.array_equal(br64, br32)
    assert np.abs(c32 - c64).max() <= 1e-4 * np.abs(c64).max()
    assert np.abs(x32 - x64).max() <= 1e-8   # m, against r = 0.5 mm


def _phase_loop(bonds, dt, nsteps):
    """The reference's bonded loop phase by phase (tst_01_BDEM:295-306), through the C ABI."""
    it = bonds.solver.integrator
    for _ in range(nsteps):
        it.stage1()
        it.stage2()
        bonds.resetForcesAndTorques()
        bonds.applyExternalForce()
        bonds.computeBondedForce(dt)
        bonds.applyBoundaryConditions()
        it.stage3()


def test_bonded_phases_equal_the_oracle_and_the_fused_loop():
    """dem_bonded_reset, dem_apply_external_force, dem_bonded_force, dem_apply_boundary_conditions
    and the stages, called one by one on the breaking bar (pulled ends, breakage): every field
    and the bond slots bit-identical to the oracle and to the fused dem_bonded_run."""
    case = S.bonded_bar(nx=32, ny=8, nz=4, pull=5.0, nsteps=600)
    st, b, status = _oracle(case, 600)
    assert int(b.broken.sum()) > 0
    phased = api.bonded_from_case(case)
    _phase_loop(phased, case["dt"], 600)
    _compare(phased, st, b, "phases")
    fused = api.bonded_from_case(case)
    fused.run_steps(600)
    _compare(fused, st, b, "fused")


def test_bonded_phases_two_particle_reference_case():
    case = S.bdem_two_particles()
    st, b, status = _oracle(case, 1500)
    bonds = api.bonded_from_case(case)
    _phase_loop(bonds, case["dt"], 1500)
    _compare(bonds, st, b, "tst01 phases")


def test_bond_slices_upload_round_trip():
    """dem_bonds_set: every bond slice written back unchanged reads back bit for bit, a
    modified history acts in the next phase as in the oracle given the same history, and a
    partner index out of range is refused."""
    case = S.bonded_bar(nx=16, ny=4, nz=4, pull=5.0, nsteps=200)
    bonds = api.bonded_from_case(case)
    bonds.run_steps(100)
    before = {k: bonds.get(k) for k in ("idx", "count", "init_len", "broken") + HIST}
    for k, v in before.items():
        bonds.set(k, v)
    for k, v in before.items():
        assert np.array_equal(bonds.get(k), v), k
    # scale the tangential bond force history, then one more phase loop step on both sides
    st = bonds.solver.particles.download()
    ob = case["bonds"].copy()
    ob.idx[:], ob.count[:], ob.init_len[:], ob.broken[:] = before["idx"], before["count"], before["init_len"], before["broken"]
    for k in HIST:
        ob.hist[k][:] = before[k] * (1.5 if k.startswith("ft") else 1.0)
    bonds.set("ft_x", ob.hist["ft_x"])
    bonds.set("ft_y", ob.hist["ft_y"])
    bonds.set("ft_z", ob.hist["ft_z"])
    O.bonded_run(st, ob, case["bparams"], case["dt"], 1, ext_force=case["ext_force"], fix_flags=case["fix_flags"],
                 pow_mode=O.POW_SQRT)
    _phase_loop(bonds, case["dt"], 1)
    _compare(bonds, st, ob, "after set")
    bad = before["idx"].copy()
    bad[0, 0] = case["state"].n
    with pytest.raises(api.DemError):
        bonds.set("idx", bad)
