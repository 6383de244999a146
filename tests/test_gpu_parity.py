"""GPU parity: the fused FP64 step (libb200dem.so, called through its C ABI) against the CPU
oracle on the same seeded inputs.

With the oracle's pow handling set to the device arithmetic (x^1.5 = x*sqrt(x)), FP64
results must be bit-identical, including the contact slot layout.  Against the oracle's
libm pow (the reference's literal arithmetic) the bar is 1e-10 relative.
"""
import numpy as np
import pytest

from cabanadem_b200 import api, scenarios as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu

STATE_F = ("x", "u", "omega", "force", "torque")
HIST_F = ("tng_idx", "tng_ss_x", "tng_ss_y", "tng_ss_z", "tng_count")
WALL_F = ("tng_sw_x", "tng_sw_y", "tng_sw_z")


def _assert_bitwise(got, ref, fields=STATE_F + HIST_F + WALL_F, where=""):
    for f in fields:
        a, b = getattr(got, f), getattr(ref, f)
        if f.startswith("tng_sw"):
            a, b = a[:, : b.shape[1]], b[:, : a.shape[1]]
        if f in ("tng_idx", "tng_ss_x", "tng_ss_y", "tng_ss_z"):
            # slots beyond the count are not part of the state
            mask = np.arange(a.shape[1])[None, :] < ref.tng_count[:, None]
            a, b = np.where(mask, a, 0), np.where(mask, b, 0)
        if not np.array_equal(a, b):
            d = np.abs(np.asarray(a, float) - np.asarray(b, float))
            raise AssertionError("%s %s differs: max |d| = %g at %s" % (where, f, d.max(), np.unravel_index(d.argmax(), d.shape)))


def _rel_close(got, ref, tol, fields=STATE_F):
    for f in fields:
        a, b = getattr(got, f), getattr(ref, f)
        scale = max(np.abs(b).max(), 1e-300)
        err = np.abs(a - b).max() / scale
        assert err <= tol, (f, err)


def _gpu_run(sc, nsteps, rebuild_every_step, chunks=1, **kw):
    s = api.from_scenario(sc, rebuild_every_step=rebuild_every_step, **kw)
    per = nsteps // chunks
    for c in range(chunks):
        s.run_steps(per if c < chunks - 1 else nsteps - per * (chunks - 1))
    return s, s.particles.download()


def _oracle(sc, nsteps, pow_mode=O.POW_SQRT):
    ref = sc.state.copy()
    st = O.run(ref, sc.walls, sc.params, sc.dt, nsteps, delta=sc.delta, skin=sc.skin, gravity=sc.gravity,
               pow_mode=pow_mode)
    return ref, st


EXAMPLES = [
    ("example01", lambda I: S.example01(I["01_elastic_normal_impact_of_two_identical_particles"])),
    ("example02", lambda I: S.example02(I["02_elastic_normal_impact_of_particle_wall"])),
    ("example03_cor0.4", lambda I: S.example03(I["03_normal_particle_wall_different_cor"], 0.4)),
    ("example04_30deg", lambda I: S.example04(I["04_oblique_particle_wall_different_angles"], 30.0)),
    ("example04_60deg", lambda I: S.example04(I["04_oblique_particle_wall_different_angles"], 60.0)),
    ("tst03", lambda I: S.tst03(I["tst_03_multiple_particles_contacts"])),
]


@pytest.mark.parametrize("name,make", EXAMPLES, ids=[e[0] for e in EXAMPLES])
@pytest.mark.parametrize("ref_mode", [True, False], ids=["rebuild_every_step", "skin"])
def test_reference_examples_bitwise(example_inputs, name, make, ref_mode):
    sc = make(example_inputs)
    if not ref_mode:
        sc.delta, sc.skin = 0.0, 0.1 * float(sc.state.rad.max())
    n = min(sc.nsteps, 3001)
    ref, _ = _oracle(sc, n)
    _, got = _gpu_run(sc, n, ref_mode, chunks=3)
    _assert_bitwise(got, ref, where=name)


@pytest.mark.parametrize("name,make", EXAMPLES[:4], ids=[e[0] for e in EXAMPLES[:4]])
def test_reference_examples_vs_libm_pow(example_inputs, name, make):
    sc = make(example_inputs)
    ref, _ = _oracle(sc, sc.nsteps, pow_mode=O.POW_LIBM)
    _, got = _gpu_run(sc, sc.nsteps, True)
    _rel_close(got, ref, 1e-10)


@pytest.mark.parametrize("quirks", [S.REF_COMPAT, 0x00], ids=["ref_compat", "fixed"])
def test_random_box_bitwise(quirks):
    """4,096 spheres in a walled 5 cm cube, gravity, friction: 300 steps, denser start so
    that many contacts form (positions compressed towards the box centre)."""
    sc = S.random_box(n=4096, quirks=quirks, nsteps=300)
    c = sc.state.x.mean(axis=0)
    sc.state.x[:] = c + (sc.state.x - c) * 0.9       # overlapping start: many contacts at once
    sc.state.rad[:] = 1e-3
    ref, _ = _oracle(sc, 300)
    s, got = _gpu_run(sc, 300, False, chunks=2)
    assert ref.tng_count.sum() > 100
    _assert_bitwise(got, ref, where="random_box")
    st = s.stats()
    assert st["rebuilds"] >= 1


@pytest.mark.parametrize("lanes", [0, 1, 4, 8], ids=["auto", "per_thread", "coop4", "coop8"])
def test_contact_kernel_forms_bitwise(lanes):
    """The step's kernel forms against the oracle on a compressed box: contacts form, break
    (slot compaction moves histories between slots) and form again over 400 steps, against
    six walls.  Three-kernel step with the per-thread or the cooperative (4 or 8 lanes)
    contact kernel; auto: dense, so after the first graph one kernel steps every particle."""
    sc = S.random_box(n=4096, nsteps=400)
    c = sc.state.x.mean(axis=0)
    sc.state.x[:] = c + (sc.state.x - c) * 0.6
    ref, _ = _oracle(sc, 400)
    s = api.from_scenario(sc, contact_lanes=lanes)
    s.run_steps(150)
    mid = s.particles.download()
    assert mid.tng_count.sum() > 1000
    s.run_steps(250)
    _assert_bitwise(s.particles.download(), ref, where="lanes%d" % lanes)
    if lanes == 0:
        # the same trajectory (so the same rebuilds) with three kernels a step launches more
        t = api.from_scenario(sc, contact_lanes=1)
        t.run_steps(400)
        assert s.stats()["rebuilds"] == t.stats()["rebuilds"]
        assert s.stats()["launches"] < t.stats()["launches"] - 400


@pytest.mark.parametrize("packing", [1.0, 0.6], ids=["gas", "compressed"])
def test_pair_parallel_dense_step_bitwise(packing):
    """The pair-parallel step (contact search per particle, pair law per contact, sums per
    particle) forced at every density (dense_form 2): bit-identical to the oracle, slots and
    wall history included, over 1,200 steps of the compressed box (contacts form, break and
    move between slots; rebuilds) and of the C1 gas."""
    sc = S.random_box(n=4096, nsteps=1200)
    c = sc.state.x.mean(axis=0)
    sc.state.x[:] = c + (sc.state.x - c) * packing
    ref, _ = _oracle(sc, 1200)
    s = api.from_scenario(sc, dense_form=2)
    for n in (500, 700):
        s.run_steps(n)
    _assert_bitwise(s.particles.download(), ref, where="pairs")
    assert s.stats()["rebuilds"] >= 1


def test_pair_parallel_contact_overflow():
    """Slot overflow (MaxCnts 2) through the pair-parallel step: status bit and state as the oracle."""
    sc = S.random_box(n=512, max_cnts=2, nsteps=5)
    c = sc.state.x.mean(axis=0)
    sc.state.x[:] = c + (sc.state.x - c) * 0.3
    ref, st = _oracle(sc, 5)
    assert st & 0x1
    s = api.from_scenario(sc, dense_form=2)
    s.run_steps(5)
    assert s.last_status & 0x004
    _assert_bitwise(s.particles.download(), ref, where="pairs overflow")


@pytest.mark.parametrize("split", [1, 2, 3, 4], ids=["one_kernel", "two_kernels", "two_branches", "staged"])
@pytest.mark.parametrize("packing", [1.0, 0.7], ids=["gas", "compressed"])
def test_streaming_pass_forms_bitwise(split, packing):
    """The three-kernel step with each form of its streaming pass (one kernel; the particles
    without listed neighbours and the rest in two persistent kernels, in sequence or as
    concurrent graph branches; one persistent kernel over tiles staged in shared memory):
    bit-identical to the oracle over 1,500 steps with rebuilds, on the C1 gas (most particles
    without a listed neighbour) and on a compressed box.  4,133 particles: the last staged
    tile is a partial one."""
    sc = S.random_box(n=4133, nsteps=1500)
    c = sc.state.x.mean(axis=0)
    sc.state.x[:] = c + (sc.state.x - c) * packing
    ref, _ = _oracle(sc, 1500)
    # particles reach the walls (the staged kernel skips the wall test of those a build found
    # out of reach)
    assert ((ref.tng_sw_x != 0) | (ref.tng_sw_y != 0) | (ref.tng_sw_z != 0)).any()
    s = api.from_scenario(sc, contact_lanes=8, stream_split=split)
    for n in (700, 800):
        s.run_steps(n)
    _assert_bitwise(s.particles.download(), ref, where="split%d" % split)
    assert s.stats()["rebuilds"] >= 1


def test_staged_streaming_wait_that_runs_out_stops_the_run():
    """The staged streaming kernel's bounded waits: with dem_solver_debug_stream_waits(drop_copies=1)
    it arms its tile barriers but issues no copy, so every wait gives up after the poll limit with
    nothing in flight, and the run stops with DEM_ERR_TIMEOUT (no hang, no fault).  With the
    default bounds back and the state set again, the same solver steps bit-identically to the
    oracle: the context stayed usable."""
    from cabanadem_b200 import _lib
    sc = S.random_box(n=4133, nsteps=60)
    ref, _ = _oracle(sc, 60)
    s = api.from_scenario(sc, contact_lanes=8, stream_split=4)
    L = _lib.lib()
    assert L.dem_solver_debug_stream_waits(s.h, 64, 1) == 0
    try:
        with pytest.raises(_lib.DemError, match="DEM_ERR_TIMEOUT"):
            s.run_steps(5)
    finally:
        assert L.dem_solver_debug_stream_waits(s.h, 0, 0) == 0
    s.particles.upload(sc.state)
    s.run_steps(60)
    _assert_bitwise(s.particles.download(), ref, where="after a timed-out run")


@pytest.mark.parametrize("lanes", [0, 1, 8, "pairs"], ids=["auto", "per_thread", "coop8", "pairs"])
def test_moving_wall_bitwise(lanes):
    """A kinematic piston (DEM_Q6_WALL_STATIC clear) driven into a compressed box at 5 m/s,
    400 steps in three runs (each run's last step must not move the walls, its next run's
    first drift must): particles and wall positions bit-identical to the oracle.  "pairs" is
    the pair-parallel step, whose wall contacts are work items of their own."""
    sc = S.piston_box(n=4096, speed=5.0, nsteps=400)
    c = sc.state.x.mean(axis=0)
    sc.state.x[:] = c + (sc.state.x - c) * 0.8
    sc.walls.x[1, 0] = float((sc.state.x[:, 0] + sc.state.rad).max())   # touching the compressed box
    ref = sc.state.copy()
    w = sc.walls.copy()
    O.run(ref, w, sc.params, sc.dt, 400, skin=sc.skin, gravity=sc.gravity, pow_mode=O.POW_SQRT)
    s = api.from_scenario(sc, **(dict(dense_form=2) if lanes == "pairs" else dict(contact_lanes=lanes)))
    for n in (150, 101, 149):
        s.run_steps(n)
    _assert_bitwise(s.particles.download(), ref, where="piston%s" % lanes)
    assert np.array_equal(s.wall_positions(), w.x)
    assert w.x[1, 0] < sc.walls.x[1, 0]
    # particles in sliding contact with the piston (history tangential to its normal, -x)
    assert ((ref.tng_sw_y[:, 1] != 0) | (ref.tng_sw_z[:, 1] != 0)).any()


@pytest.mark.parametrize("lanes", [1, 8], ids=["per_thread", "coop8"])
def test_contact_overflow_all_kernels(lanes):
    """Slot overflow (MaxCnts 2) through either contact kernel: status bit and state as the oracle."""
    sc = S.random_box(n=512, max_cnts=2, nsteps=5)
    c = sc.state.x.mean(axis=0)
    sc.state.x[:] = c + (sc.state.x - c) * 0.3
    ref, st = _oracle(sc, 5)
    assert st & 0x1
    s = api.from_scenario(sc, contact_lanes=lanes)
    s.run_steps(5)
    assert s.last_status & 0x004
    _assert_bitwise(s.particles.download(), ref, where="overflow%d" % lanes)


def test_unfused_phases_match_fused(example_inputs):
    sc = S.tst03(example_inputs["tst_03_multiple_particles_contacts"])
    steps = 400
    _, fused = _gpu_run(sc, steps, True)
    s = api.from_scenario(sc, rebuild_every_step=True)
    for _ in range(steps):
        s.integrator.stage1()
        s.integrator.stage2()
        s.build_neighbors()
        api.computeForceParticleParticleInfiniteWall(s)
        s.integrator.stage3()
    _assert_bitwise(s.particles.download(), fused, where="unfused")


@pytest.mark.parametrize("chunk", [1, 16, 64])
def test_chunked_graphs_equal_the_loop_graph(chunk):
    """The step loop as a graph while-loop (steps_per_launch 0, the default) against graphs of
    a fixed number of gated steps: the same trajectory bit for bit, through rebuilds and the
    switch between the sparse and the dense kernel forms, and the oracle's."""
    sc = S.random_box(n=4096, nsteps=500)
    c = sc.state.x.mean(axis=0)
    sc.state.x[:] = c + (sc.state.x - c) * 0.75
    ref, _ = _oracle(sc, 500)
    a = api.from_scenario(sc, contact_lanes=0)
    b = api.from_scenario(sc, contact_lanes=0, steps_per_launch=chunk)
    for n in (123, 377):
        a.run_steps(n)
        b.run_steps(n)
    _assert_bitwise(a.particles.download(), ref, where="loop")
    _assert_bitwise(b.particles.download(), ref, where="chunk%d" % chunk)
    assert a.stats()["steps"] == b.stats()["steps"] == 500


def test_split_runs_equal_one_run():
    sc = S.random_box(n=2048, nsteps=200)
    _, one = _gpu_run(sc, 200, False, chunks=1)
    _, split = _gpu_run(sc, 200, False, chunks=7)
    _assert_bitwise(split, one, where="split")


def test_deterministic_repeat():
    sc = S.random_box(n=4096, nsteps=100)
    c = sc.state.x.mean(axis=0)
    sc.state.x[:] = c + (sc.state.x - c) * 0.55
    _, a = _gpu_run(sc, 100, False)
    _, b = _gpu_run(sc, 100, False)
    _assert_bitwise(a, b, where="repeat")


@pytest.mark.parametrize("delta", [0.0, 3e-3])
def test_neighbor_list_matches_oracle(delta):
    sc = S.random_box(n=4096)
    s = api.from_scenario(sc, rebuild_every_step=delta > 0)
    if delta > 0:
        s.close()
        sc.delta = delta
        s = api.from_scenario(sc, rebuild_every_step=True)
    s.build_neighbors()
    off, idx = s.neighbors()
    roff, ridx = O.neighbor_list(sc.state, delta=sc.delta, skin=sc.skin)
    assert np.array_equal(off, roff)
    assert np.array_equal(idx, ridx)


def test_contact_overflow_reported():
    """More overlapping partners than MaxCnts: the reference writes out of bounds
    (Force.hpp:186-188); here the extra contacts are not stored and the status says so,
    exactly as in the oracle."""
    sc = S.random_box(n=512, max_cnts=2, nsteps=5)
    c = sc.state.x.mean(axis=0)
    sc.state.x[:] = c + (sc.state.x - c) * 0.3
    ref, st = _oracle(sc, 5)
    assert st & 0x1
    s = api.from_scenario(sc)
    s.run_steps(5)
    assert s.last_status & 0x004
    _assert_bitwise(s.particles.download(), ref, where="overflow")


def test_energy_matches_oracle():
    sc = S.random_box(n=4096, nsteps=50)
    s, got = _gpu_run(sc, 50, False)
    e = s.energy()
    assert abs(e[0] + e[1] - O.kinetic_energy(got)) <= 1e-12 * O.kinetic_energy(got)
    assert np.array_equal(e, s.energy())


def test_set_get_roundtrip_after_resort():
    sc = S.random_box(n=4096, nsteps=10)
    s, _ = _gpu_run(sc, 10, False)
    p = s.particles
    x = p.get("x")
    u = np.random.default_rng(5).normal(size=x.shape)
    p.set("u", u)
    assert np.array_equal(p.get("u"), u)
    buf = np.empty_like(u)
    assert p.get("u", out=buf) is buf and np.array_equal(buf, u)
    assert np.array_equal(p.get("rad"), sc.state.rad)


def test_hcp_full_size_one_step_bitwise():
    """Full benchmark size (2,000,000 spheres): 2 fused steps bit-identical to the oracle."""
    sc = S.hcp_box()
    ref, _ = _oracle(sc, 2)
    _, got = _gpu_run(sc, 2, False)
    _assert_bitwise(got, ref, fields=STATE_F + ("tng_count",), where="hcp")


def test_checkpoint_restart_continues_bitwise(tmp_path):
    """Save after 300 steps, load into fresh particles, continue 300 more: identical to the
    uninterrupted run (the list is rebuilt, sums run in caller order)."""
    sc = S.random_box(n=1024, seed=5)
    a = api.from_scenario(sc)
    a.run_steps(300)
    path = tmp_path / "state.b200dem"
    a.particles.save(path)
    a.run_steps(300)
    b = api.from_scenario(S.random_box(n=1024, seed=5))
    b.particles.load(path)
    b.run_steps(300)
    sa, sb = a.particles.download(), b.particles.download()
    for f in ("x", "u", "omega", "force", "torque", "tng_idx", "tng_count", "tng_ss_x", "tng_sw_y"):
        assert np.array_equal(getattr(sa, f), getattr(sb, f)), f


def test_checkpoint_load_of_a_truncated_file_changes_nothing(tmp_path):
    """A checkpoint cut short in its last field is refused with DEM_ERR_INVALID, and the
    particles keep every field they had before the call."""
    sc = S.random_box(n=512, seed=6)
    a = api.from_scenario(sc)
    a.run_steps(200)
    path = tmp_path / "state.b200dem"
    a.particles.save(path)
    data = path.read_bytes()
    path.write_bytes(data[:-16])
    b = api.from_scenario(S.random_box(n=512, seed=6))
    before = b.particles.download()
    with pytest.raises(api.DemError):
        b.particles.load(path)
    after = b.particles.download()
    for f in ("x", "u", "omega", "rad", "tng_idx", "tng_count", "tng_ss_x", "tng_sw_y"):
        assert np.array_equal(getattr(before, f), getattr(after, f)), f


@pytest.mark.parametrize("quirks", [0, S.REF_COMPAT], ids=["all_clear", "ref"])
def test_sliding_sphere_on_floor(quirks):
    """A glass sphere launched along a floor at 1 m/s without spin: wall friction through the
    sliding phase into rolling, with the tangential damping on (every quirk clear: the wall law
    applies its Coulomb-limited force) and off (the reference), bit for bit with the oracle."""
    from cabanadem_b200.state import ParticleState, WallState
    r, rho, E, nu = 0.01, 2600.0, 70e9, 0.25
    s = ParticleState.create(1, max_cnts=6, max_walls=1)
    s.rad[:], s.rho[:], s.E[:], s.nu[:] = r, rho, E, nu
    s.G[:] = E / (2.0 * (1.0 + nu))
    s.set_sphere_mass()
    s.x[0, 2] = r - (s.m[0] * 9.81 / (4.0 / 3.0 * E / (2.0 * (1.0 - nu * nu)) * np.sqrt(r))) ** (2.0 / 3.0)
    s.u[0, 0] = 1.0
    w = WallState.create(1)
    w.normal[0, 2] = 1.0
    w.E[:], w.nu[:], w.G[:] = E, nu, s.G[0]
    sc = S.Scenario("sliding_sphere", s, w, S._force_params(0.5, 0.5, 0.5, 0.5, quirks), 1e-6, 3000,
                    skin=0.1 * r, gravity=(0.0, 0.0, -9.81))
    ref = s.copy()
    assert O.run(ref, w.copy(), sc.params, sc.dt, 3000, skin=sc.skin, gravity=sc.gravity, pow_mode=O.POW_SQRT) == 0
    g = api.from_scenario(sc)
    g.run_steps(3000)
    _assert_bitwise(g.particles.download(), ref, where="sliding%d" % quirks)
    assert ref.u[0, 0] < 1.0 - 0.5 * 9.81 * 2e-3        # slowing down by friction


def test_uploads_from_pinned_memory_equal_pageable_ones():
    """A set from page-locked host memory is queued on the stream without waiting (the ping-pong
    buffer it writes is picked on the device): a run after such uploads, and reads into pinned
    buffers, give the same bits as the same calls with ordinary arrays."""
    import torch
    sc = S.random_box(n=4133, nsteps=200)
    outs = []
    for pinned in (False, True):
        s = api.from_scenario(sc, contact_lanes=8)
        s.run_steps(37)                    # an odd count: the current buffers are the second ones
        keep = []
        for f in ("rad", "x", "u", "omega", "m", "I"):
            a = np.ascontiguousarray(getattr(sc.state, f))
            if pinned:
                t = torch.from_numpy(a.copy()).pin_memory()
                keep.append(t)
                a = t.numpy()
            s.particles.set(f, a)
        s.particles.clear_contacts()
        s.particles.clear_forces()
        s.run_steps(150)
        got = {}
        for f in ("x", "u", "omega", "force", "torque", "tng_count"):
            ref = s.particles.get(f)
            if pinned:
                buf = torch.empty(ref.shape, dtype=torch.from_numpy(ref).dtype).pin_memory()
                got[f] = s.particles.get(f, out=buf.numpy()).copy()
            else:
                got[f] = ref
        outs.append(got)
        s.close()
    for f in outs[0]:
        assert np.array_equal(outs[0][f], outs[1][f]), f


@pytest.mark.parametrize("form", ["staged", "pairs", "one_kernel", "mixed_coop", "chunked"])
def test_dependent_launches_equal_plain_stream_order(form):
    """Every kernel of a step launched as the programmatic dependent of the kernel before it
    (launch_overlap 0, the default: its launch overlaps that kernel's tail, and it waits for
    that kernel's completion before it touches any state) against plain stream order
    (launch_overlap 2): the same trajectory bit for bit through rebuilds, for the three-kernel
    step with the staged streaming pass, the pair-parallel step, the one-kernel dense step, the
    mixed-precision cooperative step and graphs of a fixed number of steps; FP64 forms also
    against the oracle."""
    from cabanadem_b200._lib import DEM_MIXED
    sc = S.random_box(n=4133, nsteps=600)
    c = sc.state.x.mean(axis=0)
    sc.state.x[:] = c + (sc.state.x - c) * (0.6 if form == "one_kernel" else 0.7)
    kw = {"staged": dict(contact_lanes=8, stream_split=4), "pairs": dict(dense_form=2), "one_kernel": dict(),
          "mixed_coop": dict(contact_lanes=8, precision=DEM_MIXED),
          "chunked": dict(contact_lanes=8, steps_per_launch=16)}[form]
    a = api.from_scenario(sc, **kw)
    b = api.from_scenario(sc, launch_overlap=2, **kw)
    for n in (250, 350):
        a.run_steps(n)
        b.run_steps(n)
    got = a.particles.download()
    _assert_bitwise(got, b.particles.download(), where="overlap %s" % form)
    assert a.stats()["rebuilds"] == b.stats()["rebuilds"] >= 1
    if form != "mixed_coop":
        ref, _ = _oracle(sc, 600)
        _assert_bitwise(got, ref, where="overlap %s vs oracle" % form)
    assert a.stats()["launch_overlap"] == 1 and b.stats()["launch_overlap"] == 0


@pytest.mark.parametrize("case", ["gas", "compressed", "piston", "mixed", "overflow"])
def test_cooperative_step_loop_equals_graph_loop(case):
    """The one-kernel step of a small system with a run's steps in one cooperative launch and a
    grid barrier between steps (cooperative_loop 0, the default) against graph replays of the
    per-step kernel (cooperative_loop 2): the same trajectory bit for bit through rebuilds,
    runs split unevenly, a kinematic piston (each run's last step leaves the walls, the next
    run's first drift moves them), mixed precision and contact-slot overflow (MaxCnts 2), and
    the oracle's in FP64."""
    from cabanadem_b200._lib import DEM_MIXED
    if case == "piston":
        sc = S.piston_box(n=4096, speed=5.0, nsteps=400)
        c = sc.state.x.mean(axis=0)
        sc.state.x[:] = c + (sc.state.x - c) * 0.8
        sc.walls.x[1, 0] = float((sc.state.x[:, 0] + sc.state.rad).max())
    else:
        sc = S.random_box(n=4133, nsteps=400, **(dict(max_cnts=2) if case == "overflow" else {}))
        c = sc.state.x.mean(axis=0)
        sc.state.x[:] = c + (sc.state.x - c) * (1.0 if case == "gas" else 0.6)
    kw = dict(precision=DEM_MIXED) if case == "mixed" else {}
    a = api.from_scenario(sc, **kw)
    b = api.from_scenario(sc, cooperative_loop=2, **kw)
    for n in (150, 101, 149):
        a.run_steps(n)
        b.run_steps(n)
    got = a.particles.download()
    _assert_bitwise(got, b.particles.download(), where="coop %s" % case)
    sa, sb = a.stats(), b.stats()
    assert sa["cooperative_loop"] == 1 and sb["cooperative_loop"] == 0
    assert sa["rebuilds"] == sb["rebuilds"] and sa["steps"] == sb["steps"] == 400
    assert sa["launches"] < sb["launches"]
    assert a.last_status == b.last_status
    if case == "overflow":
        assert a.last_status & 0x004
    if case == "piston":
        assert np.array_equal(a.wall_positions(), b.wall_positions())
    if case != "mixed":
        ref = sc.state.copy()
        w = sc.walls.copy()
        O.run(ref, w, sc.params, sc.dt, 400, skin=sc.skin, gravity=sc.gravity, pow_mode=O.POW_SQRT)
        _assert_bitwise(got, ref, where="coop %s vs oracle" % case)
        if case == "piston":
            assert np.array_equal(a.wall_positions(), w.x)
