"""Slab decomposition (cabanadem_b200/slabs.py) on CPU gloo ranks, the oracle stepping each
rank's local set: a gas of soft spheres in a walled box, decomposed over 1, 2 and 3 slabs
along x (and over 2 slabs with a kinematic piston wall), is bit-identical to the
undecomposed oracle run (positions, velocities, forces, torques, contact counts, live
tangential history with partners as global ids, wall history).
The run has particles that change slabs and contacts across slab faces, so both the
migration and the ghost exchange are exercised.  A halo too thin for the step's drift makes
every rank raise together instead of leaving one waiting."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RADIUS, SIDE, STEPS, DT = 1e-3, 0.02, 600, 2e-6
HALO = 2.0 * RADIUS + 1e-4
LO = -1e-3      # slab faces off the lattice planes, within reach of the moving spheres


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _gas(seed=5, piston=0.0):
    """8 x 8 x 8 spheres of r = 1 mm on a 2.5 mm lattice with 0.1 mm jitter, velocities
    U[-1, 1] m/s, E = 5 MPa (contacts last about 130 steps of 2 us), six walls, gravity.
    piston > 0: the +x wall moves inwards at that speed (DEM_Q6_WALL_STATIC clear)."""
    import sys
    sys.path.insert(0, ROOT)
    from cabanadem_b200.scenarios import Q6_WALL_STATIC, REF_COMPAT, _box_walls, _force_params
    from cabanadem_b200.state import ParticleState
    rng = np.random.default_rng(seed)
    g = (np.arange(8) + 0.5) * 2.5e-3
    pos = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    pos += rng.uniform(-1e-4, 1e-4, size=pos.shape)
    s = ParticleState.create(len(pos), max_cnts=12, max_walls=6)
    s.x[:] = pos
    s.u[:] = rng.uniform(-1.0, 1.0, size=pos.shape)
    s.rad[:] = RADIUS
    s.rho[:] = 2500.0
    s.set_sphere_mass()
    s.E[:], s.nu[:] = 5e6, 0.3
    s.G[:] = s.E / (2.0 * (1.0 + s.nu))
    w = _box_walls((0.0, 0.0, 0.0), (SIDE, SIDE, SIDE), 5e6, 0.3, float(s.G[0]))
    if piston:
        w.u[1, 0] = -piston
        return s, w, _force_params(0.7, 0.7, 0.3, 0.3, REF_COMPAT & ~Q6_WALL_STATIC)
    return s, w, _force_params(0.7, 0.7, 0.3, 0.3)


def _oracle_step(walls, params):
    from oracle import oracle as O

    def step(st):
        status = O.run(st, walls, params, DT, 1, skin=0.1 * RADIUS, gravity=(0.0, 0.0, -9.81), pow_mode=O.POW_SQRT)
        assert status == 0
    return step


class _HostApi:
    """Stand-in for cabanadem_b200.api with the calls DeviceStep makes and the same host-side
    semantics (upload of the first MaxNoWalls wall-history columns, download into a state with
    max(MaxNoWalls, 1) columns, solver-owned wall positions), the oracle taking the step: it
    checks DeviceStep's glue on the CPU."""
    REF_COMPAT = 0x3F

    @staticmethod
    def default_context():
        return None

    class Force:
        def __init__(self, cor_pp, cor_pw, mu_pp, mu_pw, quirks):
            self.params = dict(cor_pp=cor_pp, cor_pw=cor_pw, mu_pp=mu_pp, mu_pw=mu_pw, quirks=quirks)

    class Particles:
        def __init__(self, n, max_cnts, max_walls, ctx=None):
            from cabanadem_b200._lib import DemError
            from cabanadem_b200.state import ParticleState
            if n <= 0:       # dem_particles_create: n > 0
                raise DemError("dem_particles_create: n > 0")
            self.mw = max_walls
            self.st = ParticleState.create(n, max_cnts, max(max_walls, 1))

        def upload(self, s):
            for k, v in s.arrays().items():
                if k.startswith("tng_sw_"):
                    getattr(self.st, k)[:, : self.mw] = v[:, : self.mw]
                else:
                    getattr(self.st, k)[...] = v

        def download(self):
            return self.st.copy()

        def close(self):
            self.st = None

    class Wall:
        def __init__(self, n, ctx=None):
            self.w = None

        def upload(self, w):
            self.w = w.copy()

        def close(self):
            self.w = None

    class SolverDEM:
        def __init__(self, p, w, force, dt, delta=0.0, skin=0.0, gravity=(0.0, 0.0, 0.0)):
            self.p, self.w, self.f = p, w, force
            self.dt, self.delta, self.skin, self.g = dt, delta, skin, gravity

        def run_steps(self, n):
            from oracle import oracle as O
            assert O.run(self.p.st, self.w.w, self.f.params, self.dt, n, delta=self.delta, skin=self.skin,
                         gravity=self.g, pow_mode=O.POW_SQRT) == 0

        def wall_positions(self):
            return self.w.w.x.copy()

        def close(self):
            pass


def _rank(rank, world, port, out, halo, piston, glue=False, hi=SIDE):
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from cabanadem_b200._lib import DemError
    from cabanadem_b200.slabs import SlabDecomposition
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s, w, prm = _gas(piston=piston)
        dec = SlabDecomposition(0, LO, hi, halo, s.max_cnts, 6)
        dec.scatter(s)
        if glue:
            from cabanadem_b200.slabs import DeviceStep
            step = DeviceStep(w, prm, DT, skin=0.1 * RADIUS, gravity=(0.0, 0.0, -9.81),
                              api=None if glue == "device" else _HostApi)
        else:
            step = _oracle_step(w.copy(), prm)
        cross, ghosts = 0, 0
        try:
            for _ in range(STEPS):
                dec.step(step)
                gid = dec.rows[:, 0].astype(np.int64)
                a, k = dec.cols["tng_idx"]
                part = dec.rows[:, a:a + k]
                cross += int(np.sum((part >= 0) & ~np.isin(part, gid)))
                ghosts = max(ghosts, dec.ghosts)
        except DemError as e:
            out[rank] = ("error", str(e))
            return
        ke = dec.kinetic_energy()
        g = dec.gather()
        out[rank] = ("ok", dec.migrated, cross, ghosts, g, ke)
    finally:
        dist.destroy_process_group()


def _spawn(world, halo=HALO, piston=0.0, glue=False, hi=SIDE):
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out, halo, piston, glue, hi)) for r in range(world)]
    # one OpenMP thread per rank, set before the children start: the runtime reads it when
    # it is first loaded, which happens while the child imports torch
    old = os.environ.get("OMP_NUM_THREADS")
    os.environ["OMP_NUM_THREADS"] = "1"
    try:
        for p in procs:
            p.start()
    finally:
        if old is None:
            del os.environ["OMP_NUM_THREADS"]
        else:
            os.environ["OMP_NUM_THREADS"] = old
    for p in procs:
        p.join(300)
    for p in procs:
        if p.exitcode is None:
            p.kill()
        assert p.exitcode == 0
    return dict(out)


def _reference(piston=0.0):
    from oracle import oracle as O
    s, w, prm = _gas(piston=piston)
    st = O.run(s, w, prm, DT, STEPS, skin=0.1 * RADIUS, gravity=(0.0, 0.0, -9.81), pow_mode=O.POW_SQRT)
    assert st == 0
    return s


@pytest.mark.parametrize("world,piston", [(1, 0.0), (2, 0.0), (3, 0.0), (2, 0.5)],
                         ids=["1", "2", "3", "2_piston"])
def test_slab_decomposition_is_bitwise_single_domain(world, piston):
    out = _spawn(world, piston=piston)
    assert all(out[r][0] == "ok" for r in range(world)), out
    got = out[0][4]
    ref = _reference(piston)
    for f in ("x", "u", "omega", "force", "torque", "tng_count"):
        assert np.array_equal(getattr(got, f), getattr(ref, f)), f
    from oracle import oracle as O
    ke = O.kinetic_energy(ref)
    assert len({out[r][5] for r in range(world)}) == 1                  # every rank has the same total
    assert abs(out[0][5] - ke) <= 1e-12 * ke
    live = np.arange(ref.max_cnts)[None, :] < ref.tng_count[:, None]
    assert live.sum() > 100                       # a contact-rich run
    for f in ("tng_idx", "tng_ss_x", "tng_ss_y", "tng_ss_z"):
        assert np.array_equal(getattr(got, f)[live], getattr(ref, f)[live]), f
    for f in ("tng_sw_x", "tng_sw_y", "tng_sw_z"):
        assert np.array_equal(getattr(got, f), getattr(ref, f)), f
    if piston:
        assert not np.array_equal(got.u, _reference(0.0).u)  # the moving wall changed the run
    if world > 1:
        assert sum(out[r][1] for r in range(world)) > 0      # particles changed slabs
        assert sum(out[r][2] for r in range(world)) > 0      # contacts across a slab face
        assert all(out[r][3] > 0 for r in range(world))      # every rank held ghosts


def test_thin_halo_fails_on_every_rank():
    """halo = 2 r exactly leaves no room for the drift: the first step's check fails and both
    ranks raise (no rank is left waiting in an exchange)."""
    out = _spawn(2, halo=2.0 * RADIUS)
    assert [out[r][0] for r in range(2)] == ["error", "error"], out
    assert any("moved more than" in out[r][1] for r in range(2))


@pytest.mark.parametrize("world,hi", [(2, SIDE), (3, 2 * SIDE + 1e-3)], ids=["2", "3_empty_slab"])
def test_device_step_glue_with_host_stand_in(world, hi):
    """DeviceStep's upload / step / download / wall-carry logic, the device calls replaced by
    the host stand-in: slabs with the piston wall stay bit-identical to the oracle run (with
    3 ranks the third slab is empty and never creates a particle set)."""
    out = _spawn(world, piston=0.5, glue="host", hi=hi)
    assert all(out[r][0] == "ok" for r in range(world)), out
    got, ref = out[0][4], _reference(0.5)
    for f in ("x", "u", "omega", "force", "torque", "tng_count", "tng_sw_y", "tng_sw_z"):
        assert np.array_equal(getattr(got, f), getattr(ref, f)), f


def test_empty_slab():
    """Slabs over [-1 mm, 41 mm] with 3 ranks: the third slab (27-41 mm) holds no particle
    and skips its steps; the result is still the single-domain run's."""
    out = _spawn(3, hi=2 * SIDE + 1e-3)
    assert all(out[r][0] == "ok" for r in range(3)), out
    got, ref = out[0][4], _reference()
    for f in ("x", "u", "omega", "force", "torque", "tng_count"):
        assert np.array_equal(getattr(got, f), getattr(ref, f)), f


@pytest.mark.gpu
def test_device_step_two_ranks_on_the_gpu():
    """DeviceStep with the device library: two gloo ranks, each stepping its slab (owned
    particles and ghosts) on the GPU through the public API, the ghost exchange and migration
    on the host between steps (the ranks' kernels never wait on one another).  With the piston
    wall, 600 steps: bit-identical to the undecomposed run (the oracle's, which the GPU
    matches bit for bit), contact history and wall history included."""
    out = _spawn(2, piston=0.5, glue="device")
    assert all(out[r][0] == "ok" for r in range(2)), out
    got, ref = out[0][4], _reference(0.5)
    for f in ("x", "u", "omega", "force", "torque", "tng_count", "tng_sw_x", "tng_sw_y", "tng_sw_z"):
        assert np.array_equal(getattr(got, f), getattr(ref, f)), f
    live = np.arange(ref.max_cnts)[None, :] < ref.tng_count[:, None]
    for f in ("tng_idx", "tng_ss_x", "tng_ss_y", "tng_ss_z"):
        assert np.array_equal(getattr(got, f)[live], getattr(ref, f)[live]), f
    assert sum(out[r][1] for r in range(2)) > 0 and sum(out[r][2] for r in range(2)) > 0
