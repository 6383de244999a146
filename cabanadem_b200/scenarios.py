"""Scenario builders: the reference's example set-ups and the seeded benchmark workloads.

Each builder returns a :class:`Scenario` (initial particle/wall state plus force model,
time step, step count and neighbour parameters).  The example builders restate the
init functors of the reference's example programs (file:line cited per function); the
workload builders generate seeded synthetic inputs with the shapes, sizes and value
distributions of the benchmark configurations:

* ``random_box``      4,096 monodisperse spheres, rejection sampled in a 5 cm walled cube
* ``hcp_box``         2,000,000 polydisperse spheres on a jittered HCP lattice
* ``bonded_bar``      256x64x8 simple-cubic bonded bar pulled at both ends
* ``batched_scenes``  1,024 independent clusters fired at one wall each
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .inputs import Inputs
from .state import BondState, ParticleState, WallState

# Reference quirk flags (bit set = reproduce the reference's behaviour).
Q1_VELJ_USES_UI = 0x01
Q2_ETA_T_ZERO = 0x02
Q3_NO_PP_TORQUE = 0x04
Q4_UNIT_HISTORY = 0x08
Q5_WALL_FT_TYPO = 0x10
Q6_WALL_STATIC = 0x20
REF_COMPAT = 0x3F


@dataclass
class Scenario:
    name: str
    state: ParticleState
    walls: WallState
    params: dict
    dt: float
    nsteps: int
    delta: float = 0.0          # uniform neighbour cutoff (reference: 3 r); 0 = per-pair r_i + r_j + skin
    skin: float = 0.0
    gravity: tuple = (0.0, 0.0, 0.0)
    output_frequency: int = 0
    extra: dict = field(default_factory=dict)


def _force_params(cor_pp, cor_pw, mu_pp, mu_pw, quirks=REF_COMPAT):
    return dict(cor_pp=float(cor_pp), cor_pw=float(cor_pw), mu_pp=float(mu_pp), mu_pw=float(mu_pw),
                quirks=int(quirks))


def _material(state, inp, prefix="particle_"):
    state.rho[:] = inp[prefix + "density"]
    state.rad[:] = inp[prefix + "radius"]
    state.E[:] = inp[prefix + "youngs_modulus"]
    state.G[:] = inp[prefix + "shear_modulus"]
    state.nu[:] = inp[prefix + "poissons_ratio"]
    _mass(state, float(inp[prefix + "radius"]), float(inp[prefix + "density"]))


def _mass(state, radius, rho):
    # examples/01_elastic_normal_impact_of_two_identical_particles.cpp:106-107 (scalar form)
    m_p_i = 4. / 3. * math.pi * radius * radius * radius * rho
    I_p_i = 2. / 5. * m_p_i * radius * radius
    state.m[:] = m_p_i
    state.I[:] = I_p_i


def _one_wall(inp, x, normal):
    w = WallState.create(1)
    w.x[0] = x
    w.normal[0] = normal
    w.E[0] = inp["wall_youngs_modulus"]
    w.G[0] = inp["wall_shear_modulus"]
    w.nu[0] = inp["wall_poissons_ratio"]
    return w


def example01(inp: Inputs) -> Scenario:
    """examples/01_elastic_normal_impact_of_two_identical_particles.cpp:103-188."""
    r, v = float(inp["particle_radius"]), float(inp["velocity_p"])
    s = ParticleState.create(2, max_cnts=6, max_walls=1)
    _material(s, inp)
    for pid in range(2):
        s.x[pid, 0] = -r + pid * (2. * r) + pid * r / 100.
    s.u[0, 0], s.u[1, 0] = v, -v
    w = _one_wall(inp, (0., -3. * r, 0.), (0., 1., 0.))
    fp = _force_params(inp["coefficient_of_restitution_pp"], inp["coefficient_of_restitution_pw"],
                       inp["friction_pp"], inp["friction_pw"])
    return Scenario("example01", s, w, fp, float(inp["timestep"]), inp["num_steps"] + 1, delta=3. * r,
                    output_frequency=int(inp["output_frequency"]))


def _single_over_wall(inp, name, ux, uy, cor_pw=None):
    r = float(inp["particle_radius"])
    s = ParticleState.create(1, max_cnts=6, max_walls=1)
    _material(s, inp)
    s.x[0, 1] = r + r / 1000000.
    s.u[0, 0], s.u[0, 1] = ux, uy
    w = _one_wall(inp, (0., 0., 0.), (0., 1., 0.))
    fp = _force_params(inp["coefficient_of_restitution_pp"],
                       cor_pw if cor_pw is not None else inp["coefficient_of_restitution_pw"],
                       inp["friction_pp"], inp["friction_pw"])
    return Scenario(name, s, w, fp, float(inp["timestep"]), inp["num_steps"] + 1, delta=3. * r,
                    output_frequency=int(inp["output_frequency"]))


def example02(inp: Inputs) -> Scenario:
    """examples/02_elastic_normal_impact_of_particle_wall.cpp:99-171."""
    return _single_over_wall(inp, "example02", 0.0, -float(inp["velocity_p"]))


def example03(inp: Inputs, cor_pw: float) -> Scenario:
    """examples/03_normal_particle_wall_different_cor.cpp:105-174 (cor_pw from --cor_pw=)."""
    return _single_over_wall(inp, "example03", 0.0, -float(inp["velocity_p"]), cor_pw=cor_pw)


def example04(inp: Inputs, incident_angle: float) -> Scenario:
    """examples/04_oblique_particle_wall_different_angles.cpp:117-195 (angle from --angle=)."""
    angle = incident_angle / 180. * math.pi
    v = float(inp["velocity_p"])
    return _single_over_wall(inp, "example04", v * math.sin(angle), -v * math.cos(angle))


def tst03(inp: Inputs) -> Scenario:
    """examples/tst_03_multiple_particles_contacts.cpp:103-193 (wall normal is zero)."""
    r, v = float(inp["particle_radius"]), float(inp["velocity_p"])
    s = ParticleState.create(3, max_cnts=6, max_walls=1)
    _material(s, inp)
    for pid in range(3):
        s.x[pid, 0] = -r + pid * (2. * r) + pid * r / 100.
        s.x[pid, 1] = 0.
        if pid == 1:
            s.x[pid, 0] = -r + 1 * (1.5 * r) + 1 * r / 100.
            s.x[pid, 1] = r + r / 2.
        if pid == 2:
            s.x[pid, 0] = -r + 1 * (1.5 * r) + 1 * r / 100.
            s.x[pid, 1] = - r - r / 2.
    s.u[0, 0] = v
    w = _one_wall(inp, (0., -3. * r, 0.), (0., 0., 0.))
    fp = _force_params(inp["coefficient_of_restitution_pp"], inp["coefficient_of_restitution_pw"],
                       inp["friction_pp"], inp["friction_pw"])
    return Scenario("tst03", s, w, fp, float(inp["timestep"]), inp["num_steps"] + 1, delta=3. * r,
                    output_frequency=int(inp["output_frequency"]))


def tst04_points(length=1.0, height=1.0, spacing=0.1):
    """Zigzag lattice of examples/tst_04_granular_dam_break_2d.cpp:14-52 (create_points): rows
    and columns int(extent / spacing), odd rows shifted by half a spacing, points inside the
    rectangle kept in row-major order."""
    cols, rows = int(length / spacing), int(height / spacing)
    pts = []
    for i in range(rows):
        off = 0.0 if i % 2 == 0 else spacing / 2.0
        for j in range(cols):
            x, y = j * spacing + off, i * spacing
            if x <= length and y <= height:
                pts.append((x, y))
    return np.array(pts, dtype=np.float64).reshape(-1, 2)


def tst04(inp: Inputs, box_walls: bool = False) -> Scenario:
    """examples/tst_04_granular_dam_break_2d.cpp:120-267.  The reference sets a left wall, a
    floor and a right wall (:189-222) and then overwrites all three in its wall functor
    (:224-248): every wall at (0, -3 r, 0) with a zero normal, i.e. inert.  box_walls=True keeps
    the three walls as first set.  Three wall-history slots per particle (the reference declares
    one for its three walls)."""
    r = float(inp["particle_radius"])
    pts = tst04_points(1.0, 1.0, 2.0 * r)
    s = ParticleState.create(len(pts), max_cnts=6, max_walls=3)
    _material(s, inp)
    s.x[:, 0], s.x[:, 1] = pts[:, 0], pts[:, 1]
    w = WallState.create(3)
    if box_walls:
        w.x[:] = [(-2. * r, 0.5, 0.), (0.8, 0., 0.), (1.4, 0.5, 0.)]
        w.normal[:] = [(1., 0., 0.), (0., 1., 0.), (-1., 0., 0.)]
    else:
        w.x[:] = (0., -3. * r, 0.)
    w.E[:] = inp["wall_youngs_modulus"]
    w.G[:] = inp["wall_shear_modulus"]
    w.nu[:] = inp["wall_poissons_ratio"]
    fp = _force_params(inp["coefficient_of_restitution_pp"], inp["coefficient_of_restitution_pw"],
                       inp["friction_pp"], inp["friction_pw"])
    return Scenario("tst04", s, w, fp, float(inp["timestep"]), inp["num_steps"] + 1, delta=3. * r,
                    output_frequency=int(inp["output_frequency"]))


def bonded_bar(nx=256, ny=64, nz=8, radius=0.5e-3, pull=0.05, dt=2e-8, nsteps=50_000, kn=1e7, kt=4e6,
               break_strain=0.01, max_bonds=8, bond_quirks=0x04):
    """Simple-cubic bar of nx*ny*nz spheres (r = 0.5 mm, pitch 1 mm), every pair within
    1.05 diameters bonded (normal stiffness 1e7 N/m, shear 4e6 N/m, bond radius 0.5 r,
    breakage at 1% strain).  The two end layers along x move apart at +-0.05 m/s (force and
    torque zeroed each step); dt = 2e-8 s, 50,000 steps.  Bond history is slot-indexed and the
    stiffness explicit (the reference's partner-indexed history and hard-coded stiffness,
    BondedDEM_Force.hpp:186-207, do not define this case); vel_j keeps the reference's form."""
    n = nx * ny * nz
    k = np.arange(n)
    ix, iy, iz = k % nx, (k // nx) % ny, k // (nx * ny)
    pitch = 2.0 * radius
    s = ParticleState.create(n, max_cnts=1, max_walls=1)
    s.x[:, 0], s.x[:, 1], s.x[:, 2] = (ix + 0.5) * pitch, (iy + 0.5) * pitch, (iz + 0.5) * pitch
    _apply_glass(s, radius)
    fix = np.zeros(n, dtype=np.uint8)
    left, right = ix == 0, ix == nx - 1
    fix[left | right] = 0x3
    s.u[left, 0], s.u[right, 0] = -pull, pull
    b = BondState.create(n, max_bonds)
    return dict(state=s, bonds=b, dt=dt, nsteps=nsteps, ext_force=None, fix_flags=fix, bond_factor=2.1,
                search_cutoff=1.1 * pitch, length=(nx - 1) * pitch, area=ny * nz * pitch * pitch,
                bparams=dict(quirks=bond_quirks, beta=0.1, radius_factor=0.5, kn=kn, kt=kt,
                             break_strain=break_strain))


def batched_scenes(nscenes=1024, nmin=2, nmax=8192, radius=1e-3, seed=3, dt=1e-7, nsteps=20_000,
                   quirks=REF_COMPAT, max_cnts=16):
    """Independent scenes in one batch: scene k is a compact random cluster of n_k spheres
    (n_k log-uniform in [2, 8192]) of r = 1 mm glass, fired at its own plane y = 0 at an angle
    U[0, 90] degrees from the normal and a speed U[1, 5] m/s, with restitution U[0.3, 0.95]
    and friction U[0.1, 0.5] (pp and pw alike).  All scenes share local coordinates; the
    scene index keeps them apart.  dt = 1e-7 s."""
    rng = np.random.default_rng(seed)
    counts = np.floor(np.exp(rng.uniform(np.log(nmin), np.log(nmax), size=nscenes))).astype(int)
    counts = np.clip(counts, nmin, nmax)
    # lattice points of pitch 2.05 r sorted by distance from the origin: a scene takes the first n_k
    pitch = 2.05 * radius
    m = int(np.ceil((nmax * 6 / np.pi) ** (1 / 3))) + 2
    g = np.arange(-m, m + 1)
    lat = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1).reshape(-1, 3).astype(float) * pitch
    lat = lat[np.argsort((lat ** 2).sum(axis=1), kind="stable")][:nmax]
    n = int(counts.sum())
    s = ParticleState.create(n, max_cnts=max_cnts, max_walls=1)
    scene = np.repeat(np.arange(nscenes), counts).astype(np.int32)
    params, walls = [], WallState.create(nscenes)
    off = 0
    for k in range(nscenes):
        c = counts[k]
        pts = lat[:c] + rng.uniform(-0.02, 0.02, size=(c, 3)) * radius
        theta = np.deg2rad(rng.uniform(0.0, 90.0))
        speed = rng.uniform(1.0, 5.0)
        e, mu = rng.uniform(0.3, 0.95), rng.uniform(0.1, 0.5)
        pts[:, 1] += -pts[:, 1].min() + radius * 1.02     # lowest sphere just above the plane
        s.x[off:off + c] = pts
        s.u[off:off + c] = (speed * np.sin(theta), -speed * np.cos(theta), 0.0)
        params.append((e, e, mu, mu))
        walls.x[k] = (0.0, 0.0, 0.0)
        walls.normal[k] = (0.0, 1.0, 0.0)
        off += c
    _apply_glass(s, radius)
    walls.E[:], walls.nu[:], walls.G[:] = GLASS["E"], GLASS["nu"], s.G[0]
    sc = Scenario("batched_%d" % nscenes, s, walls, _force_params(0.8, 0.8, 0.3, 0.3, quirks), dt, nsteps,
                  skin=0.1 * radius)
    sc.extra = dict(scene=scene, scene_params=params, walls_per_scene=1, counts=counts)
    return sc


def scene_subset(sc, k):
    """Scenario of scene k of a batched_scenes set on its own (its particles, wall and
    restitution/friction), for checking the batch against separate runs."""
    counts = sc.extra["counts"]
    start = int(counts[:k].sum())
    c = int(counts[k])
    st = ParticleState.create(c, max_cnts=sc.state.max_cnts, max_walls=1)
    for f, v in sc.state.arrays().items():
        if f.startswith("tng_sw"):
            getattr(st, f)[:] = v[start:start + c, :1]
        else:
            getattr(st, f)[...] = v[start:start + c]
    w = WallState.create(1)
    for f in ("x", "u", "omega", "normal"):
        getattr(w, f)[0] = getattr(sc.walls, f)[k]
    for f in ("E", "nu", "G"):
        getattr(w, f)[0] = getattr(sc.walls, f)[k]
    e_pp, e_pw, mu_pp, mu_pw = sc.extra["scene_params"][k]
    return Scenario("scene_%d" % k, st, w, _force_params(e_pp, e_pw, mu_pp, mu_pw, sc.params["quirks"]), sc.dt,
                    sc.nsteps, skin=sc.skin, gravity=sc.gravity)


SCENE_BUCKETS = (64, 1024)   # scene-size bucket edges of the batched workload


def scene_bucket_of(count, edges=SCENE_BUCKETS):
    """Index of the size bucket of a scene with `count` particles: [2, 64), [64, 1024), [1024, ...)."""
    return int(np.searchsorted(np.asarray(edges), count, side="right"))


def split_scenes(sc, edges=SCENE_BUCKETS):
    """The scenes of a batched_scenes set grouped by size bucket: a list of (bucket, scenario,
    scene ids) with one batched scenario per non-empty bucket, its scenes renumbered 0..k-1 in
    their original order and keeping their particles, wall, restitution and friction.  A scene
    evolves the same in any batch (scenes never interact), so each bucket can run with launch
    settings of its own."""
    counts = np.asarray(sc.extra["counts"])
    starts = np.concatenate([[0], np.cumsum(counts)])
    buckets = np.array([scene_bucket_of(c, edges) for c in counts])
    out = []
    for b in range(len(edges) + 1):
        ids = np.nonzero(buckets == b)[0]
        if len(ids) == 0:
            continue
        rows = np.concatenate([np.arange(starts[k], starts[k + 1]) for k in ids])
        n = len(rows)
        st = ParticleState.create(n, max_cnts=sc.state.max_cnts, max_walls=sc.state.max_walls)
        for f, v in sc.state.arrays().items():
            getattr(st, f)[...] = v[rows]
        w = WallState.create(len(ids))
        for f in ("x", "u", "omega", "normal", "E", "nu", "G"):
            getattr(w, f)[...] = getattr(sc.walls, f)[ids]
        sub = Scenario("%s_bucket%d" % (sc.name, b), st, w, dict(sc.params), sc.dt, sc.nsteps, skin=sc.skin,
                       gravity=sc.gravity)
        sub.extra = dict(scene=np.repeat(np.arange(len(ids)), counts[ids]).astype(np.int32),
                         scene_params=[sc.extra["scene_params"][k] for k in ids], walls_per_scene=1,
                         counts=counts[ids], rows=rows)
        out.append((b, sub, ids))
    return out


# Quasi-2D granular dam break.  The stiffness is not fixed by the workload: E = 1 GPa keeps the
# largest Hertz overlap of a 4 m/s collision near 3.4 % of r (below the surrogate's 5 % check;
# E = 30 MPa would reach 14 %) and the static overlap at the foot of a 1 m column near 0.2 %,
# and allows dt = 1 us (about 30 steps per collision at 4 m/s).
DAM = dict(rho=2600.0, E=1e9, nu=0.25, mu=0.4, cor=0.5, dt=1e-6)


def dam_break(n=200_000, aspect=None, seed=11, rmin=0.9e-3, rmax=1.1e-3, nsteps=1_000_000, max_cnts=12,
              quirks=REF_COMPAT, dt=DAM["dt"]):
    """n disks (spheres with z = 0, in-plane motion only) with r ~ U[0.9, 1.1] mm on a jittered
    hexagonal lattice of pitch 2.25 mm filling a column of width W and height aspect * W
    (aspect ~ U[0.5, 4] unless given) against the left wall x = 0, on the floor y = 0, with
    a right wall far downstream; released at rest under gravity -y.  mu = 0.4, e = 0.5
    (pp and pw), E = 1 GPa, rho = 2600.  nsteps = 1 s at dt = 1 us.  Verlet skin 0.4 r_mean:
    the flow reaches a few m/s, and a thinner skin would rebuild the list every few steps."""
    rng = np.random.default_rng(seed)
    if aspect is None:
        aspect = float(rng.uniform(0.5, 4.0))
    pitch = 2.25e-3
    rowh = pitch * math.sqrt(3.0) / 2.0
    width = math.sqrt(n * pitch * rowh / aspect)
    ncol = max(2, int(round(width / pitch)))
    nrow = int(math.ceil(n / ncol))
    k = np.arange(n)
    row, col = k // ncol, k % ncol
    x = (col + 0.5 * (row % 2)) * pitch + rmax + 0.1e-3
    y = row * rowh + rmax + 0.1e-3
    rad = rng.uniform(rmin, rmax, size=n)
    room = 0.5 * pitch - rad
    # |jitter| <= room / sqrt(2) per particle: lattice neighbours (all at distance pitch) keep a gap
    x = x + rng.uniform(-0.5, 0.5, size=n) * room
    y = y + rng.uniform(-0.5, 0.5, size=n) * room
    st = ParticleState.create(n, max_cnts=max_cnts, max_walls=3)
    st.x[:, 0], st.x[:, 1] = x, y
    st.rad[:] = rad
    st.rho[:] = DAM["rho"]
    st.E[:], st.nu[:], st.G[:] = DAM["E"], DAM["nu"], DAM["E"] / (2.0 * (1.0 + DAM["nu"]))
    st.m[:] = 4. / 3. * math.pi * rad ** 3 * DAM["rho"]
    st.I[:] = 2. / 5. * st.m * rad * rad
    col_w = (ncol + 0.5) * pitch + 2.0 * rmax
    length = col_w * (2.0 + 3.0 * aspect)
    w = WallState.create(3)
    w.x[0], w.normal[0] = (0.0, 0.0, 0.0), (0.0, 1.0, 0.0)          # floor
    w.x[1], w.normal[1] = (0.0, 0.0, 0.0), (1.0, 0.0, 0.0)          # back wall
    w.x[2], w.normal[2] = (length, 0.0, 0.0), (-1.0, 0.0, 0.0)      # far wall
    w.E[:], w.nu[:], w.G[:] = DAM["E"], DAM["nu"], DAM["E"] / (2.0 * (1.0 + DAM["nu"]))
    sc = Scenario("dam_break_%d" % n, st, w, _force_params(DAM["cor"], DAM["cor"], DAM["mu"], DAM["mu"], quirks), dt,
                  nsteps, skin=0.4 * 0.5 * (rmin + rmax), gravity=(0.0, -9.81, 0.0))
    sc.extra = dict(aspect=aspect, column_width=col_w, column_height=nrow * rowh, length=length,
                    r_mean=0.5 * (rmin + rmax), r_std=(rmax - rmin) / math.sqrt(12.0))
    return sc


def combine_scenes(scenarios, name="batch"):
    """Independent scenarios as one batch of scenes (same dt, gravity and walls per scene):
    particles concatenated in order, scene k owns walls [k*W, (k+1)*W)."""
    first = scenarios[0]
    W = first.walls.n
    mc = max(sc.state.max_cnts for sc in scenarios)
    n = sum(sc.state.n for sc in scenarios)
    st = ParticleState.create(n, max_cnts=mc, max_walls=W)
    walls = WallState.create(W * len(scenarios))
    scene = np.zeros(n, dtype=np.int32)
    params, counts, off = [], [], 0
    for k, sc in enumerate(scenarios):
        if sc.walls.n != W or sc.dt != first.dt or tuple(sc.gravity) != tuple(first.gravity):
            raise ValueError("scenes need the same wall count, dt and gravity")
        c = sc.state.n
        for f in ("x", "u", "omega", "m", "rho", "rad", "I", "E", "nu", "G"):
            getattr(st, f)[off:off + c] = getattr(sc.state, f)
        for f in ("x", "u", "omega", "normal", "E", "nu", "G"):
            getattr(walls, f)[k * W:(k + 1) * W] = getattr(sc.walls, f)
        scene[off:off + c] = k
        p = sc.params
        params.append((p["cor_pp"], p["cor_pw"], p["mu_pp"], p["mu_pw"]))
        counts.append(c)
        off += c
    out = Scenario(name, st, walls, dict(first.params), first.dt, first.nsteps, delta=first.delta, skin=first.skin,
                   gravity=first.gravity)
    out.extra = dict(scene=scene, scene_params=params, walls_per_scene=W, counts=np.asarray(counts))
    return out


def bdem_two_particles():
    """examples/tst_01_BDEM_two_particles_tensile_3D.cpp:162-302: two bonded spheres
    pulled apart by +-1e3 N, particle 0's force zeroed after the bond pass."""
    radius, rho, E, G, nu = 0.5, 2000., 1e4, 1e3, 0.25
    s = ParticleState.create(2, max_cnts=1, max_walls=1)
    for i in range(2):
        s.x[i, 0] = -radius + i * (2. * radius)
    s.rad[:], s.rho[:], s.E[:], s.G[:], s.nu[:] = radius, rho, E, G, nu
    _mass(s, radius, rho)
    b = BondState.create(2, 27)
    ext = np.zeros((2, 3))
    ext[0, 0], ext[1, 0] = -1e3, 1e3
    fix = np.zeros(2, dtype=np.uint8)
    fix[0] = 1  # zero force (not torque) of particle 0
    dt = 1e-4
    return dict(state=s, bonds=b, dt=dt, nsteps=int(4. / dt) + 1, ext_force=ext, fix_flags=fix,
                bond_factor=3.0, search_cutoff=4. * radius,
                bparams=dict(quirks=0x07, beta=0.1, radius_factor=1.0, kn=0.0, kt=0.0, break_strain=0.0))


# ----------------------------------------------------------------------------------------
# Seeded benchmark workloads
# ----------------------------------------------------------------------------------------
GLASS = dict(rho=2600.0, E=70e9, nu=0.25)  # G = E / (2 (1 + nu)) = 28 GPa


def _box_walls(lo, hi, E, nu, G):
    """Six planes bounding [lo, hi]^3, normals pointing inwards."""
    w = WallState.create(6)
    k = 0
    for d in range(3):
        for side, (pt, sgn) in enumerate(((lo, 1.0), (hi, -1.0))):
            w.x[k, d] = pt[d]
            w.normal[k, d] = sgn
            k += 1
    w.E[:], w.nu[:], w.G[:] = E, nu, G
    return w


def _apply_glass(s, rad):
    E, nu, rho = GLASS["E"], GLASS["nu"], GLASS["rho"]
    s.rad[:] = rad
    s.rho[:] = rho
    s.E[:], s.nu[:], s.G[:] = E, nu, E / (2.0 * (1.0 + nu))
    s.m[:] = 4. / 3. * math.pi * s.rad * s.rad * s.rad * s.rho
    s.I[:] = 2. / 5. * s.m * s.rad * s.rad


def random_box(n=4096, radius=1e-3, side=0.05, seed=1, vmax=0.1, max_cnts=16, quirks=REF_COMPAT,
               dt=1e-7, nsteps=10_000):
    """4,096 monodisperse r = 1 mm glass spheres, non-overlapping by uniform rejection
    sampling in a 5 cm cube with 6 walls; v ~ U[-0.1, 0.1]^3, gravity -z, dt = 1e-7,
    Verlet skin 0.1 r, mu = 0.3, e = 0.8."""
    rng = np.random.default_rng(seed)
    pos = np.zeros((n, 3))
    cell = 2.0 * radius
    grid = {}
    k = tries = 0
    while k < n:
        tries += 1
        if tries > 200 * n:
            raise ValueError("random_box: cannot place %d spheres of r = %g in a cube of side %g" % (n, radius, side))
        p = rng.uniform(radius, side - radius, size=3)
        c = tuple((p // cell).astype(int))
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for q in grid.get((c[0] + dx, c[1] + dy, c[2] + dz), ()):
                        if np.sum((pos[q] - p) ** 2) < (2.0 * radius) ** 2:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if not ok:
                break
        if ok:
            pos[k] = p
            grid.setdefault(c, []).append(k)
            k += 1
    s = ParticleState.create(n, max_cnts=max_cnts, max_walls=6)
    s.x[:] = pos
    s.u[:] = rng.uniform(-vmax, vmax, size=(n, 3))
    _apply_glass(s, radius)
    w = _box_walls((0.0, 0.0, 0.0), (side, side, side), GLASS["E"], GLASS["nu"], s.G[0])
    return Scenario("random_box_4096", s, w, _force_params(0.8, 0.8, 0.3, 0.3, quirks), dt, nsteps,
                    skin=0.1 * radius, gravity=(0.0, 0.0, -9.81))


def piston_box(n=4096, speed=2.0, seed=1, nsteps=400, quirks=REF_COMPAT & ~Q6_WALL_STATIC):
    """random_box with its +x wall (wall 1) moved to touch the outermost sphere and driven
    inwards at `speed` m/s: a kinematic wall (DEM_Q6_WALL_STATIC clear; the reference's walls
    never move, src/CabanaDEM_Force.hpp:529)."""
    sc = random_box(n=n, seed=seed, quirks=quirks, nsteps=nsteps)
    sc.walls.x[1, 0] = float((sc.state.x[:, 0] + sc.state.rad).max())
    sc.walls.u[1, 0] = -float(speed)
    sc.name = "piston_box_%d" % n
    return sc


def mesh_hopper(n=2048, radius=1e-3, seed=4, nsteps=2000, speed=0.0, quirks=REF_COMPAT, max_contacts=8,
                drop_speed=2.0, band=0.01):
    """Spheres falling into a V-shaped trough made of triangles (no reference counterpart):
    two planes sloping at 35 degrees towards the line x = 0.025 m, y = 0, each made of 6
    rectangular panels split along a diagonal, closed by two vertical end plates (plane walls
    at z = 0 and z = 0.05).  The spheres start within `band` m above touching the trough,
    moving down at drop_speed.  Glass, e = 0.8, mu = 0.3, gravity -y, dt 1e-7, skin 0.1 r.
    speed > 0 drives the whole trough upwards (Q6 cleared)."""
    from .state import MeshState
    rng = np.random.default_rng(seed)
    L, depth = 0.05, 0.05
    tan = math.tan(math.radians(35.0))
    s = ParticleState.create(n, max_cnts=16, max_walls=2)
    pts, cell, grid, k, tries = np.zeros((n, 3)), 2.0 * radius, {}, 0, 0
    while k < n:   # non-overlapping, above the trough
        tries += 1
        if tries > 200 * n:
            raise ValueError("mesh_hopper: %d spheres do not fit in the release layer" % n)
        p = rng.uniform((2 * radius, 0.0, 2 * radius), (L - 2 * radius, band, depth - 2 * radius))
        p[1] += abs(p[0] - L / 2) * tan + 1.25 * radius / math.cos(math.radians(35.0))
        c = tuple((p // cell).astype(int))
        if all(np.sum((pts[q] - p) ** 2) >= (2.0 * radius) ** 2
               for dx in (-1, 0, 1) for dy in (-1, 0, 1) for dz in (-1, 0, 1)
               for q in grid.get((c[0] + dx, c[1] + dy, c[2] + dz), ())):
            pts[k] = p
            grid.setdefault(c, []).append(k)
            k += 1
    s.x[:] = pts
    s.u[:, 1] = -float(drop_speed)
    _apply_glass(s, radius)
    tri = []
    for side in (-1.0, 1.0):
        xs = np.linspace(L / 2, L / 2 + side * (L / 2 + 4 * radius), 7)
        zs = np.linspace(0.0, depth, 2)
        for a in range(6):
            for b in range(1):
                p00 = (xs[a], abs(xs[a] - L / 2) * tan, zs[b])
                p10 = (xs[a + 1], abs(xs[a + 1] - L / 2) * tan, zs[b])
                p01 = (xs[a], abs(xs[a] - L / 2) * tan, zs[b + 1])
                p11 = (xs[a + 1], abs(xs[a + 1] - L / 2) * tan, zs[b + 1])
                tri += [(p00, p10, p11), (p00, p11, p01)]
    mesh = MeshState.create(np.array(tri), n, GLASS["E"], GLASS["nu"], s.G[0], u=(0.0, speed, 0.0),
                            max_contacts=max_contacts)
    w = WallState.create(2)
    w.x[1, 2] = depth
    w.normal[0, 2], w.normal[1, 2] = 1.0, -1.0
    w.E[:], w.nu[:], w.G[:] = GLASS["E"], GLASS["nu"], s.G[0]
    if speed:
        quirks = quirks & ~Q6_WALL_STATIC
    sc = Scenario("mesh_hopper_%d" % n, s, w, _force_params(0.8, 0.8, 0.3, 0.3, quirks), 1e-7, nsteps,
                  skin=0.1 * radius, gravity=(0.0, -9.81, 0.0))
    sc.extra["mesh"] = mesh
    return sc


def hcp_box(n=2_000_000, rmin=0.8e-3, rmax=1.2e-3, seed=2, vmax=0.1, max_cnts=16, quirks=REF_COMPAT,
            dt=5e-8, nsteps=2000, jitter=0.05):
    """Polydisperse spheres (r ~ U[0.8, 1.2] mm) on a hexagonal-close-packed lattice of
    pitch a = 2 r_max, each site jittered by U(-1, 1) * 0.05 * (a/2 - r_i) per axis (no
    initial overlap), inside a walled box; v ~ U[-0.1, 0.1]^3, gravity -z, dt = 5e-8,
    skin 0.1 r_mean, neighbour rebuild when the displacement bound exceeds skin / 2."""
    rng = np.random.default_rng(seed)
    a = 2.0 * rmax
    side = (n * a ** 3 / math.sqrt(2.0)) ** (1.0 / 3.0)
    nx = max(1, int(round(side / a)))
    ny = max(1, int(round(side / (a * math.sqrt(3.0) / 2.0))))
    nz = int(math.ceil(n / (nx * ny)))
    k = np.arange(n)
    ix, iy, iz = k % nx, (k // nx) % ny, k // (nx * ny)
    px = a * (ix + 0.5 * ((iy + iz) % 2))
    py = a * math.sqrt(3.0) / 2.0 * (iy + (iz % 2) / 3.0)
    pz = a * math.sqrt(2.0 / 3.0) * iz
    rad = rng.uniform(rmin, rmax, size=n)
    pos = np.stack([px, py, pz], axis=1)
    pos += rng.uniform(-1.0, 1.0, size=(n, 3)) * (jitter * (a / 2.0 - rad))[:, None]
    pos += a  # margin from the walls
    s = ParticleState.create(n, max_cnts=max_cnts, max_walls=6)
    s.x[:] = pos
    s.u[:] = rng.uniform(-vmax, vmax, size=(n, 3))
    _apply_glass(s, rad)
    hi = pos.max(axis=0) + a
    w = _box_walls((0.0, 0.0, 0.0), tuple(hi), GLASS["E"], GLASS["nu"], s.G[0])
    return Scenario("hcp_box_%d" % n, s, w, _force_params(0.8, 0.8, 0.3, 0.3, quirks), dt, nsteps,
                    skin=0.1 * 0.5 * (rmin + rmax), gravity=(0.0, 0.0, -9.81))
