"""Analytic known-answer checks of the oracle's physics, independent of the reference's data
files.  An elastic head-on impact (e = 1, mu = 0) gives back the kinetic energy it started
with and swaps the velocities.  A damped one separates at e times the approach speed (the
damping law of src/CabanaDEM_Force.hpp:206-215).  A sphere resting on a floor settles at
the Hertz static overlap, and one sliding without spin ends up rolling at 5/7 of its initial
speed (the wall's Mindlin spring and Coulomb limit, Force.hpp:448-678), with the tangential
damping off (the reference) or on (DEM_Q2 clear).  Colliding clusters with friction and damping
keep their total momentum: with every reference quirk cleared, each pair's forces are equal and
opposite.  A bond at its rest length exerts no force.  The device FP64 path is bit-identical to
the oracle, so these hold for it too."""
import numpy as np
import pytest

from cabanadem_b200.scenarios import Q2_ETA_T_ZERO, _force_params
from cabanadem_b200.state import BondState, ParticleState, WallState
from oracle import oracle as O

R, RHO, E, NU = 0.01, 2600.0, 70e9, 0.25


def _pair(v=0.5, gap=1e-5):
    """Two glass spheres of r = 1 cm closing head-on along x at +-v."""
    s = ParticleState.create(2, max_cnts=6, max_walls=1)
    s.x[0, 0], s.x[1, 0] = -R - gap / 2, R + gap / 2
    s.u[0, 0], s.u[1, 0] = v, -v
    s.rad[:], s.rho[:], s.E[:], s.nu[:] = R, RHO, E, NU
    s.G[:] = E / (2.0 * (1.0 + NU))
    s.set_sphere_mass()
    return s


def _run(s, cor, mu, nsteps, quirks=None, dt=1e-6):
    prm = _force_params(cor, cor, mu, mu) if quirks is None else _force_params(cor, cor, mu, mu, quirks)
    assert O.run(s, None, prm, dt, nsteps, skin=0.1 * R, pow_mode=O.POW_SQRT) == 0
    return s


def test_elastic_head_on_impact_conserves_energy():
    """The kinetic energy after an e = 1 impact equals the energy before, up to velocity
    Verlet's error, which shrinks at least 3x each time dt halves (6e-5 at 1 us, 9e-7 at 0.25 us
    for this contact of about 60 us)."""
    err = []
    for dt in (1e-6, 5e-7, 2.5e-7):
        s = _pair()
        ke0 = O.kinetic_energy(s)
        _run(s, 1.0, 0.0, int(round(600e-6 / dt)), dt=dt)     # closes, touches, separates
        assert s.tng_count.sum() == 0 and s.x[1, 0] - s.x[0, 0] > 2 * R   # separated
        err.append(abs(O.kinetic_energy(s) - ke0) / ke0)
        assert abs(s.u[0, 0] + 0.5) <= 1e-4 and abs(s.u[1, 0] - 0.5) <= 1e-4     # velocities swapped
    assert err[0] / err[1] >= 3.0 and err[1] / err[2] >= 3.0, err
    assert err[2] < 2e-6, err


@pytest.mark.parametrize("cor", [0.3, 0.5, 0.8])
def test_damped_head_on_impact_separates_at_e_times_approach(cor):
    s = _pair()
    _run(s, cor, 0.0, 800)
    assert s.x[1, 0] - s.x[0, 0] > 2 * R
    assert abs((s.u[1, 0] - s.u[0, 0]) / 1.0 - cor) <= 0.02 * cor


def _floor():
    w = WallState.create(1)
    w.normal[0, 2] = 1.0
    w.E[:], w.nu[:], w.G[:] = E, NU, E / (2.0 * (1.0 + NU))
    return w


def _ball(z, vx=0.0):
    s = ParticleState.create(1, max_cnts=6, max_walls=1)
    s.x[0, 2], s.u[0, 0] = z, vx
    s.rad[:], s.rho[:], s.E[:], s.nu[:] = R, RHO, E, NU
    s.G[:] = E / (2.0 * (1.0 + NU))
    s.set_sphere_mass()
    return s


def _hertz_rest_overlap(m, g=9.81):
    """m g = 4/3 E* sqrt(R) delta^1.5 with 1/E* = (1 - nu_i^2)/E_i + (1 - nu_w^2)/E_w."""
    e_star = 1.0 / (2.0 * (1.0 - NU * NU) / E)
    return (m * g / (4.0 / 3.0 * e_star * np.sqrt(R))) ** (2.0 / 3.0)


def test_sphere_on_floor_settles_at_hertz_overlap():
    s = _ball(R)                                   # touching the floor, at rest
    d_eq = _hertz_rest_overlap(s.m[0])
    prm = _force_params(0.5, 0.5, 0.3, 0.3)
    assert O.run(s, _floor(), prm, 1e-6, 20000, skin=0.1 * R, gravity=(0.0, 0.0, -9.81), pow_mode=O.POW_SQRT) == 0
    assert abs((R - s.x[0, 2]) / d_eq - 1.0) < 1e-3, (R - s.x[0, 2]) / d_eq
    assert abs(s.u[0, 2]) < 1e-6


@pytest.mark.parametrize("quirks", [0, Q2_ETA_T_ZERO], ids=["all_clear", "Q2_set"])
def test_sliding_sphere_rolls_at_five_sevenths(quirks):
    """Launched along the floor at 1 m/s without spin (friction 0.5, tangential damping on or
    off): it slides, friction spins it up, and it rolls on at 5/7 m/s.
    The reference's contact-point velocity is u + a (omega x n) with n from the contact
    towards the centre, and its torque a (n x f_t) (src/CabanaDEM_Force.hpp:520-527, :661-663;
    the pair law likewise, :114-139): its omega is the physical angular velocity negated,
    consistently, so rolling reads v = -omega_y R."""
    s0 = _ball(R)
    s = _ball(R - _hertz_rest_overlap(s0.m[0]), vx=1.0)
    prm = _force_params(0.5, 0.5, 0.5, 0.5, quirks)
    assert O.run(s, _floor(), prm, 1e-6, 100000, skin=0.1 * R, gravity=(0.0, 0.0, -9.81), pow_mode=O.POW_SQRT) == 0
    v, w = s.u[0, 0], s.omega[0, 1]
    assert abs(v / (5.0 / 7.0) - 1.0) < 0.01, v
    assert abs(v + w * R) < 0.01 * v, (v, w * R)


@pytest.mark.parametrize("quirks", [0, Q2_ETA_T_ZERO], ids=["all_clear", "Q2_set"])
def test_sliding_sphere_slows_at_mu_g(quirks):
    """A sphere sliding along the floor decelerates at mu g (plus the small rolling-resistance
    share of the spin-up), with the tangential damping off (DEM_Q2 set, the reference) and on
    (DEM_Q2 clear).  The reference adds eta_t v_t back to the limited wall force
    (src/CabanaDEM_Force.hpp:640-643); with its eta_t = 0 that changes nothing, but with
    eta_t > 0 it would push along the sliding direction (1 -> 54 m/s in 300 steps).  With
    DEM_Q2 clear the limited force acts and the damping only resets the spring."""
    s = _ball(R - _hertz_rest_overlap(_ball(R).m[0]), vx=1.0)
    assert O.run(s, _floor(), _force_params(0.5, 0.5, 0.5, 0.5, quirks), 1e-6, 300, skin=0.1 * R,
                 gravity=(0.0, 0.0, -9.81), pow_mode=O.POW_SQRT) == 0
    assert abs(s.u[0, 0] - (1.0 - 0.5 * 9.81 * 300e-6)) < 1e-3, s.u[0, 0]


def test_sliding_pair_contact_is_at_the_coulomb_limit():
    """Two spheres closing at 0.5 m/s while grazing at 2 m/s (e = 1, friction 0.3, every quirk
    clear but DEM_Q2): the contact slides throughout, and at every step of it the tangential
    force is mu times the normal force in the contact frame (the limit of
    src/CabanaDEM_Force.hpp:290-301).  With damping (e < 1) the normal force turns tensile near
    the end of the contact, so the friction impulse then exceeds mu times the normal impulse."""
    s = _pair(v=0.25)
    s.u[0, 1], s.u[1, 1] = 1.0, -1.0
    ratio = []
    for _ in range(300):
        _run(s, 1.0, 0.3, 1, quirks=Q2_ETA_T_ZERO)
        if s.tng_count[0]:
            n = (s.x[0] - s.x[1]) / np.linalg.norm(s.x[0] - s.x[1])
            fn = s.force[0] @ n
            ratio.append(np.linalg.norm(s.force[0] - fn * n) / fn)
    assert len(ratio) >= 50 and s.tng_count[0] == 0
    assert np.abs(np.array(ratio) - 0.3).max() < 1e-12


def _elastic_energy(s, w):
    """Hertz elastic energy 2/5 k_n delta^(5/2) of every particle-particle and particle-wall
    overlap (k_n = 4/3 E* sqrt(R*), Force.hpp:196-203 and :561-568)."""
    e = 0.0
    for i in range(s.n):
        for j in range(i + 1, s.n):
            d = s.rad[i] + s.rad[j] - np.linalg.norm(s.x[i] - s.x[j])
            if d > 0:
                es = 1.0 / ((1 - s.nu[i] ** 2) / s.E[i] + (1 - s.nu[j] ** 2) / s.E[j])
                rs = 1.0 / (1.0 / s.rad[i] + 1.0 / s.rad[j])
                e += 0.4 * (4.0 / 3.0 * es * np.sqrt(rs)) * d ** 2.5
        for k in range(w.n):
            d = s.rad[i] - (s.x[i] - w.x[k]) @ w.normal[k]
            if d > 0:
                es = 1.0 / ((1 - s.nu[i] ** 2) / s.E[i] + (1 - w.nu[k] ** 2) / w.E[k])
                e += 0.4 * (4.0 / 3.0 * es * np.sqrt(s.rad[i])) * d ** 2.5
    return e


def test_elastic_gas_conserves_energy_with_the_reference_bits():
    """60 spheres bouncing in a walled box for 25 ms with the reference's bits (e = 1, mu = 0):
    kinetic plus Hertz elastic energy stays constant to velocity Verlet's error (1e-5) through
    their collisions with each other and the walls."""
    from cabanadem_b200.scenarios import _box_walls
    rng = np.random.default_rng(3)
    g = (np.arange(4) + 0.5) * 2.6 * R
    pos = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)[:60]
    s = ParticleState.create(60, max_cnts=12, max_walls=6)
    s.x[:] = pos + rng.uniform(-0.1 * R, 0.1 * R, size=pos.shape)
    s.u[:] = rng.uniform(-1.0, 1.0, size=pos.shape)
    s.rad[:], s.rho[:], s.E[:], s.nu[:] = R, RHO, E, NU
    s.G[:] = E / (2.0 * (1.0 + NU))
    s.set_sphere_mass()
    w = _box_walls((0.0, 0.0, 0.0), (10.4 * R,) * 3, E, NU, float(s.G[0]))
    e0 = O.kinetic_energy(s) + _elastic_energy(s, w)
    in_contact = 0
    for _ in range(200):                      # 25 ms
        assert O.run(s, w, _force_params(1.0, 1.0, 0.0, 0.0), 2.5e-7, 500, skin=0.1 * R, pow_mode=O.POW_SQRT) == 0
        ke = O.kinetic_energy(s)
        e = ke + _elastic_energy(s, w)
        ep, ew = O.elastic_energy(s, w)                    # the oracle's C restatement agrees
        assert abs(ep + ew - (e - ke)) <= 1e-12 * e0
        in_contact += int(ke < (1.0 - 1e-4) * e)          # energy stored in some contact
        assert abs(e - e0) <= 1e-5 * e0, (e - e0) / e0
    assert in_contact >= 5


@pytest.mark.parametrize("quirks,stands", [(0x3F, False), (0x3F & ~0x04, True)], ids=["reference", "Q3_clear"])
def test_three_sphere_pyramid(quirks, stands):
    """Two spheres on a floor with a third on top (friction 0.5, statically stable in physics:
    it needs mu > tan 15 deg).  With the pair contact's torque (DEM_Q3 clear) it settles and
    stands.  The reference's pair contacts add no torque (src/CabanaDEM_Force.hpp:324-326): the
    floor's friction turns the base spheres and nothing at the top contact resists it, so
    they roll apart."""
    d_eq = _hertz_rest_overlap(_ball(R).m[0])
    s = ParticleState.create(3, max_cnts=6, max_walls=1)
    s.x[0] = [-R + 0.5e-6, 0.0, R - d_eq]
    s.x[1] = [R - 0.5e-6, 0.0, R - d_eq]
    s.x[2] = [0.0, 0.0, R - d_eq + np.sqrt(3.0) * R]
    s.rad[:], s.rho[:], s.E[:], s.nu[:] = R, RHO, E, NU
    s.G[:] = E / (2.0 * (1.0 + NU))
    s.set_sphere_mass()
    assert O.run(s, _floor(), _force_params(0.5, 0.5, 0.5, 0.5, quirks), 1e-6, 20000, skin=0.1 * R,
                 gravity=(0.0, 0.0, -9.81), pow_mode=O.POW_SQRT) == 0
    spread = s.x[1, 0] - s.x[0, 0] - 2.0 * R
    if stands:
        assert spread < 5e-5 and np.abs(s.u).max() < 1e-4, (spread, np.abs(s.u).max())
    else:
        assert spread > 2e-4 and np.abs(s.u).max() > 5e-3, (spread, np.abs(s.u).max())


@pytest.mark.parametrize("uz", [-0.6, 0.6], ids=["opposite_signs", "same_signs"])
def test_reference_wall_friction_depends_on_direction(uz):
    """src/CabanaDEM_Force.hpp:624 takes |f_t| as sqrt(f_x^2 + f_y^2 + f_z f_y) (DEM_Q5).  A
    sphere pressed on a wall with normal +x and sliding with (v_y, v_z) = (0.3, -0.6) has
    f_z f_y < -f_y^2: the square root is NaN, `ft_magn > 1e-12` is false, the direction stays
    zero and no friction acts at all (the velocity is unchanged; nothing becomes NaN).  Sliding
    with (0.3, 0.6) the wrong magnitude is sqrt(3) f_y instead of sqrt(5) f_y, the direction
    vector is sqrt(5/3) long, and friction acts 1.29 times too strongly.  With the bit clear it
    slows the sphere at mu g in both directions."""
    from cabanadem_b200.scenarios import Q5_WALL_FT_TYPO, REF_COMPAT
    w = WallState.create(1)
    w.normal[0, 0] = 1.0
    w.E[:], w.nu[:], w.G[:] = E, NU, E / (2.0 * (1.0 + NU))
    got = {}
    for q in (REF_COMPAT, REF_COMPAT & ~Q5_WALL_FT_TYPO):
        s = _ball(R)
        s.x[0] = [R - _hertz_rest_overlap(s.m[0]), 0.0, 0.0]
        s.u[0] = [0.0, 0.3, uz]
        assert O.run(s, w, _force_params(0.5, 0.5, 0.5, 0.5, q), 1e-6, 200, skin=0.1 * R,
                     gravity=(-9.81, 0.0, 0.0), pow_mode=O.POW_SQRT) == 0
        assert np.isfinite(s.u).all() and np.isfinite(s.force).all()
        got[q] = np.hypot(s.u[0, 1], s.u[0, 2])
    v0, slowed = np.hypot(0.3, uz), np.hypot(0.3, uz) - 0.5 * 9.81 * 200e-6
    assert abs(got[REF_COMPAT & ~Q5_WALL_FT_TYPO] - slowed) < 2e-5
    if uz < 0:
        assert abs(got[REF_COMPAT] - v0) < 1e-12
    else:
        ratio = (v0 - got[REF_COMPAT]) / (v0 - got[REF_COMPAT & ~Q5_WALL_FT_TYPO])
        assert abs(ratio - np.sqrt(5.0 / 3.0)) < 0.01, ratio


def test_reference_pair_friction_ignores_sliding_across_y_and_z():
    """src/CabanaDEM_Force.hpp:133-137 builds the partner's contact velocity in y and z from
    particle i's own velocity (DEM_Q1).  For two spheres colliding along x while sliding past
    each other along y, the relative sliding velocity is then lost, and friction takes almost
    nothing off the sliding speed.  The 0.002 m/s that does go comes from the contact normal
    tilting as they pass.  With the bit clear the sliding speed drops by mu times the normal
    speed change, as in the Coulomb test above."""
    from cabanadem_b200.scenarios import Q1_VELJ_USES_UI, REF_COMPAT
    drop = {}
    for q in (REF_COMPAT, REF_COMPAT & ~Q1_VELJ_USES_UI):
        s = _pair(v=0.25)
        s.u[0, 1], s.u[1, 1] = 1.0, -1.0
        _run(s, 1.0, 0.3, 300, quirks=q)
        # sliding speed lost by sphere 0, normal speed change of sphere 1 (-0.25 -> about +0.24)
        drop[q] = (1.0 - s.u[0, 1], s.u[1, 0] + 0.25)
    (ref_t, _), (fix_t, fix_n) = drop[REF_COMPAT], drop[REF_COMPAT & ~Q1_VELJ_USES_UI]
    assert ref_t < 0.01 and ref_t < 0.1 * fix_t
    assert abs(fix_t / fix_n - 0.3) < 0.03


def test_cluster_collision_conserves_momentum():
    """Two jittered 3x3x3 clusters meet off-centre (oblique contacts, friction 0.4, e = 0.7,
    rotation): total momentum is unchanged to round-off."""
    rng = np.random.default_rng(7)
    g = np.arange(3) * 2.05 * R
    block = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    pos = np.vstack([block, block + [5.7 * R, 1.0 * R, 1.0 * R]])      # closest centres 2.12 R apart
    pos += rng.uniform(-0.02 * R, 0.02 * R, size=pos.shape)
    n = len(pos)
    s = ParticleState.create(n, max_cnts=12, max_walls=1)
    s.x[:] = pos
    s.u[:27, 0], s.u[27:, 0] = 0.8, -0.8
    s.u[:] += rng.uniform(-0.05, 0.05, size=(n, 3))
    s.rad[:] = R * rng.uniform(0.95, 1.0, size=n)
    s.rho[:], s.E[:], s.nu[:] = RHO, E, NU
    s.G[:] = E / (2.0 * (1.0 + NU))
    s.set_sphere_mass()
    p0 = (s.m[:, None] * s.u).sum(0)
    scale = (s.m[:, None] * np.abs(s.u)).sum()
    contacts = 0
    for _ in range(160):
        _run(s, 0.7, 0.4, 25, quirks=0)
        contacts = max(contacts, int(s.tng_count.sum()))
    assert contacts >= 10                                        # the clusters collided
    assert np.abs(s.omega).max() > 0                             # oblique contacts spun them
    p1 = (s.m[:, None] * s.u).sum(0)
    assert np.abs(p1 - p0).max() <= 1e-12 * scale, np.abs(p1 - p0).max() / scale


def _bonded_pair():
    s = ParticleState.create(2, max_cnts=1, max_walls=1)
    s.x[1, 0] = 1.0
    s.rad[:], s.rho[:], s.E[:], s.G[:], s.nu[:] = 0.5, 2000.0, 1e4, 1e3, 0.25
    s.set_sphere_mass()
    b = BondState.create(2, 4)
    O.setup_bonds(b, s, 3.0, 2.0)
    assert b.count.tolist() == [1, 1] and b.idx[:, 0].tolist() == [1, 0]
    return s, b


def test_bond_at_rest_length_exerts_no_force():
    """Two bonded spheres at rest (setupBonds sets the rest length to the current distance),
    the reference's bond law with its history indexed by bond slot (DEM_BQ10 clear): zero force
    and torque, and no motion, however many steps."""
    s, b = _bonded_pair()
    x0 = s.x.copy()
    prm = dict(quirks=O.BOND_REF_COMPAT & ~0x01, beta=0.1, radius_factor=1.0)
    assert O.bonded_run(s, b, prm, 1e-4, 1000, pow_mode=O.POW_SQRT) == 0
    assert np.array_equal(s.x, x0)
    assert not s.force.any() and not s.torque.any() and not s.u.any() and not s.omega.any()


def test_reference_bond_indexing_pulls_a_bond_at_rest():
    """src/CabanaBondedDEM_Force.hpp:207 reads the rest length as bond_init_len(i, j), with the
    partner's id j in place of the bond's slot.  Particle 0's bond (partner 1) is in slot 0,
    so it reads slot 1, an empty rest length of 0, and is pulled towards particle 1 by
    k_n * rij.  Particle 1's partner 0 is its slot 0, so it reads its own rest length and feels
    nothing.  The oracle reproduces this with DEM_BQ10 set."""
    s, b = _bonded_pair()
    assert O.bonded_run(s, b, dict(quirks=O.BOND_REF_COMPAT, beta=0.1, radius_factor=1.0), 1e-4, 1,
                        pow_mode=O.POW_SQRT) == 0
    r = 0.5
    k_n = 1e4 * np.pi * r ** 2 / (2 * r)               # E A / (r_i + r_j), BondedDEM_Force.hpp:194
    assert s.force[0, 0] > 0.9 * k_n and s.force[1, 0] == 0.0
