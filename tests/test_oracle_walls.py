"""Kinematic walls in the CPU oracle (DEM_Q6_WALL_STATIC clear): the reference's walls never
move and its wall contact uses vel_j = 0 (src/CabanaDEM_Force.hpp:529); with the bit clear a
wall drifts by dt * u each step with the particles and the contact uses the relative
velocity.  Checked against mechanics: an elastic, frictionless sphere at rest struck by a
wall moving at V leaves at 2 V; with the bit set the same wall neither moves nor matters."""
import numpy as np

from cabanadem_b200 import scenarios as S
from cabanadem_b200.state import ParticleState, WallState
from oracle import oracle as O


def _sphere_and_wall(quirks, speed=0.5):
    r = 1e-3
    s = ParticleState.create(1, max_cnts=4, max_walls=1)
    s.rad[:] = r
    s.rho[:] = 2600.0
    s.E[:], s.nu[:] = 70e9, 0.25
    s.G[:] = 70e9 / 2.5
    s.set_sphere_mass()
    s.x[0] = (0.0, 0.0, 0.0)
    w = WallState.create(1)
    w.x[0] = (r + 1e-6, 0.0, 0.0)
    w.normal[0] = (-1.0, 0.0, 0.0)
    w.u[0] = (-speed, 0.0, 0.0)
    w.E[:], w.nu[:], w.G[:] = 70e9, 0.25, 70e9 / 2.5
    fp = dict(cor_pp=1.0, cor_pw=1.0, mu_pp=0.0, mu_pw=0.0, quirks=quirks)
    return s, w, fp


def test_moving_wall_reflects_sphere_at_twice_its_speed():
    s, w, fp = _sphere_and_wall(S.REF_COMPAT & ~S.Q6_WALL_STATIC)
    x0 = w.x.copy()
    dt, n = 1e-8, 4000
    O.run(s, w, fp, dt, n)
    assert abs(s.u[0, 0] / (-2 * 0.5) - 1.0) < 1e-3, s.u[0]
    assert s.tng_count[0] == 0
    # the wall's drift: n additions of dt * u, as the device performs them
    x = x0[0, 0]
    for _ in range(n):
        x = x + dt * w.u[0, 0]
    assert w.x[0, 0] == x and w.x[0, 1] == 0.0


def test_static_walls_ignore_their_velocity():
    s, w, fp = _sphere_and_wall(S.REF_COMPAT)
    x0 = w.x.copy()
    O.run(s, w, fp, 1e-8, 4000)
    assert np.array_equal(w.x, x0)
    assert np.array_equal(s.u, np.zeros((1, 3)))


def test_piston_compresses_the_box():
    sc = S.piston_box(n=512, speed=5.0, nsteps=300)
    st, w = sc.state.copy(), sc.walls.copy()
    O.run(st, w, sc.params, sc.dt, 300, skin=sc.skin, gravity=sc.gravity)
    assert w.x[1, 0] < sc.walls.x[1, 0]
    touching = st.x[:, 0] + st.rad > w.x[1, 0]
    assert touching.any() and (st.u[touching, 0] < 0).all()
