"""Triangle-mesh walls in the CPU oracle (no reference counterpart; the reference has only a
Python intersection prototype).  A mesh contact acts as a plane through the closest point of
the triangle; a shared edge or vertex seen from two triangles, or an edge of a triangle the
particle rests on by its face, makes no second contact.  Checked against plane walls: a
sphere sliding across the diagonal of a two-triangle floor follows the plane-floor
trajectory; a sphere dropped on a roof ridge bounces as off a single plane."""
import numpy as np

from cabanadem_b200 import scenarios as S
from cabanadem_b200.state import MeshState, ParticleState, WallState
from oracle import oracle as O

R = 1e-3
MAT = dict(E=70e9, nu=0.25, G=70e9 / 2.5)


def _sphere(x, u):
    s = ParticleState.create(1, max_cnts=4, max_walls=1)
    s.rad[:] = R
    s.rho[:] = 2600.0
    s.E[:], s.nu[:], s.G[:] = MAT["E"], MAT["nu"], MAT["G"]
    s.set_sphere_mass()
    s.x[0] = x
    s.u[0] = u
    return s


def _floor_wall():
    w = WallState.create(1)
    w.normal[0] = (0.0, 1.0, 0.0)
    w.E[:], w.nu[:], w.G[:] = MAT["E"], MAT["nu"], MAT["G"]
    return w


FP = dict(cor_pp=0.5, cor_pw=0.5, mu_pp=0.3, mu_pw=0.3, quirks=S.REF_COMPAT & ~S.Q5_WALL_FT_TYPO)


def test_two_triangle_floor_matches_plane_across_the_diagonal():
    # square [-L, L]^2 in the y = 0 plane split along the diagonal x = z
    L = 0.01
    tri = [[(-L, 0, -L), (L, 0, -L), (L, 0, L)], [(-L, 0, -L), (L, 0, L), (-L, 0, L)]]
    # resting on the floor under gravity (Hertz equilibrium overlap ~1.6 nm), sliding across x = z
    x0, u0 = (-0.0012, R - 1.6e-9, -0.001), (0.5, 0.0, 0.1)
    g = (0.0, -9.81, 0.0)
    a = _sphere(x0, u0)
    O.run(a, _floor_wall(), FP, 1e-7, 20000, skin=0.1 * R, gravity=g)
    b = _sphere(x0, u0)
    m = MeshState.create(tri, 1, **MAT)
    O.run(b, WallState.create(0), FP, 1e-7, 20000, skin=0.1 * R, gravity=g, mesh=m)
    assert b.x[0, 0] > b.x[0, 2]                        # crossed the diagonal
    assert a.tng_sw_x[0, 0] != 0.0 or a.tng_sw_z[0, 0] != 0.0   # still in sliding contact
    assert np.abs(b.x - a.x).max() < 1e-9
    assert np.abs(b.u - a.u).max() < 1e-6 * np.abs(a.u).max()
    assert m.cnt[0] <= 1


def test_roof_ridge_is_one_contact():
    # two triangles meeting at the ridge y = 0 along z, sloping down on either side
    L = 0.01
    tri = [[(0, 0, -L), (-L, -L, -L), (0, 0, L)], [(0, 0, -L), (0, 0, L), (L, -L, L)]]
    s = _sphere((0.0, R + 1e-6, 0.0), (0.0, -1.0, 0.0))
    m = MeshState.create(tri, 1, **MAT)
    fp = dict(FP, cor_pw=1.0, mu_pw=0.0)
    O.run(s, WallState.create(0), fp, 1e-8, 3000, skin=0.1 * R, mesh=m)
    p = _sphere((0.0, R + 1e-6, 0.0), (0.0, -1.0, 0.0))
    O.run(p, _floor_wall(), fp, 1e-8, 3000, skin=0.1 * R)
    assert abs(s.u[0, 1] - p.u[0, 1]) < 1e-6 and s.u[0, 1] > 0.99      # one elastic bounce
    assert abs(s.u[0, 0]) < 1e-12


def test_moving_mesh_drifts_and_pushes():
    L = 0.01
    tri = [[(-L, 0, -L), (L, 0, -L), (L, 0, L)], [(-L, 0, -L), (L, 0, L), (-L, 0, L)]]
    s = _sphere((0.0, R + 1e-6, 0.0), (0.0, 0.0, 0.0))
    m = MeshState.create(tri, 1, **MAT, u=(0.0, 0.5, 0.0))
    O.run(s, WallState.create(0), dict(FP, cor_pw=1.0, mu_pw=0.0, quirks=S.REF_COMPAT & ~S.Q6_WALL_STATIC), 1e-8,
          4000, skin=0.1 * R, mesh=m)
    D = 0.0
    for _ in range(4000):
        D = D + 1e-8 * 0.5
    assert m.D[1] == D
    assert abs(s.u[0, 1] / 1.0 - 1.0) < 1e-3         # elastic: leaves at twice the mesh speed
    static = MeshState.create(tri, 1, **MAT, u=(0.0, 0.5, 0.0))
    t = _sphere((0.0, R + 1e-6, 0.0), (0.0, 0.0, 0.0))
    O.run(t, WallState.create(0), dict(FP, cor_pw=1.0, mu_pw=0.0), 1e-8, 4000, skin=0.1 * R, mesh=static)
    assert static.D[1] == 0.0 and t.u[0, 1] == 0.0
