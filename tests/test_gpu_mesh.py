"""Triangle-mesh walls on the GPU (no reference counterpart) against the CPU oracle: spheres
dropped into a V-shaped trough of 24 triangles between two end plates, static and driven
upwards (DEM_Q6_WALL_STATIC clear), through every form of the step, in three runs.  FP64
results are bit-identical to the oracle's, and the mesh translation is the oracle's."""
import numpy as np
import pytest

from cabanadem_b200 import api, scenarios as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu

STATE_F = ("x", "u", "omega", "force", "torque", "tng_count")


@pytest.mark.parametrize("speed", [0.0, 0.5], ids=["static", "moving"])
@pytest.mark.parametrize("lanes", [0, 1, 8, "pairs"], ids=["auto", "per_thread", "coop8", "pairs"])
def test_mesh_hopper_bitwise(lanes, speed):
    sc = S.mesh_hopper(n=384, nsteps=4000, band=0.002, drop_speed=4.0, speed=speed)
    ref, m = sc.state.copy(), sc.extra["mesh"].copy()
    st = O.run(ref, sc.walls.copy(), sc.params, sc.dt, 4000, skin=sc.skin, gravity=sc.gravity, pow_mode=O.POW_SQRT,
               mesh=m)
    assert st == 0
    assert (ref.u[:, 1] > 0).sum() > 50        # bounced off the trough
    if lanes == "pairs":
        s = api.from_scenario(sc, dense_form=2)
    else:
        s = api.from_scenario(sc, contact_lanes=lanes)
    for n in (1500, 1001, 1499):
        s.run_steps(n)
    got = s.particles.download()
    for f in STATE_F:
        a, b = getattr(got, f), getattr(ref, f)
        assert np.array_equal(a, b), (f, np.abs(np.asarray(a, float) - np.asarray(b, float)).max())
    assert np.array_equal(s.mesh_translation(), m.D)
    assert s.last_status == 0


def test_mesh_removed_is_plain_dem():
    """set_mesh with no triangles: the solver is the plain DEM again."""
    sc = S.mesh_hopper(n=384, nsteps=300, band=0.002, drop_speed=4.0)
    s = api.from_scenario(sc)
    s.set_mesh(np.zeros((0, 3, 3)), 1.0, 0.25, 1.0)
    s.run_steps(300)
    ref = sc.state.copy()
    O.run(ref, sc.walls.copy(), sc.params, sc.dt, 300, skin=sc.skin, gravity=sc.gravity, pow_mode=O.POW_SQRT)
    got = s.particles.download()
    for f in ("x", "u", "omega"):
        assert np.array_equal(getattr(got, f), getattr(ref, f)), f


def test_set_mesh_rejects_bad_arguments():
    """More than 4,096 triangles, max_contacts outside 1..16 or a non-positive modulus are
    refused with DEM_ERR_INVALID and leave the solver as it was: the next steps are the plain
    DEM's, bit for bit."""
    from cabanadem_b200._lib import DemError
    sc = S.mesh_hopper(n=384, nsteps=200, band=0.002, drop_speed=4.0)
    tri = np.asarray(sc.extra["mesh"].tri).reshape(-1, 3, 3)
    s = api.from_scenario(sc)
    s.set_mesh(np.zeros((0, 3, 3)), 1.0, 0.25, 1.0)
    for args, kw, what in ((np.zeros((4097, 3, 3)), {}, "triangles"),
                           (tri, {"max_contacts": 0}, "max_contacts"),
                           (tri, {"max_contacts": 17}, "max_contacts"),
                           (tri, {"E": 0.0}, "E, G")):
        p = {"E": 1e9, "nu": 0.25, "G": 4e8, **kw}
        mc = p.pop("max_contacts", 8)
        with pytest.raises(DemError, match=what):
            s.set_mesh(args, p["E"], p["nu"], p["G"], max_contacts=mc)
    s.run_steps(200)
    ref = sc.state.copy()
    O.run(ref, sc.walls.copy(), sc.params, sc.dt, 200, skin=sc.skin, gravity=sc.gravity, pow_mode=O.POW_SQRT)
    got = s.particles.download()
    for f in ("x", "u", "omega"):
        assert np.array_equal(getattr(got, f), getattr(ref, f)), f
