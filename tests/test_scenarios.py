"""The seeded benchmark workloads are what their descriptions say (CPU, reduced sizes of the
same generators): no initial overlap, radii, velocities and positions in the stated ranges,
particles inside their walls, scene sizes log-uniform in [2, 8192]."""
import numpy as np
import pytest
from scipy.spatial import cKDTree

from cabanadem_b200 import scenarios as S


def _min_gap(x, rad):
    """Smallest surface gap over all pairs closer than 2 r_max (inf if none)."""
    pairs = cKDTree(x).query_pairs(2.0 * rad.max(), output_type="ndarray")
    if len(pairs) == 0:
        return np.inf
    d = np.linalg.norm(x[pairs[:, 0]] - x[pairs[:, 1]], axis=1)
    return float((d - rad[pairs[:, 0]] - rad[pairs[:, 1]]).min())


def _inside_walls(st, w):
    """Signed distance of every sphere surface from every wall plane (>= 0: no overlap)."""
    d = ((st.x[:, None, :] - w.x[None, :, :]) * w.normal[None, :, :]).sum(-1) - st.rad[:, None]
    return float(d.min())


def test_hcp_box():
    sc = S.hcp_box(n=20000)
    st = sc.state
    assert st.n == 20000 and sc.dt == 5e-8
    assert st.rad.min() >= 0.8e-3 and st.rad.max() <= 1.2e-3
    assert _min_gap(st.x, st.rad) > 0.0
    assert _inside_walls(st, sc.walls) >= 0.0
    assert np.abs(st.u).max() <= 0.1
    assert sc.gravity == (0.0, 0.0, -9.81) and sc.skin == pytest.approx(0.1 * st.rad.mean(), rel=0.05)


def test_random_box():
    sc = S.random_box(n=1000)
    st = sc.state
    assert np.all(st.rad == 1e-3) and _min_gap(st.x, st.rad) >= 0.0
    assert st.x.min() >= 1e-3 and st.x.max() <= 0.05 - 1e-3
    assert np.abs(st.u).max() <= 0.1 and sc.dt == 1e-7
    with pytest.raises(ValueError):
        S.random_box(n=200, side=0.006)        # cannot be placed: refused, not an endless loop


def test_dam_break():
    sc = S.dam_break(n=5000, aspect=2.0, seed=101)
    st = sc.state
    assert np.all(st.x[:, 2] == 0.0)            # disks in the plane z = 0
    assert st.rad.min() >= 0.9e-3 and st.rad.max() <= 1.1e-3
    assert _min_gap(st.x, st.rad) > 0.0
    assert _inside_walls(st, sc.walls) >= 0.0
    assert not st.u.any()                       # released at rest
    h = st.x[:, 1].max() - st.x[:, 1].min()
    wdt = st.x[:, 0].max() - st.x[:, 0].min()
    assert 1.6 < h / wdt < 2.4                  # column of aspect 2


def test_batched_scenes():
    sc = S.batched_scenes(nscenes=64, seed=3)
    scene = sc.extra["scene"]
    counts = np.bincount(scene)
    assert len(counts) == 64 and counts.min() >= 2 and counts.max() <= 8192
    assert 0.5 < np.log(counts).std() / (np.log(8192 / 2) / np.sqrt(12)) < 1.5   # log-uniform spread
    st = sc.state
    for k in range(64):
        sel = scene == k
        assert _min_gap(st.x[sel], st.rad[sel]) > 0.0, k
    prm = np.array(sc.extra["scene_params"])
    assert prm[:, 0].min() >= 0.3 and prm[:, 0].max() <= 0.95          # restitution
    assert prm[:, 2].min() >= 0.1 and prm[:, 2].max() <= 0.5           # friction


def test_bonded_bar():
    case = S.bonded_bar(nx=8, ny=4, nz=2)
    st = case["state"]
    assert st.n == 64 and np.all(st.rad == 0.5e-3)
    assert _min_gap(st.x, st.rad) == pytest.approx(0.0, abs=1e-12)   # touching on the 1 mm lattice
    left, right = st.x[:, 0] == st.x[:, 0].min(), st.x[:, 0] == st.x[:, 0].max()
    assert np.all(st.u[left, 0] == -0.05) and np.all(st.u[right, 0] == 0.05)
    assert np.all(case["fix_flags"][left | right] == 3)


def test_state_resized():
    """ParticleState.resized (the host half of Particles.resize, Particles.hpp:273-297): the
    first particles keep every field, added ones are zeroed with empty contact slots."""
    st = S.random_box(n=50).state
    st.tng_idx[:5, 0], st.tng_count[:5] = 7, 1
    grow, shrink = st.resized(80), st.resized(20)
    for name, a in st.arrays().items():
        assert np.array_equal(getattr(grow, name)[:50], a), name
        assert np.array_equal(getattr(shrink, name), a[:20]), name
    assert not grow.x[50:].any() and not grow.m[50:].any() and not grow.tng_count[50:].any()
    assert np.all(grow.tng_idx[50:] == -1)
    assert grow.n == 80 and shrink.n == 20 and grow.tng_sw_x.shape == (80, st.tng_sw_x.shape[1])
