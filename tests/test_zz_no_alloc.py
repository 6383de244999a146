"""dem_neighbor_list_noalloc: the neighbour build for callers that cannot allocate device
memory where they need the list (their memory belongs to another allocator, or a cudaMalloc
would stall a time loop that shares the GPU).  It takes the caller's device arrays and uses a
fixed scratch array inside the library instead of allocating.

Checked through the C ABI against the allocating path (dem_build_neighbors, read back with
dem_neighbors_get) on two calls in a row with different inputs, so that contents left in the
shared scratch by the first call cannot leak into the second.  Neighbour indices are integer
results, so the comparison is exact.  This file is collected last on purpose."""
import numpy as np
import pytest

from cabanadem_b200 import _lib, api, scenarios as S

pytestmark = pytest.mark.gpu


def _noalloc(state, delta, skin, max_nb=48):
    import torch
    n = state.n
    x = torch.tensor(state.x, dtype=torch.float64, device="cuda").contiguous()
    r = torch.tensor(state.rad, dtype=torch.float64, device="cuda").contiguous()
    nn = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    idx = torch.full((max_nb * n,), -7, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    st = _lib.lib().dem_neighbor_list_noalloc(x.data_ptr(), r.data_ptr(), n, float(delta), float(skin), max_nb,
                                              nn.data_ptr(), idx.data_ptr(), torch.cuda.current_stream().cuda_stream)
    nn = nn.cpu().numpy()
    idx = idx.cpu().numpy().reshape(max_nb, n)
    off = np.concatenate([[0], np.cumsum(nn)]).astype(np.int32)
    keep = np.arange(max_nb)[None, :] < nn[:, None]
    return st, off, idx.T[keep]


def _allocating(sc):
    s = api.from_scenario(sc, rebuild_every_step=sc.delta > 0)
    s.build_neighbors()
    off, idx = s.neighbors()
    s.close()
    return off, idx


def test_noalloc_matches_allocating_build_twice():
    first = S.random_box(n=4096, seed=11)                 # skin cutoff r_i + r_j + skin
    c = first.state.x.mean(axis=0)
    first.state.x[:] = c + (first.state.x - c) * 0.8
    second = S.random_box(n=3000, seed=12)                 # uniform cutoff, different size
    second.delta = 3.0e-3
    for sc in (first, second):
        st, off, idx = _noalloc(sc.state, sc.delta, sc.skin)
        assert st == 0
        roff, ridx = _allocating(sc)
        assert off[-1] > 0
        assert np.array_equal(off, roff)
        assert np.array_equal(idx, ridx)


def test_noalloc_rejects_too_many_particles():
    assert _lib.NOALLOC_MAX_PARTICLES == 32768
    st = _lib.lib().dem_neighbor_list_noalloc(1, 1, _lib.NOALLOC_MAX_PARTICLES + 1, 0.0, 1e-4, 16, 1, 1, None)
    assert st == 0x001   # DEM_ERR_INVALID, nothing launched


def test_noalloc_rejects_too_many_neighbours_per_particle():
    # the list build keeps DEM_NOALLOC_MAX_NEIGHBORS candidates per particle; a larger list
    # capacity is refused before anything is launched, so nothing is written
    import torch
    sc = S.random_box(n=256, seed=5)
    assert _lib.NOALLOC_MAX_NEIGHBORS == 128
    st, off, idx = _noalloc(sc.state, sc.delta, sc.skin, max_nb=_lib.NOALLOC_MAX_NEIGHBORS)
    assert st == 0
    n = sc.state.n
    nn = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    x = torch.tensor(sc.state.x, dtype=torch.float64, device="cuda")
    r = torch.tensor(sc.state.rad, dtype=torch.float64, device="cuda")
    big = torch.full((200 * n,), -7, dtype=torch.int32, device="cuda")
    st = _lib.lib().dem_neighbor_list_noalloc(x.data_ptr(), r.data_ptr(), n, 0.0, float(sc.skin), 200,
                                              nn.data_ptr(), big.data_ptr(), None)
    assert st == 0x001   # DEM_ERR_INVALID
    torch.cuda.synchronize()
    assert bool((nn == -7).all()) and bool((big == -7).all())


def test_noalloc_cut_lists_on_overflow():
    # a dense cluster with a list capacity of 4: DEM_ERR_NEIGHBOR_OVERFLOW, and each list holds
    # the first 4 partners (ascending index) of the full list the allocating build produces
    sc = S.random_box(n=2048, seed=21)
    c = sc.state.x.mean(axis=0)
    sc.state.x[:] = c + (sc.state.x - c) * 0.5
    st, off, idx = _noalloc(sc.state, sc.delta, sc.skin, max_nb=4)
    assert st == 0x008
    roff, ridx = _allocating(sc)
    full = np.diff(roff)
    assert full.max() > 4
    cut = np.minimum(full, 4)
    assert np.array_equal(np.diff(off), cut)
    for i in range(sc.state.n):
        assert np.array_equal(idx[off[i]:off[i + 1]], ridx[roff[i]:roff[i] + cut[i]])


def test_noalloc_non_finite_position_empties_every_list():
    sc = S.random_box(n=1024, seed=23)
    sc.state.x[17, 1] = np.nan
    st, off, idx = _noalloc(sc.state, sc.delta, sc.skin)
    assert st == 0x010   # DEM_ERR_NAN
    assert off[-1] == 0
    # the next call on clean input starts from a cleared status and gives the full list
    good = S.random_box(n=1024, seed=23)
    st, off, idx = _noalloc(good.state, good.delta, good.skin)
    assert st == 0
    roff, ridx = _allocating(good)
    assert np.array_equal(off, roff) and np.array_equal(idx, ridx)
