"""The CPU restatement of the surrogate network: its backward pass against central finite
differences of its own float64 forward pass (the oracle that the GPU gradients are then
checked against)."""
import numpy as np

from oracle import gnn_oracle as G

PRM = dict(radius_graph=3.0e-3, sigma_d=1.0e-3, sigma_a=2.0e-4, r_mean=1.0e-3, r_std=5.8e-5, wall_clip=5.0e-3,
           walls=[((0.0, 0.0, 0.0), (0.0, 1.0, 0.0)), ((0.0, 0.0, 0.0), (1.0, 0.0, 0.0))])


def _case(n=12, seed=0):
    rng = np.random.default_rng(seed)
    cur = np.zeros((n, 3))
    cur[:, 0] = rng.uniform(1e-3, 7e-3, n)
    cur[:, 1] = rng.uniform(1e-3, 5e-3, n)
    prev = cur.copy()
    prev[:, :2] -= rng.normal(0, 3e-4, (n, 2))
    nxt = cur.copy()
    nxt[:, :2] += (cur[:, :2] - prev[:, :2]) + rng.normal(0, 2e-4, (n, 2))
    rad = rng.uniform(0.9e-3, 1.1e-3, n)
    return prev, cur, nxt, rad


def _params(seed=1):
    rng = np.random.default_rng(seed)
    parts = []
    for kin, nout in G.SHAPES:
        parts += [rng.normal(0, (2.0 / kin) ** 0.5, G.H * kin), rng.normal(0, 0.1, G.H),
                  rng.normal(0, (1.0 / G.H) ** 0.5, nout * G.H), rng.normal(0, 0.1, nout)]
    return np.concatenate(parts)


def test_graph_is_symmetric_and_sorted():
    prev, cur, nxt, rad = _case(30)
    recv, send, offs = G.graph(cur, np.zeros(30, dtype=int), PRM["radius_graph"])
    assert len(recv) > 0
    assert np.all(G.reverse_edges(recv, send) >= 0)
    for i in range(30):
        s = send[offs[i]:offs[i + 1]]
        assert np.all(np.diff(s) > 0)


def test_backward_matches_finite_differences():
    prev, cur, nxt, rad = _case()
    flat = _params()
    loss, g, _ = G.loss_and_grad(flat, PRM, prev, cur, nxt, rad)
    rng = np.random.default_rng(5)
    # offsets of every layer's four tensors; sample parameters in each
    checks, o = [], 0
    for kin, nout in G.SHAPES:
        for size in (G.H * kin, G.H, nout * G.H, nout):
            checks += list(o + rng.integers(0, size, 2))
            o += size
    errs = []
    for k in checks:
        eps = 1e-6 * max(1.0, abs(flat[k]))
        fp, fm = flat.copy(), flat.copy()
        fp[k] += eps
        fm[k] -= eps
        lp = G.loss_and_grad(fp, PRM, prev, cur, nxt, rad)[0]
        lm = G.loss_and_grad(fm, PRM, prev, cur, nxt, rad)[0]
        fd = (lp - lm) / (2 * eps)
        errs.append(abs(fd - g[k]) / (abs(g).max() + 1e-300))
    errs = np.asarray(errs)
    assert np.median(errs) < 1e-7
    assert np.mean(errs < 1e-5) >= 0.9      # a parameter whose unit sits on a ReLU kink may differ
    assert errs.max() < 1e-3
