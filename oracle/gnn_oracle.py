"""CPU restatement of the learned surrogate's network, for checking the GPU kernels.

TEST INFRASTRUCTURE ONLY: imported by tests, never by the library.

Follows cabanadem_b200/csrc/dem_surrogate.cu (graph, features, network, loss, backward) and
cabanadem_b200/csrc/dem_nn.cu (two-layer perceptron y = W2 relu(W1 x + b1) + b2 (+ res)).
The network has no counterpart in the reference (CabanaDEM has no learned component); it is
restated here from our own design so that the GPU forward/backward can be compared with an
independent implementation.

Arithmetic is float64.  With `q=bf16` every value that the GPU stores in BF16 (features,
weights, hidden activations, latents, aggregates, upstream gradients) is rounded to BF16
(round to nearest even, via float32) at the same point, so the comparison isolates
summation order; with `q=None` the network is exact float64 (used for finite differences).
"""
from __future__ import annotations

import numpy as np

H = 128
F = 16
SHAPES = [(16, 128), (16, 128), (384, 128), (256, 128), (384, 128), (256, 128), (384, 128), (256, 128), (128, 16)]
ENC_N, ENC_E, DEC = 0, 1, 8


def MSG(l):
    return 2 + 2 * l


def UPD(l):
    return 3 + 2 * l


def bf16(x):
    """Round to BF16 (nearest even) through float32; returns float64."""
    f = np.asarray(x, dtype=np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def f32(x):
    return np.asarray(x, dtype=np.float32).astype(np.float64)


def _id(x):
    return np.asarray(x, dtype=np.float64)


def unpack(flat):
    """Flat FP32 parameter vector (dem_surrogate_get_params layout) -> per-layer dicts."""
    flat = np.asarray(flat, dtype=np.float64)
    out, o = [], 0
    for kin, nout in SHAPES:
        p = {}
        p["w1t"] = flat[o:o + H * kin].reshape(H, kin); o += H * kin
        p["b1"] = flat[o:o + H]; o += H
        p["w2t"] = flat[o:o + nout * H].reshape(nout, H); o += nout * H
        p["b2"] = flat[o:o + nout]; o += nout
        out.append(p)
    assert o == flat.size
    return out


def pack(layers):
    return np.concatenate([np.concatenate([p["w1t"].ravel(), p["b1"], p["w2t"].ravel(), p["b2"]]) for p in layers])


def graph(cur, frame, radius):
    """Edges (i <- j), j != i, same frame, |x_i - x_j| <= radius (2D), sorted by (i, j)."""
    n = cur.shape[0]
    recv, send = [], []
    for i in range(n):
        d = cur[:, :2] - cur[i, :2]
        r2 = d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]
        ok = (r2 <= radius * radius) & (frame == frame[i])
        ok[i] = False
        js = np.nonzero(ok)[0]
        recv.extend([i] * len(js))
        send.extend(js.tolist())
    recv = np.asarray(recv, dtype=np.int64)
    send = np.asarray(send, dtype=np.int64)
    offs = np.zeros(n + 1, dtype=np.int64)
    np.add.at(offs, recv + 1, 1)
    return recv, send, np.cumsum(offs)


def features(prev, cur, rad, recv, send, prm):
    disp = cur[:, :2] - prev[:, :2]
    n = cur.shape[0]
    xn = np.zeros((n, F))
    xn[:, 0:2] = disp / prm["sigma_d"]
    for w, (wx, wn) in enumerate(prm["walls"]):
        wn = np.asarray(wn[:2], dtype=np.float64)
        wn = wn / np.linalg.norm(wn)
        dist = (cur[:, 0] - wx[0]) * wn[0] + (cur[:, 1] - wx[1]) * wn[1] - rad
        xn[:, 2 + w] = np.clip(dist / prm["wall_clip"], -1.0, 1.0)
    xn[:, 6] = (rad - prm["r_mean"]) / prm["r_std"]
    ne = len(recv)
    xe = np.zeros((ne, F))
    if ne:
        dx = cur[send, :2] - cur[recv, :2]
        dist = np.sqrt(dx[:, 0] ** 2 + dx[:, 1] ** 2)
        xe[:, 0:2] = dx / prm["radius_graph"]
        xe[:, 2] = dist / prm["radius_graph"]
        xe[:, 3] = (dist - rad[recv] - rad[send]) / prm["r_mean"]
        xe[:, 4:6] = (disp[send] - disp[recv]) / prm["sigma_d"]
    return xn, xe, disp


class Net:
    def __init__(self, flat, q=None):
        self.layers = unpack(flat)
        self.q = q or _id
        self.f = f32 if q else _id
        # weights as the GPU reads them
        self.W = [{"w1t": self.q(p["w1t"]), "b1": self.f(p["b1"]), "w2t": self.q(p["w2t"]), "b2": self.f(p["b2"])}
                  for p in self.layers]

    def mlp(self, l, x, resid=None, out_q=True):
        W, q, f = self.W[l], self.q, self.f
        h = q(np.maximum(f(x @ W["w1t"].T) + W["b1"], 0.0))
        y = f(h @ W["w2t"].T) + W["b2"]
        if resid is not None:
            y = f(y + resid)
        return (q(y) if out_q else f(y)), h

    def mlp_back(self, l, x, h, dy, want_dx):
        """dy (already rounded as the GPU's BF16 upstream gradient) -> dx, grads."""
        W, q, f = self.W[l], self.q, self.f
        dz = q(f(dy @ W["w2t"]) * (h > 0))
        g = {"w1t": dz.T @ x, "b1": dz.sum(0), "w2t": dy.T @ h, "b2": dy.sum(0)}
        dx = f(dz @ W["w1t"]) if want_dx else None
        return dx, g

    def msg(self, l, e, h, recv, send):
        """Edge update e + W2 relu(W1e e + P[recv] + Q[send] + b1) + b2 with P = W1i h, Q = W1j h
        (W1 = [W1e | W1i | W1j]); P and Q are stored in BF16 on the GPU."""
        W, q, f = self.W[l], self.q, self.f
        w1 = W["w1t"]
        P = q(f(h @ w1[:, H:2 * H].T))
        Q = q(f(h @ w1[:, 2 * H:].T))
        z = f(f(f(e @ w1[:, :H].T) + W["b1"]) + P[recv] + Q[send])
        h1 = q(np.maximum(z, 0.0))
        y = f(f(h1 @ W["w2t"].T) + f(W["b2"] + e))
        return q(y), h1

    def msg_back(self, l, e, h, h1, dy, recv, send, rev):
        """-> dE (input latent), dh contribution, grads (BF16 dz, dP, dQ as on the GPU)."""
        W, q, f = self.W[l], self.q, self.f
        w1 = W["w1t"]
        n = h.shape[0]
        dz = q(f(dy @ W["w2t"]) * (h1 > 0))
        dE = f(dz @ w1[:, :H])
        dP = np.zeros((n, H))
        np.add.at(dP, recv, dz)
        dQ = np.zeros((n, H))
        ok = rev >= 0
        np.add.at(dQ, recv[ok], dz[rev[ok]])
        dP, dQ = q(f(dP)), q(f(dQ))
        dh = f(dP @ w1[:, H:2 * H] + dQ @ w1[:, 2 * H:])
        gw1t = np.concatenate([dz.T @ e, dP.T @ h, dQ.T @ h], axis=1)
        g = {"w1t": gw1t, "b1": dz.sum(0), "w2t": dy.T @ h1, "b2": dy.sum(0)}
        return dE, dh, g

    def forward(self, xn, xe, recv, send, offs):
        q = self.q
        n = xn.shape[0]
        c = {"xn": q(xn), "xe": q(xe)}
        c["h"], c["e"], c["agg"], c["h1"] = [None] * 4, [None] * 4, [None] * 3, [None] * 9
        c["h"][0], c["h1"][ENC_N] = self.mlp(ENC_N, c["xn"])
        c["e"][0], c["h1"][ENC_E] = self.mlp(ENC_E, c["xe"])
        for l in range(3):
            c["e"][l + 1], c["h1"][MSG(l)] = self.msg(MSG(l), c["e"][l], c["h"][l], recv, send)
            agg = np.zeros((n, H))
            np.add.at(agg, recv, c["e"][l + 1])
            c["agg"][l] = q(self.f(agg))
            xu = np.concatenate([c["h"][l], c["agg"][l]], axis=1)
            c["h"][l + 1], c["h1"][UPD(l)] = self.mlp(UPD(l), xu, resid=c["h"][l])
        out, c["h1"][DEC] = self.mlp(DEC, c["h"][3], out_q=False)
        return out, c

    def backward(self, dout, c, recv, send, rev):
        q, f = self.q, self.f
        n = c["h"][0].shape[0]
        ne = len(recv)
        grads = [None] * 9
        dh, grads[DEC] = self.mlp_back(DEC, c["h"][3], c["h1"][DEC], dout, True)
        de = np.zeros((ne, H))
        for l in (2, 1, 0):
            xu = np.concatenate([c["h"][l], c["agg"][l]], axis=1)
            dxn, grads[UPD(l)] = self.mlp_back(UPD(l), xu, c["h1"][UPD(l)], q(dh), True)
            dh = f(dh + dxn[:, :H])
            de = f(de + dxn[recv, H:])
            dE, dhm, grads[MSG(l)] = self.msg_back(MSG(l), c["e"][l], c["h"][l], c["h1"][MSG(l)], q(de), recv, send,
                                                   rev)
            dh = f(dh + dhm)
            de = f(de + dE)
        _, grads[ENC_E] = self.mlp_back(ENC_E, c["xe"], c["h1"][ENC_E], q(de), False)
        _, grads[ENC_N] = self.mlp_back(ENC_N, c["xn"], c["h1"][ENC_N], q(dh), False)
        return grads


def reverse_edges(recv, send):
    key = {(int(i), int(j)): e for e, (i, j) in enumerate(zip(recv, send))}
    return np.array([key.get((int(j), int(i)), -1) for i, j in zip(recv, send)], dtype=np.int64)


def loss_and_grad(flat, prm, prev, cur, nxt, rad, frame=None, q=None):
    """Loss (mean over particles and the two components of (a - target)^2, target the change of
    displacement / sigma_a) and the flat gradient (the GPU's layout)."""
    n = cur.shape[0]
    frame = np.zeros(n, dtype=np.int64) if frame is None else np.asarray(frame)
    recv, send, offs = graph(cur, frame, prm["radius_graph"])
    rev = reverse_edges(recv, send)
    xn, xe, disp = features(prev, cur, rad, recv, send, prm)
    net = Net(flat, q)
    out, c = net.forward(xn, xe, recv, send, offs)
    tgt = ((nxt[:, :2] - cur[:, :2]) - disp) / prm["sigma_a"]
    err = out[:, :2] - tgt
    loss = float((err * err).sum() / (2.0 * n))
    dout = np.zeros((n, F))
    dout[:, :2] = 2.0 * err / (2.0 * n)
    grads = net.backward((q or _id)(f32(dout) if q else dout), c, recv, send, rev)
    return loss, pack(grads), out
