"""Learned surrogate on the GPU: gradients of the library's forward/backward kernels against
the CPU restatement of the network, the DEM fallback (a rejected stride leaves exactly the
DEM trajectory), and what a trained network gains over the method without it."""
import numpy as np
import pytest
import torch

from cabanadem_b200 import api, scenarios as S, surrogate as SG
from oracle import gnn_oracle as G

pytestmark = pytest.mark.gpu


def _setup(n=400, strides=8, aspect=1.0, seed=3, max_nodes=4096):
    ctx = api.Context(0)
    sc = S.dam_break(n=n, aspect=aspect, seed=seed)
    traj, rad, _ = SG.record_rollout(sc, ctx, strides)
    prm = SG.params_for(sc, sigma_a=2.0e-4, max_nodes=max_nodes, max_frames=4)
    return ctx, sc, traj, rad, prm


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _cos(a, b):
    return float(np.dot(a, b) / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("two_frames", [False, True])
def test_gradients_match_cpu_oracle(two_frames):
    ctx, sc, traj, rad, prm = _setup()
    sg = SG.Surrogate(ctx, prm)
    sg.init_params(7)
    with torch.cuda.stream(sg.stream):
        if two_frames:   # two frames at overlapping coordinates: edges must stay inside a frame
            prev, cur, nxt, rad2, frame = SG.batch([(traj, rad)], [(0, 4), (0, 6)], traj.device)
        else:
            prev, cur, nxt, rad2 = traj[4].contiguous(), traj[5].contiguous(), traj[6].contiguous(), rad
            frame = None
    nframes = 2 if two_frames else 1
    loss, g = sg.loss_grad(prev, cur, nxt, rad2, frame, nframes)
    flat = sg.get_params()
    fr = frame.cpu().numpy() if frame is not None else None
    loss_o, g_o, _ = G.loss_and_grad(flat, SG.prm_dict(prm), prev.cpu().numpy(), cur.cpu().numpy(),
                                     nxt.cpu().numpy(), rad2.cpu().numpy(), fr, q=G.bf16)
    assert abs(loss - loss_o) <= 1e-3 * abs(loss_o)
    o = 0
    for kin, nout in G.SHAPES:
        for size in (G.H * kin, G.H, nout * G.H, nout):
            a, b = g[o:o + size].astype(np.float64), g_o[o:o + size]
            o += size
            if np.linalg.norm(b) == 0.0:
                assert np.linalg.norm(a) == 0.0
                continue
            assert _rel(a, b) <= 2e-2, (kin, nout, size, _rel(a, b))
            assert _cos(a, b) >= 0.999, (kin, nout, size, _cos(a, b))
    sg.close()
    ctx.close()


def test_rollout_without_network_is_plain_dem():
    ctx = api.Context(0)
    sc = S.dam_break(n=600, aspect=2.0, seed=4)
    prm = SG.params_for(sc, sigma_a=2.0e-4, max_nodes=1024)
    a = api.from_scenario(sc, ctx=ctx)
    sg = SG.Surrogate(ctx, prm)
    st = sg.rollout(a, 6, use_network=False)
    assert st["strides_dem"] == 6 and st["strides_network"] == 0
    b = api.from_scenario(S.dam_break(n=600, aspect=2.0, seed=4), ctx=ctx)
    b.run_steps(6 * SG.STRIDE)
    sa, sb = a.particles.download(), b.particles.download()
    for f in ("x", "u", "omega", "force", "torque", "tng_count"):
        assert np.array_equal(getattr(sa, f), getattr(sb, f)), f
    sg.close()
    ctx.close()


def test_rejected_strides_fall_back_to_exact_dem():
    """A network that violates the overlap bound every stride: every stride is run by DEM from
    the state before it, so the result is the DEM trajectory bit for bit."""
    ctx = api.Context(0)
    sc = S.dam_break(n=600, aspect=2.0, seed=4)
    prm = SG.params_for(sc, sigma_a=1.0, max_nodes=1024)   # sigma_a = 1 m: huge predicted moves
    sg = SG.Surrogate(ctx, prm)
    sg.init_params(3)
    a = api.from_scenario(sc, ctx=ctx)
    st = sg.rollout(a, 5, use_network=True)
    assert st["strides_network"] == 0 and st["strides_dem"] == 5
    assert st["fallback_overlap"] + st["fallback_energy"] == 4
    b = api.from_scenario(S.dam_break(n=600, aspect=2.0, seed=4), ctx=ctx)
    b.run_steps(5 * SG.STRIDE)
    sa, sb = a.particles.download(), b.particles.download()
    for f in ("x", "u", "omega"):
        assert np.array_equal(getattr(sa, f), getattr(sb, f)), f
    sg.close()
    ctx.close()


def test_trained_network_beats_extrapolation():
    """After a short training run on DEM rollouts the network's one-stride prediction error on
    held-out frames of another column is below that of the method without it (constant
    displacement, which is what the network starts from)."""
    ctx = api.Context(0)
    train = []
    for k, a in enumerate((1.0, 3.0)):
        sc = S.dam_break(n=1500, aspect=a, seed=20 + k)
        traj, rad, _ = SG.record_rollout(sc, ctx, 80)
        train.append((traj, rad))
    sig = SG.sigma_a_of(train)
    test_sc = S.dam_break(n=1500, aspect=2.0, seed=30)
    test_traj, test_rad, _ = SG.record_rollout(test_sc, ctx, 80)
    prm = SG.params_for(test_sc, sigma_a=sig, max_nodes=8 * 1500, max_frames=8)
    sg = SG.Surrogate(ctx, prm)
    sg.init_params(1)
    z = sg.get_params()
    o = sum(G.H * kin + G.H + nout * G.H + nout for kin, nout in G.SHAPES[:-1])
    z[o + G.H * G.H + G.H:] = 0.0          # decoder output layer zeroed: prediction = constant displacement
    sg.set_params(z)

    def err(net):
        e = []
        for k in range(10, 79, 6):
            pred = net.predict(test_traj[k - 1], test_traj[k], test_rad)
            torch.cuda.synchronize()
            d = (pred - test_traj[k + 1])[:, :2]
            e.append(float((d * d).sum()))
        return float(np.sum(e))

    e0 = err(sg)
    losses = SG.train(sg, train, steps=400, batch_frames=4, lr0=1e-3, lr1=1e-4, seed=2)
    e1 = err(sg)
    assert np.mean(losses[-50:]) < np.mean(losses[:50])
    assert e1 < e0, (e1, e0)
    sg.close()
    ctx.close()
