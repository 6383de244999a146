"""Train the dam-break surrogate on DEM rollouts and save its weights.

    python -m cabanadem_b200.train_surrogate --out cabanadem_b200/data/dam_break_surrogate.npz

Training columns (seeded): `--columns` dam breaks of n ~ U[n_min, n_max] disks and aspect
ratio ~ U[0.5, 4] run together as independent scenes of one DEM batch for `--seconds`,
recorded every stride (200 steps) into device memory; then `--steps` Adam steps on batches
of `--batch` random frames with input noise `--noise` x sigma_a.  Everything is seeded, and
the GPU reductions are fixed-order, so a rerun reproduces the weights."""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import api, scenarios as S, surrogate as SG


def make_columns(k, n_min, n_max, seed):
    rng = np.random.default_rng(seed)
    cols = []
    for c in range(k):
        n = int(rng.integers(n_min, n_max + 1))
        a = float(rng.uniform(0.5, 4.0))
        cols.append(S.dam_break(n=n, aspect=a, seed=seed * 1000 + c))
    return cols


def record_columns(ctx, cols, strides):
    """One batched DEM run of all columns; returns [(traj view [frames, n_k, 3], rad_k)]."""
    batch = S.combine_scenes(cols, "dam_break_columns")
    traj, rad, secs = SG.record_rollout(batch, ctx, strides)
    out, off = [], 0
    for sc in cols:
        c = sc.state.n
        out.append((traj[:, off:off + c], rad[off:off + c]))
        off += c
    return out, secs, batch.state.n


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--out", required=True)
    ap.add_argument("--columns", type=int, default=8)
    ap.add_argument("--n-min", type=int, default=8000)
    ap.add_argument("--n-max", type=int, default=30000)
    ap.add_argument("--seconds", type=float, default=1.0)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--noise", type=float, default=0.5, help="input noise std in units of sigma_a")
    ap.add_argument("--lr0", type=float, default=1e-3)
    ap.add_argument("--lr1", type=float, default=1e-5)
    ap.add_argument("--seed", type=int, default=7)
    args = ap.parse_args(argv)

    ctx = api.Context(0)
    cols = make_columns(args.columns, args.n_min, args.n_max, args.seed)
    strides = int(round(args.seconds / (SG.STRIDE * cols[0].dt)))
    trajs, dem_secs, ntot = record_columns(ctx, cols, strides)
    sig = SG.sigma_a_of(trajs)
    maxn = args.batch * max(sc.state.n for sc in cols)
    prm = SG.params_for(cols[0], sigma_a=sig, max_nodes=maxn, max_frames=args.batch)
    sg = SG.Surrogate(ctx, prm)
    sg.init_params(args.seed)
    t0 = time.perf_counter()
    losses = SG.train(sg, trajs, steps=args.steps, batch_frames=args.batch, lr0=args.lr0, lr1=args.lr1,
                      noise=args.noise * sig, seed=args.seed)
    torch.cuda.synchronize()
    train_secs = time.perf_counter() - t0
    meta = dict(sigma_a=sig, radius_graph=prm.radius_graph, sigma_d=prm.sigma_d, wall_clip=prm.wall_clip,
                steps_per_stride=SG.STRIDE, dt=cols[0].dt, columns=args.columns, n_min=args.n_min, n_max=args.n_max,
                seconds=args.seconds, steps=args.steps, batch=args.batch, noise=args.noise, seed=args.seed,
                dem_particles=ntot, dem_seconds=dem_secs, train_seconds=train_secs,
                loss_first=float(np.mean(losses[:50])), loss_last=float(np.mean(losses[-50:])))
    np.savez(args.out, params=sg.get_params(), meta=json.dumps(meta), losses=np.asarray(losses, dtype=np.float32))
    print(json.dumps(meta))
    sg.close()
    ctx.close()


if __name__ == "__main__":
    main()
