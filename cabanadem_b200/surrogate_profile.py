"""Time network strides of the dam-break surrogate on its own (no DEM run).

    python -m cabanadem_b200.surrogate_profile [--n 200000] [--strides 3]

Builds the dam-break column of n disks (aspect 2), loads the shipped weights and runs
`--strides` network strides (graph build, features, network, wall projection, contact
projection) from the initial lattice with a small downward displacement; prints the mean
wall-clock per stride.  A short, self-contained command for profilers."""
from __future__ import annotations

import argparse
import json
import os
import time

import torch

from . import api, scenarios as S, surrogate as SG


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--n", type=int, default=200_000)
    ap.add_argument("--strides", type=int, default=3)
    args = ap.parse_args(argv)
    ctx = api.Context(0)
    sc = S.dam_break(n=args.n, aspect=2.0, seed=101)
    weights = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "dam_break_surrogate.npz")
    sg = SG.load(ctx, weights, sc)
    x = torch.as_tensor(sc.state.x).cuda()
    x2 = x.clone()
    x2[:, 1] -= 1e-6
    rad = torch.as_tensor(sc.state.rad).cuda()
    sg.predict(x, x2, rad)            # first call sizes the buffers
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.strides):
        sg.predict(x, x2, rad)
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) / max(args.strides, 1) * 1e3
    print(json.dumps({"n": args.n, "strides": args.strides, "ms_per_stride": ms}))
    sg.close()
    ctx.close()


if __name__ == "__main__":
    main()
