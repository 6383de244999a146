"""Time the fused DEM step on a scenario, optionally from a saved state (for profilers).

    python -m cabanadem_b200.dem_profile --scenario dam_break --n 200000 --advance 300000 \\
        --save /tmp/dam.ckpt --steps 0
    python -m cabanadem_b200.dem_profile --scenario dam_break --n 200000 --load /tmp/dam.ckpt \\
        --steps 60 [--precision mixed] [--contact-lanes 8]

The first form runs `--advance` steps from the scenario's initial state and saves the particle
state (a dense phase of a flow, for instance); the second loads it and runs `--steps` more,
printing the device time per step (CUDA events on the library's stream) and the solver
statistics as one JSON line.  A short, self-contained command for ncu captures of a late
phase without running the steps that lead to it under the profiler."""
from __future__ import annotations

import argparse
import json

import torch

from . import api, scenarios as S
from ._lib import DEM_FP64, DEM_MIXED

SCENARIOS = {
    "dam_break": lambda n: S.dam_break(n=n, aspect=2.0, seed=101),
    "hcp_box": lambda n: S.hcp_box(n=n, seed=2),
    "random_box": lambda n: S.random_box(n=n),
}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--scenario", choices=sorted(SCENARIOS), default="dam_break")
    ap.add_argument("--n", type=int, default=200_000)
    ap.add_argument("--advance", type=int, default=0, help="steps to run before saving")
    ap.add_argument("--save", default="")
    ap.add_argument("--load", default="")
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--precision", choices=("fp64", "mixed"), default="fp64")
    ap.add_argument("--contact-lanes", type=int, default=0)
    args = ap.parse_args(argv)
    ctx = api.Context(0)
    s = api.from_scenario(SCENARIOS[args.scenario](args.n), ctx=ctx,
                          precision=DEM_MIXED if args.precision == "mixed" else DEM_FP64,
                          contact_lanes=args.contact_lanes)
    out = {"scenario": args.scenario, "n": args.n, "precision": args.precision,
           "contact_lanes": args.contact_lanes}
    if args.load:
        s.particles.load(args.load)
    if args.advance > 0:
        s.run_steps(args.advance)
        out["advanced"] = args.advance
    if args.save:
        s.particles.save(args.save)
        out["saved"] = args.save
    if args.steps > 0:
        stream = torch.cuda.ExternalStream(ctx.stream_ptr())
        s.run_steps(min(args.steps, 64))            # graph capture, density switch and build outside the window
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.run_steps(args.steps)
        e1.record(stream)
        e1.synchronize()
        out["us_per_step"] = round(e0.elapsed_time(e1) / args.steps * 1e3, 2)
    out["stats"] = s.stats()
    print(json.dumps(out))
    s.close()
    s.particles.close()
    ctx.close()


if __name__ == "__main__":
    main()
