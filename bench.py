#!/usr/bin/env python
"""Throughput of the DEM contact step on one or more B200s (particle-steps/s).

Workload: 2,000,000 polydisperse glass spheres (r ~ U[0.8, 1.2] mm) on a jittered
hexagonal-close-packed lattice in a 6-wall box, gravity on, dt = 5e-8 s, 2,000 steps,
Verlet skin 0.1 r_mean with rebuild when the displacement bound reaches skin/2
(seeded synthetic input, `cabanadem_b200.scenarios.hcp_box`).

  python bench.py [--gpus N --steps K --warmup W] [--precision fp64|mixed]
  python bench.py --impl reference ...   # the reference algorithm on the host cores
  python bench.py --workload random_box|batched|bonded|dam_break   # the other configurations

The other workloads (one JSON line each, device-timed particle-steps/s):
  random_box  4,096 r = 1 mm spheres in a 5 cm walled cube, dt 1e-7 (latency-bound size)
  batched     1,024 independent scenes of log-uniform [2, 8192] spheres fired at their own
              walls, FP32 forces / FP64 state, grouped by scene size, each group a solver with
              launch settings from the autotuner, the groups concurrent
  bonded      256 x 64 x 8 bonded bar pulled at both ends, FP64
  dam_break   200,000 quasi-2D disks: full DEM rollout vs the learned surrogate with DEM
              fallback over the same simulated time (wall-clock of each, runout front and
              deposit profile errors against DEM)
  dense       the 200,000-disk dam break advanced --dense-advance steps (or loaded from
              --load), then --steps timed steps; --save writes the advanced state, so that a
              profiler can start from it without running the steps that lead to it
  surrogate_stride  --steps network strides of the dam-break surrogate on 200,000 disks
              (graph, features, network, projections; mean wall-clock per stride)

Prints one JSON line (rank 0).  `value` is device-timed (CUDA events on the library's
stream, inputs resident in HBM); `e2e` is the same metric through the C ABI with host
buffers (upload of the fields a new run sets, steps, download of the state, all inside the
timed region); `roofline` is the fused step's algorithmic bytes per step over its
CUDA-event-timed device time per step in the timed region; `cpu_baseline` is the CPU
oracle (a C++ restatement of the reference's step, run in the reference's
rebuild-every-step mode) on a bounded sample of the same workload.  Three device-timed
sub-measurements follow the timed region on the same GPU and are reported beside it:
`mixed` (the same lattice with FP32 contact forces), `dense` (the 200,000-disk dam break
at t = 0.3 s, a contact-dense flow, FP64 and mixed) and `rebuild` (one full neighbour
rebuild of the 2,000,000-sphere state); then the other configurations, each measured as its
own workload above measures it: `c1` (random_box), `c3` (batched, with the packaged B200
launch settings), `c4` (bonded) and `c5` (dam_break over --seconds; --seconds 0 skips it).
--no-configs skips those four.
"""
from __future__ import annotations

import argparse
import atexit
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "particle-steps/s"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--n", type=int, default=2_000_000)
    ap.add_argument("--cpu-seconds", type=float, default=20.0, help="budget of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="hcp",
                    choices=["hcp", "random_box", "batched", "bonded", "dam_break", "dense", "surrogate_stride"])
    ap.add_argument("--save", default="", help="dense: checkpoint the state after --dense-advance steps")
    ap.add_argument("--load", default="", help="dense: start from a checkpoint instead of advancing")
    ap.add_argument("--contact-lanes", type=int, default=0, help="dense: contact kernel form (0 automatic)")
    ap.add_argument("--dense-form", type=int, default=0, help="dense: 1 one kernel, 2 pair-parallel (0 automatic)")
    ap.add_argument("--stream-split", type=int, default=0,
                    help="hcp: streaming pass form (0 automatic: 4, staged tiles; 1 one thread per particle)")
    ap.add_argument("--steps-per-launch", type=int, default=0,
                    help="0: the step loop as a graph while-loop; else steps per captured graph (for profilers)")
    ap.add_argument("--seconds", type=float, default=0.25, help="dam_break: simulated time of both rollouts")
    ap.add_argument("--sub-steps", type=int, default=1000,
                    help="steps timed in each sub-measurement (mixed, dense); at least --steps")
    ap.add_argument("--dense-advance", type=int, default=300_000,
                    help="steps of the dam break run before the dense measurement (0: no dense measurement)")
    ap.add_argument("--no-sub", action="store_true", help="skip the mixed, dense and rebuild sub-measurements")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the C1, C3, C4 and C5 sub-measurements of the headline line")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(x: float) -> float:
    """The largest value of x over all ranks (the job's time is its slowest rank's); x on a
    single rank.  Works with the nccl (GPU tensor) and gloo (CPU tensor) backends."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def hbm_peak():
    try:
        with open(PEAKS_FILE) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device, cmd=None):
        self.device = device
        self.proc = None
        self.path = os.path.join("/tmp", "bench_clocks_%d_%d.csv" % (os.getpid(), device))
        self.cmd = cmd or ["nvidia-smi", "-i", str(device), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                           "-lms", "20"]

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(self.cmd, stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        atexit.register(self._end)   # a timed region that raises leaves no sampler behind
        # nvidia-smi takes a while to start: the timed region begins once it samples, so that
        # even a sub-second timed region is covered
        t0 = time.time()
        while time.time() - t0 < 10.0 and self.proc.poll() is None:
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.01)
        self.skip = sum(1 for _ in open(self.path))   # samples taken before the timed region

    def _end(self):
        if self.proc and self.proc.poll() is None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if os.path.exists(self.path):
            self.f.close()
            os.unlink(self.path)

    def mark(self):
        """Note the end of the timed region: stop() also summarises the samples taken between
        start() and this call (`timed_region`)."""
        if self.proc:
            self.f.flush()
            self.marked = sum(1 for _ in open(self.path))

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        out = self._summary(getattr(self, "skip", 0), None)
        if getattr(self, "marked", None) is not None:
            tr = self._summary(getattr(self, "skip", 0), self.marked)
            out["timed_region"] = {"sm_mhz": tr["sm_mhz"], "samples": tr["samples"], "reasons": tr["reasons"]}
        os.unlink(self.path)
        return out

    def _summary(self, lo, hi):
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for k, line in enumerate(open(self.path)):
            if k < lo or (hi is not None and k >= hi):
                continue
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def workload(n, seed=2):
    from cabanadem_b200 import scenarios as S
    return S.hcp_box(n=n, seed=seed)


def algorithmic_bytes(sc, state, off):
    """Per-particle-step bytes of the fused step: 168 (read x,u,omega + write x,u,omega +
    read r, m, I, all FP64) + 4 n_nbr + 56 n_c + 48 n_wc."""
    n = state.n
    n_nbr = float(off[-1]) / n
    n_c = float(state.tng_count.sum()) / n
    w = sc.walls
    d = (state.x[:, None, :] - w.x[None, :, :]) * w.normal[None, :, :]
    n_wc = float(((state.rad[:, None] - d.sum(axis=2)) > 0).sum()) / n
    b = 168.0 + 4.0 * n_nbr + 56.0 * n_c + 48.0 * n_wc
    return b, dict(n_nbr=round(n_nbr, 4), n_contacts=round(n_c, 6), n_wall_contacts=round(n_wc, 6))


def cpu_baseline(n, budget_s, max_steps=None):
    """The oracle (reference algorithm: rebuild every step with delta = 3 r_max) on the
    host cores; steps until the time budget is used."""
    from oracle import oracle as O
    sc = workload(n)
    delta = 3.0 * float(sc.state.rad.max())
    st = sc.state
    O.run(st, sc.walls, sc.params, sc.dt, 1, delta=delta, gravity=sc.gravity)   # warm-up step
    steps, t0 = 0, time.perf_counter()
    while True:
        O.run(st, sc.walls, sc.params, sc.dt, 1, delta=delta, gravity=sc.gravity)
        steps += 1
        el = time.perf_counter() - t0
        if el >= budget_s or (max_steps and steps >= max_steps):
            break
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return dict(value=n * steps / el, unit=METRIC, cores=cores, kind="port",
                sample="%d reference steps (rebuild every step, delta = 3 r_max) of the %d-sphere workload, %.1f s"
                % (steps, n, el))


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    n = args.n
    budget = max(5.0, min(args.cpu_seconds, 120.0))
    cb = cpu_baseline(n, budget, max_steps=max(1, args.steps))
    line = {"metric": METRIC, "value": cb["value"], "unit": METRIC, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "impl": "reference", "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "hcp_box_%d: %d polydisperse spheres r~U[0.8,1.2] mm, jittered HCP, 6 walls, "
                                   "gravity, dt 5e-8 s, skin 0.1 r_mean" % (n, n),
                       "precision": "fp64", "parallelism": "single",
                       "algorithm": "the reference's CPU path: neighbour list rebuilt every step with cutoff "
                                    "3 r_max (the skin is not used)"},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def _timed(ctx, fn):
    """Device time (ms) of fn() on the library's stream, synchronised on both sides."""
    import torch
    stream = torch.cuda.ExternalStream(ctx.stream_ptr())
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fn()
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def run_other(args):
    """The configurations other than the headline lattice (single GPU; N > 1 runs replicas)."""
    ws, rank, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    from cabanadem_b200 import api, autotune, scenarios as S, surrogate as SG
    from cabanadem_b200._lib import DEM_FP64, DEM_MIXED
    ctx = api.Context(local)
    clocks = ClockSampler(local)
    line = {"metric": METRIC, "unit": METRIC, "n_gpus": ws, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "data": "synthetic"}
    if args.workload == "dense":
        from cabanadem_b200._lib import DEM_FP64 as _F64
        prec = DEM_MIXED if args.precision == "mixed" else _F64
        sc = S.dam_break(n=200_000, aspect=2.0, seed=101)
        s = api.from_scenario(sc, ctx=ctx, precision=prec, contact_lanes=args.contact_lanes, dense_form=args.dense_form,
                              steps_per_launch=args.steps_per_launch)
        desc = "dam_break_200000 (dense flow)"
        if args.load:
            s.particles.load(args.load)
            desc += " from %s" % os.path.basename(args.load)
        elif args.dense_advance > 0:
            s.run_steps(args.dense_advance)
            desc += " at t = %.3f s" % (args.dense_advance * sc.dt)
        if args.save:
            s.particles.save(args.save)
        line.update({"steps": args.steps, "dtype": "f64" if prec == _F64 else "f64 state / f32 force",
                     "config": {"workload": desc, "contact_lanes": args.contact_lanes, "dense_form": args.dense_form,
                                "steps_per_launch": args.steps_per_launch}})
        if args.steps > 0:
            s.run_steps(min(args.steps, 64))      # graph capture, kernel-form choice, build
            clocks.start()
            ms = _timed(ctx, lambda: s.run_steps(args.steps))
            line["clocks"] = clocks.stop()
            line.update({"value": sc.state.n * args.steps / (ms / 1e3), "ms_per_step": ms / args.steps,
                         "stats": s.stats()})
        if rank == 0:
            print(json.dumps(line), flush=True)
        ctx.close()
        return 0
    if args.workload == "surrogate_stride":
        sc = S.dam_break(n=200_000, aspect=2.0, seed=101)
        weights = os.path.join(ROOT, "cabanadem_b200", "data", "dam_break_surrogate.npz")
        sg = SG.load(ctx, weights, sc)
        x = torch.as_tensor(sc.state.x).cuda()
        x2 = x.clone()
        x2[:, 1] -= 1e-6
        rad = torch.as_tensor(sc.state.rad).cuda()
        sg.predict(x, x2, rad)            # the first call sizes the buffers
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(max(args.steps, 1)):
            sg.predict(x, x2, rad)
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) / max(args.steps, 1) * 1e3
        line.update({"metric": "ms per network stride", "unit": "ms", "value": ms, "higher_is_better": False,
                     "steps": args.steps, "dtype": "bf16 network (fp32 accumulate)",
                     "config": {"workload": "dam_break_200000 network strides from the initial lattice"}})
        if rank == 0:
            print(json.dumps(line), flush=True)
        sg.close()
        ctx.close()
        return 0
    if args.workload in ("random_box", "batched", "bonded"):
        if args.workload == "random_box":
            sc = S.random_box(seed=1 + rank)
            obj = api.from_scenario(sc, ctx=ctx)
            n, steps, dtype = sc.state.n, args.steps, "f64"
            desc = ("random_box_4096: 4096 r=1 mm glass spheres, non-overlapping, 5 cm cube, 6 walls, gravity, "
                    "dt 1e-7 s, skin 0.1 r")
            extra = {}
        elif args.workload == "batched":
            sc = S.batched_scenes(seed=3 + rank)
            obj = api.BatchRunner(sc, precision=DEM_MIXED, tune=True, device=local)
            n, steps, dtype = sc.state.n, args.steps, "f64 state / f32 force"
            desc = ("batched_1024_scenes: %d spheres in 1024 independent scenes (log-uniform [2,8192] per scene), "
                    "one plane per scene, e~U[0.3,0.95], mu~U[0.1,0.5], dt 1e-7 s, measured window %d steps; "
                    "scenes grouped by size bucket, each bucket a graph-looped solver with its own tuned "
                    "settings on its own stream, the buckets concurrent; wall-clock timing" % (n, steps))
            extra = {"autotuned": {str(p["bucket"]): dict(p["config"], particles=p["scenario"].state.n,
                                                          scenes=len(p["scenes"])) for p in obj.parts}}
        else:
            case = S.bonded_bar()
            obj = api.bonded_from_case(case, ctx=ctx)
            n, steps, dtype = case["state"].n, args.steps, "f64"
            desc = ("bonded_bar_256x64x8: %d spheres r=0.5 mm, 6-neighbour bonds within 1.05 d, kn 1e7, kt 4e6, "
                    "ends pulled at 0.05 m/s, break at 1 %% strain, dt 2e-8 s, measured window %d steps"
                    % (n, steps))
            extra = {}
        obj.run_steps(max(3, args.warmup))
        clocks.start()
        if args.workload == "batched":
            # several contexts: the run returns once every bucket's device work is done
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            obj.run_steps(steps)
            torch.cuda.synchronize()
            ms = (time.perf_counter() - t0) * 1e3
        else:
            ms = _timed(ctx, lambda: obj.run_steps(steps))
        ck = clocks.stop()
        if args.workload == "bonded":
            extra["broken_bonds"] = obj.broken()
        if args.workload == "batched":
            obj.close()
        line.update({"value": ws * n * steps / (ms / 1e3), "steps": steps, "ms_per_step": ms / steps,
                     "dtype": dtype, "config": {"workload": desc, "parallelism": "replicas" if ws > 1 else "single",
                                                "l2": "state %s L2" % ("larger than" if n * 330 > 126e6 else
                                                                       "smaller than (latency-bound size)"), **extra},
                     "clocks": ck})
    else:
        n = 200_000
        mk = lambda: S.dam_break(n=n, aspect=2.0, seed=101 + rank)
        weights = os.path.join(ROOT, "cabanadem_b200", "data", "dam_break_surrogate.npz")
        sg = SG.load(ctx, weights, mk())
        clocks.start()
        res = SG.evaluate(sg, mk, args.seconds, ctx)
        ck = clocks.stop()
        line.update({"value": ws * res["surrogate_particle_steps_per_s"], "steps": res["strides"] * SG.STRIDE,
                     "ms_per_step": res["surrogate_wall_s"] * 1e3 / (res["strides"] * SG.STRIDE),
                     "dtype": "bf16 network (fp32 accumulate) + f64 DEM fallback",
                     "config": {"workload": "dam_break_200000: quasi-2D disks r~U[0.9,1.1] mm, column aspect 2, "
                                            "mu 0.4, e 0.5, E 1 GPa, dt 1e-6 s, %.2f s simulated; learned surrogate "
                                            "(200-step strides) vs plain FP64 DEM" % args.seconds},
                     "dem_reference": {"value": res["dem_particle_steps_per_s"], "unit": METRIC,
                                       "wall_s": res["dem_wall_s"]},
                     "surrogate": {k: res[k] for k in ("speedup", "surrogate_wall_s", "front_error", "runout_error",
                                                       "profile_error", "depth_error", "strides_network", "strides_dem",
                                                       "fallback_overlap", "fallback_energy", "max_overlap_seen",
                                                       "front_dem", "front_surrogate")},
                     "clocks": ck})
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def _device_ms(stream, fn):
    """Device time (ms) of the work fn() queues on `stream`, synchronised on both sides."""
    import torch
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fn()
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def _step_roofline(solver, sc, stats0, stats1, peak):
    """Algorithmic bytes per particle-step of the state now (168 + 4 n_nbr + 56 n_c + 48 n_wc)
    over the fused step's device time per step between two stats() snapshots."""
    n = sc.state.n
    g_steps = stats1["graph_steps"] - stats0["graph_steps"]
    kernel_ms = (stats1["graph_ms"] - stats0["graph_ms"]) / max(g_steps, 1)
    state = solver.particles.download()
    off, _ = solver.neighbors()
    b_step, occ = algorithmic_bytes(sc, state, off)
    achieved = n * b_step / (kernel_ms / 1e3) / 1e9
    return {"achieved": round(achieved, 1), "frac": round(achieved / peak, 4), "kernel_ms": round(kernel_ms, 5),
            "bytes_per_particle_step": round(b_step, 2), "graph_steps": g_steps, **occ}, state, off


def measure_mixed(ctx, args, stream, peak, n_steps, fp64_ms):
    """The headline lattice with FP32 contact forces (DEM_MIXED), same warm-up and step count."""
    from cabanadem_b200 import api
    from cabanadem_b200._lib import DEM_MIXED
    sc = workload(args.n, seed=2)
    s = api.from_scenario(sc, ctx=ctx, precision=DEM_MIXED, stream_split=args.stream_split)
    s.run_steps(max(3, args.warmup))
    st0 = s.stats()
    ms = _device_ms(stream, lambda: s.run_steps(n_steps))
    st1 = s.stats()
    roof, _, _ = _step_roofline(s, sc, st0, st1, peak)
    s.close()
    s.particles.close()
    return {"value": sc.state.n * n_steps / (ms / 1e3), "unit": METRIC, "ms_per_step": ms / n_steps,
            "steps": n_steps, "speedup_vs_fp64": round((fp64_ms / n_steps) / (ms / n_steps), 4) if fp64_ms else None,
            "dtype": "f64 state / f32 force", "roofline": roof}


def measure_dense(ctx, args, stream, peak, n_steps):
    """The 200,000-disk dam break advanced to t = dense_advance * 1 us (0.3 s: the column is
    collapsing, about 3 contacts per disk), then n_steps timed in FP64 and, from the same
    saved state, in mixed precision."""
    import tempfile
    from cabanadem_b200 import api, scenarios as S
    from cabanadem_b200._lib import DEM_FP64, DEM_MIXED
    mk = lambda: S.dam_break(n=200_000, aspect=2.0, seed=101)
    sc = mk()
    out = {"workload": "dam_break_200000 at t = %.3f s: quasi-2D disks r~U[0.9,1.1] mm, column aspect 2, mu 0.4, "
                       "e 0.5, E 1 GPa, dt 1e-6 s" % (args.dense_advance * sc.dt),
           "steps": n_steps, "unit": METRIC}
    s = api.from_scenario(sc, ctx=ctx, precision=DEM_FP64)
    t0 = time.perf_counter()
    s.run_steps(args.dense_advance)
    ctx.sync()
    out["advance_s"] = round(time.perf_counter() - t0, 2)
    with tempfile.TemporaryDirectory() as d:
        ck = os.path.join(d, "dense.ckpt")
        s.particles.save(ck)
        for name, prec, solver in (("fp64", DEM_FP64, s), ("mixed", DEM_MIXED, None)):
            if solver is None:
                solver = api.from_scenario(mk(), ctx=ctx, precision=prec)
                solver.particles.load(ck)
            solver.run_steps(64)            # graph capture, kernel-form choice and any rebuild
            st0 = solver.stats()
            ms = _device_ms(stream, lambda: solver.run_steps(n_steps))
            st1 = solver.stats()
            roof, state, _ = _step_roofline(solver, sc, st0, st1, peak)
            out[name] = {"value": sc.state.n * n_steps / (ms / 1e3), "us_per_step": round(ms / n_steps * 1e3, 2),
                         "rebuilds": st1["rebuilds"] - st0["rebuilds"],
                         "in_contact": round(float((state.tng_count > 0).mean()), 4), "roofline": roof}
            solver.close()
            solver.particles.close()
    out["mixed_speedup"] = round(out["fp64"]["us_per_step"] / out["mixed"]["us_per_step"], 4)
    return out


def measure_configs(local, ctx, stream, args):
    """The other configurations of the suite, each device-timed on this GPU after the headline
    (so that the driver's line records them): C1 (4,096 spheres in a walled box), C3 (the
    1,024-scene batch, mixed, size buckets with the packaged B200 settings, wall-clock over the
    concurrent buckets), C4 (the bonded bar, FP64) and C5 (learned surrogate against plain DEM on
    the 200k-disk dam break, --seconds simulated)."""
    import torch
    from cabanadem_b200 import api, scenarios as S, surrogate as SG
    from cabanadem_b200._lib import DEM_MIXED
    steps = max(args.steps, args.sub_steps)
    out = {}
    sc = S.random_box(seed=1)
    s = api.from_scenario(sc, ctx=ctx)
    s.run_steps(max(3, args.warmup))
    ms = _device_ms(stream, lambda: s.run_steps(steps))
    out["c1"] = {"workload": "random_box_4096: 4096 r=1 mm spheres, 5 cm cube, 6 walls, gravity, dt 1e-7 s, FP64",
                 "value": sc.state.n * steps / (ms / 1e3), "ms_per_step": round(ms / steps, 5), "steps": steps}
    s.close()
    s.particles.close()
    sc = S.batched_scenes(seed=3)
    runner = api.BatchRunner(sc, precision=DEM_MIXED, device=local)
    runner.run_steps(max(3, args.warmup))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    runner.run_steps(steps)
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) * 1e3
    out["c3"] = {"workload": "batched_1024_scenes: %d spheres in 1024 scenes (log-uniform [2,8192]), mixed; size "
                             "buckets with the packaged B200 settings, concurrent; wall-clock" % sc.state.n,
                 "value": sc.state.n * steps / (ms / 1e3), "ms_per_step": round(ms / steps, 5), "steps": steps}
    runner.close()
    case = S.bonded_bar()
    b = api.bonded_from_case(case, ctx=ctx)
    b.run_steps(max(3, args.warmup))
    ms = _device_ms(stream, lambda: b.run_steps(steps))
    out["c4"] = {"workload": "bonded_bar_256x64x8: %d spheres, 6-neighbour bonds, ends pulled, FP64" % case["state"].n,
                 "value": case["state"].n * steps / (ms / 1e3), "ms_per_step": round(ms / steps, 5), "steps": steps}
    b.close()
    if args.seconds > 0:
        mk = lambda: S.dam_break(n=200_000, aspect=2.0, seed=101)
        sg = SG.load(ctx, os.path.join(ROOT, "cabanadem_b200", "data", "dam_break_surrogate.npz"), mk())
        res = SG.evaluate(sg, mk, args.seconds, ctx)
        out["c5"] = {"workload": "dam_break_200000, %.2f s simulated: learned surrogate (200-step strides) against "
                                 "plain FP64 DEM" % args.seconds,
                     "value": res["surrogate_particle_steps_per_s"], "dem_value": res["dem_particle_steps_per_s"],
                     "speedup": round(res["speedup"], 3), "front_error": round(res["front_error"], 4),
                     "surrogate_wall_s": round(res["surrogate_wall_s"], 3), "dem_wall_s": round(res["dem_wall_s"], 3)}
        sg.close()
    return out


def measure_rebuild(solver, stream, state, off, peak, n):
    """One full rebuild of the solver's state (Morton re-sort with history remap, new list),
    device-timed; algorithmic bytes per particle 24 + 2*168 + 4 n_nbr + 56 n_c."""
    ms = _device_ms(stream, solver.rebuild)
    n_nbr = float(off[-1]) / n
    n_c = float(state.tng_count.sum()) / n
    b = 24.0 + 2.0 * 168.0 + 4.0 * n_nbr + 56.0 * n_c
    gbs = n * b / (ms / 1e3) / 1e9
    return {"ms": round(ms, 4), "bytes_per_particle": round(b, 2), "achieved_gbs": round(gbs, 1),
            "frac": round(gbs / peak, 4)}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload != "hcp":
        return run_other(args)
    ws, rank, local = dist_env()
    import torch
    if ws > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    from cabanadem_b200 import api
    from cabanadem_b200._lib import DEM_FP64, DEM_MIXED

    prec = DEM_FP64 if args.precision == "fp64" else DEM_MIXED
    sc = workload(args.n, seed=2 + rank)
    ctx = api.Context(local)
    solver = api.from_scenario(sc, ctx=ctx, precision=prec, steps_per_launch=args.steps_per_launch,
                               stream_split=args.stream_split)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=torch.device("cuda", local))

    def barrier():
        if ws > 1:
            torch.distributed.barrier()

    clocks = ClockSampler(local)
    solver.run_steps(max(3, args.warmup))
    clocks.start()
    stats0 = solver.stats()
    barrier()
    torch.cuda.synchronize(local)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    solver.run_steps(args.steps)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize(local)
    barrier()
    clocks.mark()
    ms = e0.elapsed_time(e1)
    stats1 = solver.stats()
    ms = max_over_ranks(ms)
    n = args.n
    value = ws * n * args.steps / (ms / 1e3)
    peak, peak_kind = hbm_peak()
    # roofline of the fused step: algorithmic bytes over the device time of the step-graph
    # replays of the timed region (CUDA events around each replay; host gaps excluded)
    sr, state, off = _step_roofline(solver, sc, stats0, stats1, peak)
    occ = {k: sr[k] for k in ("n_nbr", "n_contacts", "n_wall_contacts")}
    roof = {"bound": "hbm", "achieved": sr["achieved"], "peak": peak, "unit": "GB/s", "frac": sr["frac"],
            "traffic": None,
            "traffic_note": "not measured in this run (ncu is not run inside the bench); DRAM bytes of the same "
                            "kernels from a separate ncu capture are in the profile summaries",
            "peak_kind": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
            "kernel": "fused step: k_stream + k_contact + k_apply (FP64 force + integration)",
            "kernel_ms": sr["kernel_ms"],
            "kernel_ms_source": "CUDA events around each step-graph replay of the timed region (%d steps)"
                                % sr["graph_steps"],
            "bytes_per_particle_step": sr["bytes_per_particle_step"], **occ}

    # device-timed sub-measurements on this GPU, after the timed region
    sub = {}
    if not args.no_sub and ws == 1:
        sub_steps = max(args.steps, args.sub_steps)
        sub["rebuild"] = measure_rebuild(solver, stream, state, off, peak, n)
        fp64_ms = _device_ms(stream, lambda: solver.run_steps(sub_steps)) if prec == DEM_FP64 else None
        if prec == DEM_FP64:
            sub["fp64_sub_ms_per_step"] = round(fp64_ms / sub_steps, 5)
            sub["mixed"] = measure_mixed(ctx, args, stream, peak, sub_steps, fp64_ms)
        if args.dense_advance > 0:
            sub["dense"] = measure_dense(ctx, args, stream, peak, sub_steps)
        if not args.no_configs:
            sub.update(measure_configs(local, ctx, stream, args))

    # end to end through the C ABI with host buffers (pinned): a new run sets positions,
    # velocities, spins, radii, masses, inertias and material constants, clears the contact
    # state and the stored force and torque on the device (a fresh start, as new particles
    # have them), steps, and reads the state back
    barrier()
    host = sc.state.copy()
    pinned = []
    up_fields = ("rad", "x", "u", "omega", "m", "I", "rho", "E", "nu", "G")
    for f in up_fields:
        t = torch.from_numpy(np.ascontiguousarray(getattr(host, f))).pin_memory()
        pinned.append(t)
        setattr(host, f, t.numpy())
    h2d = sum(getattr(host, f).nbytes for f in up_fields)
    outbuf = {}
    for f in ("x", "u", "omega"):
        t = torch.empty((n, 3), dtype=torch.float64).pin_memory()
        pinned.append(t)
        outbuf[f] = t.numpy()
    def e2e_call():
        for f in up_fields:
            solver.particles.set(f, getattr(host, f))
        solver.particles.clear_contacts()
        solver.particles.clear_forces()
        solver.run_steps(args.steps)
        return {f: solver.particles.get(f, out=outbuf[f]) for f in outbuf}

    e2e_call()   # untimed warm-up call (first use of the pinned buffers and of the upload path)
    barrier()
    torch.cuda.synchronize(local)
    t0 = time.perf_counter()
    a0 = torch.cuda.Event(enable_timing=True)
    a1 = torch.cuda.Event(enable_timing=True)
    a0.record(stream)
    out = e2e_call()
    a1.record(stream)
    a1.synchronize()
    e2e_ms = a0.elapsed_time(a1)
    wall_ms = (time.perf_counter() - t0) * 1e3
    d2h = sum(v.nbytes for v in out.values())
    e2e_ms = max_over_ranks(e2e_ms)
    e2e = {"value": ws * n * args.steps / (e2e_ms / 1e3), "unit": METRIC,
           "h2d_bytes_per_step": int(h2d / args.steps), "d2h_bytes_per_step": int(d2h / args.steps),
           "wall_ms": round(wall_ms, 2),
           "uploaded": list(up_fields) + ["(contact state, force and torque cleared on the device)"], "downloaded": list(outbuf)}
    ck = clocks.stop()
    ck["window"] = "timed region, the sub-measurements and the end-to-end run (the timed region alone: timed_region)"

    rebuilds = stats1["rebuilds"] - stats0["rebuilds"]
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if prec == DEM_FP64 else "f64 state / f32 force",
            "data": "synthetic",
            "config": {"workload": "hcp_box_%d: %d polydisperse spheres r~U[0.8,1.2] mm, jittered HCP, 6 walls, "
                                   "gravity, dt 5e-8 s, skin 0.1 r_mean" % (n, n),
                       "precision": args.precision, "parallelism": "replicas" if ws > 1 else "single",
                       "l2": "inputs larger than L2 (device state ~%.2f GB)" % (n * 330 / 1e9),
                       "rebuilds_in_timed_region": rebuilds, "neighbors_per_particle": occ["n_nbr"]},
            "roofline": roof, "e2e": e2e, "clocks": ck,
            "gpu_launches": int(stats1["launches"] - stats0["launches"])}
    line.update(sub)
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(n, args.cpu_seconds)
    if rank == 0:
        print(json.dumps(line), flush=True)
    solver.close()
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
