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
              walls, one launch per step for all scenes, FP32 forces / FP64 state, launch
              settings from the autotuner
  bonded      256 x 64 x 8 bonded bar pulled at both ends, FP64
  dam_break   200,000 quasi-2D disks: full DEM rollout vs the learned surrogate with DEM
              fallback over the same simulated time (wall-clock of each, runout front and
              deposit profile errors against DEM)

Prints one JSON line (rank 0).  `value` is device-timed (CUDA events on the library's
stream, inputs resident in HBM); `e2e` is the same metric through the C ABI with host
buffers (state upload + steps + state download inside the timed region);
`roofline` is the fused step kernel's algorithmic bytes per launch over its
CUDA-event-timed mean launch duration; `cpu_baseline` is the CPU oracle (a C++
restatement of the reference's step, run in the reference's rebuild-every-step mode) on
a bounded sample of the same workload.
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
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "fused_step_fp64_hcp.md")


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
    ap.add_argument("--profile-steps", type=int, default=50)
    ap.add_argument("--workload", default="hcp", choices=["hcp", "random_box", "batched", "bonded", "dam_break"])
    ap.add_argument("--seconds", type=float, default=0.25, help="dam_break: simulated time of both rollouts")
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


def traffic_per_particle_step():
    """DRAM bytes per particle-step of the fused kernel from the committed ncu summary."""
    try:
        for line in open(TRAFFIC_FILE):
            if line.strip().startswith("dram_bytes_per_particle_step:"):
                return float(line.split(":", 1)[1].split()[0])
    except Exception:
        pass
    return None


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

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for k, line in enumerate(open(self.path)):
            if k < getattr(self, "skip", 0):
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
        os.unlink(self.path)
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
            cfg = autotune.tune(sc, precision=DEM_MIXED, warmup=5, steps=40)
            sc2 = S.batched_scenes(seed=3 + rank)
            kw = autotune.apply(sc2, cfg)
            obj = api.from_scenario(sc2, ctx=ctx, precision=DEM_MIXED, **kw)
            n, steps, dtype = sc.state.n, args.steps, "f64 state / f32 force"
            desc = ("batched_1024_scenes: %d spheres in 1024 independent scenes (log-uniform [2,8192] per scene), "
                    "one plane per scene, e~U[0.3,0.95], mu~U[0.1,0.5], dt 1e-7 s, measured window %d steps"
                    % (n, steps))
            extra = {"autotuned": cfg}
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
        ms = _timed(ctx, lambda: obj.run_steps(steps))
        ck = clocks.stop()
        if args.workload == "bonded":
            extra["broken_bonds"] = obj.broken()
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
    solver = api.from_scenario(sc, ctx=ctx, precision=prec)
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
    ck = clocks.stop()
    ms = e0.elapsed_time(e1)
    stats1 = solver.stats()
    ms = max_over_ranks(ms)
    n = args.n
    value = ws * n * args.steps / (ms / 1e3)
    # fused-step device time inside the timed region: CUDA events around every step-graph
    # replay (host gaps between replays excluded), per step
    g_steps = stats1["graph_steps"] - stats0["graph_steps"]
    kernel_ms = (stats1["graph_ms"] - stats0["graph_ms"]) / max(g_steps, 1)
    profile_ms = solver.profile_steps(args.profile_steps) if args.profile_steps > 0 else None

    # roofline of the fused step kernel
    state = solver.particles.download()
    off, _ = solver.neighbors()
    b_step, occ = algorithmic_bytes(sc, state, off)
    peak, peak_kind = hbm_peak()
    achieved = n * b_step / (kernel_ms / 1e3) / 1e9
    tpps = traffic_per_particle_step()
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": (round(tpps * n) if tpps else None),
            "peak_kind": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
            "kernel": "fused step: k_stream + k_contact + k_apply (FP64 force + integration)", "kernel_ms": round(kernel_ms, 5),
            "kernel_ms_source": "CUDA events around each step-graph replay of the timed region (%d steps)" % g_steps,
            "profile_ms_after": round(profile_ms, 5) if profile_ms else None,
            "bytes_per_particle_step": round(b_step, 2), **occ}

    # end to end through the C ABI with host buffers: the caller's state lives in pinned
    # (page-locked) host memory, so the uploads are DMA copies
    barrier()
    host = sc.state.copy()
    pinned = []
    for f, a in list(host.arrays().items()):
        t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        pinned.append(t)
        setattr(host, f, t.numpy())
    h2d = sum(getattr(host, f).nbytes for f in ("rad", "x", "u", "omega", "force", "torque", "m", "I", "rho", "E",
                                                 "nu", "G", "tng_idx", "tng_ss_x", "tng_ss_y", "tng_ss_z",
                                                 "tng_count", "tng_sw_x", "tng_sw_y", "tng_sw_z"))
    outbuf = {}
    for f in ("x", "u", "omega", "force", "torque"):
        t = torch.empty((n, 3), dtype=torch.float64).pin_memory()
        pinned.append(t)
        outbuf[f] = t.numpy()
    torch.cuda.synchronize(local)
    t0 = time.perf_counter()
    a0 = torch.cuda.Event(enable_timing=True)
    a1 = torch.cuda.Event(enable_timing=True)
    a0.record(stream)
    solver.particles.upload(host)
    solver.run_steps(args.steps)
    out = {f: solver.particles.get(f, out=outbuf[f]) for f in outbuf}
    a1.record(stream)
    a1.synchronize()
    e2e_ms = a0.elapsed_time(a1)
    wall_ms = (time.perf_counter() - t0) * 1e3
    d2h = sum(v.nbytes for v in out.values())
    e2e_ms = max_over_ranks(e2e_ms)
    e2e = {"value": ws * n * args.steps / (e2e_ms / 1e3), "unit": METRIC,
           "h2d_bytes_per_step": int(h2d / args.steps), "d2h_bytes_per_step": int(d2h / args.steps),
           "wall_ms": round(wall_ms, 2)}

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
