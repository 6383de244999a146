"""Learned surrogate of the quasi-2D granular dam break (C ABI dem_surrogate_*).

A message-passing network over the contact graph predicts, from the positions at the last
two strides, the change of the per-stride displacement; one stride replaces 200 DEM steps.
It is trained on rollouts that the DEM kernels generate (recorded into device memory), by
the library's own forward/backward kernels (tensor-core dense layers, fixed-order
reductions) and Adam; plain DEM takes over any stride whose overlap or energy residual
exceeds the thresholds, and a full DEM rollout is the judge of the surrogate's rollout.

torch is only the allocator and the batch assembler (tensor slicing) here."""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np
import torch

from . import api
from . import scenarios as S
from ._lib import DEM_FP64, RolloutStats, SurrogateParams, check, lib

STRIDE = 200   # DEM steps per network stride


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def params_for(sc, sigma_a, max_nodes, max_frames=8, radius_graph=3.0e-3, sigma_d=1.0e-3, wall_clip=5.0e-3,
               max_overlap=0.05, energy_tol=0.05, steps_per_stride=STRIDE, nwalls=2, project_iters=6,
               project_allow=0.01):
    """Surrogate parameters for a dam_break scenario (radii, gravity, dt from it).  The network
    sees the first `nwalls` walls (floor and back wall); the far wall of a dam break is placed
    beyond the runout and left out, so one network serves columns of any length."""
    p = SurrogateParams()
    p.radius_graph = radius_graph
    p.steps_per_stride = steps_per_stride
    p.dt = sc.dt
    p.sigma_d = sigma_d
    p.sigma_a = sigma_a
    p.r_mean = sc.extra["r_mean"]
    p.r_std = sc.extra["r_std"]
    nw = min(sc.walls.n, nwalls)
    if nw > 4:
        raise ValueError("at most 4 walls")
    p.nwalls = nw
    for w in range(nw):
        for d in range(3):
            p.wall_x[w][d] = float(sc.walls.x[w, d])
            p.wall_n[w][d] = float(sc.walls.normal[w, d])
    p.wall_clip = wall_clip
    for d in range(3):
        p.gravity[d] = float(sc.gravity[d])
    p.max_overlap = max_overlap
    p.energy_tol = energy_tol
    p.max_nodes = int(max_nodes)
    p.max_frames = int(max_frames)
    p.project_iters = int(project_iters)
    p.project_allow = float(project_allow)
    return p


class Surrogate:
    def __init__(self, ctx: api.Context, prm: SurrogateParams):
        self.ctx, self.prm = ctx, prm
        h = C.c_void_p()
        check(lib().dem_surrogate_create(ctx.h, C.byref(prm), C.byref(h)), ctx.h, "dem_surrogate_create")
        self.h = h
        ctx.adopt(self)
        self.stream = torch.cuda.ExternalStream(ctx.stream_ptr())

    @property
    def num_params(self) -> int:
        return int(lib().dem_surrogate_num_params(self.h))

    def get_params(self) -> np.ndarray:
        a = np.empty(self.num_params, dtype=np.float32)
        check(lib().dem_surrogate_get_params(self.h, a.ctypes.data, a.size), self.ctx.h, "get_params")
        return a

    def set_params(self, a):
        a = np.ascontiguousarray(a, dtype=np.float32)
        check(lib().dem_surrogate_set_params(self.h, a.ctypes.data, a.size), self.ctx.h, "set_params")

    def init_params(self, seed: int):
        check(lib().dem_surrogate_init_params(self.h, int(seed)), self.ctx.h, "init_params")

    def loss_grad(self, prev, cur, nxt, rad, frame=None, nframes=1, noise=0.0, seed=0, want_grads=True):
        loss = C.c_double(0.0)
        g = np.empty(self.num_params, dtype=np.float32) if want_grads else None
        st = lib().dem_surrogate_loss_grad(self.h, int(cur.shape[0]), _p(prev), _p(cur), _p(nxt), _p(rad), _p(frame),
                                           int(nframes), float(noise), int(seed), C.byref(loss),
                                           g.ctypes.data if g is not None else None)
        check(st, self.ctx.h, "dem_surrogate_loss_grad")
        return loss.value, g

    def train_step(self, prev, cur, nxt, rad, frame=None, nframes=1, noise=0.0, seed=0, lr=1e-3) -> float:
        loss = C.c_double(0.0)
        st = lib().dem_surrogate_train_step(self.h, int(cur.shape[0]), _p(prev), _p(cur), _p(nxt), _p(rad), _p(frame),
                                            int(nframes), float(noise), int(seed), float(lr), C.byref(loss))
        check(st, self.ctx.h, "dem_surrogate_train_step")
        return loss.value

    def predict(self, prev, cur, rad, frame=None, nframes=1):
        with torch.cuda.stream(self.stream):
            out = torch.empty_like(cur)
        st = lib().dem_surrogate_predict(self.h, int(cur.shape[0]), _p(prev), _p(cur), _p(rad), _p(frame), int(nframes),
                                         _p(out))
        check(st, self.ctx.h, "dem_surrogate_predict")
        return out

    def rollout(self, solver: api.SolverDEM, nstrides: int, use_network: bool = True) -> dict:
        s = RolloutStats()
        st = lib().dem_surrogate_rollout(self.h, solver.h, int(nstrides), 1 if use_network else 0, C.byref(s))
        check(st, self.ctx.h, "dem_surrogate_rollout")
        return {k: getattr(s, k) for k, _ in s._fields_}

    def close(self):
        if self.h and self.ctx.alive:
            lib().dem_surrogate_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------------------
# data: DEM rollouts recorded every stride into device memory
# ---------------------------------------------------------------------------------------
def record_rollout(sc, ctx: api.Context, strides: int, precision=DEM_FP64, stride=STRIDE):
    """Run the DEM solver on `sc` for `strides` strides; returns (positions float64
    [strides + 1, n, 3] on the device, radii float64 [n] on the device, DEM seconds)."""
    s = api.from_scenario(sc, ctx=ctx, precision=precision)
    n = sc.state.n
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.ExternalStream(ctx.stream_ptr())
    with torch.cuda.stream(stream):
        traj = torch.empty(strides + 1, n, 3, dtype=torch.float64, device=dev)
        rad = torch.as_tensor(sc.state.rad, dtype=torch.float64).to(dev)
    s.particles.get_device("x", traj[0])
    t0 = time.perf_counter()
    for f in range(1, strides + 1):
        s.run_steps(stride)
        s.particles.get_device("x", traj[f])
    ctx.sync()
    secs = time.perf_counter() - t0
    s.close()
    s.particles.close()
    return traj, rad, secs


def sigma_a_of(trajs) -> float:
    """RMS (over particles, components and frames) of the change of per-stride displacement."""
    acc, cnt = 0.0, 0
    for traj, _ in trajs:
        a = traj[2:, :, :2] - 2.0 * traj[1:-1, :, :2] + traj[:-2, :, :2]
        acc += float((a * a).sum())
        cnt += a.numel()
    return math.sqrt(acc / max(cnt, 1))


def batch(trajs, picks, dev):
    """Frames (rollout r, stride k) concatenated as one disjoint graph: prev, cur, next, rad,
    frame id."""
    prev = torch.cat([trajs[r][0][k - 1] for r, k in picks])
    cur = torch.cat([trajs[r][0][k] for r, k in picks])
    nxt = torch.cat([trajs[r][0][k + 1] for r, k in picks])
    rad = torch.cat([trajs[r][1] for r, k in picks])
    frame = torch.cat([torch.full((trajs[r][0].shape[1],), b, dtype=torch.int32, device=dev)
                       for b, (r, k) in enumerate(picks)])
    return prev.contiguous(), cur.contiguous(), nxt.contiguous(), rad.contiguous(), frame


def train(sg: Surrogate, trajs, steps: int, batch_frames=4, lr0=1e-3, lr1=1e-5, noise=0.0, seed=0, log_every=0):
    """Adam on randomly drawn frames; learning rate decays exponentially lr0 -> lr1."""
    rng = np.random.default_rng(seed)
    dev = trajs[0][0].device
    losses = []
    with torch.cuda.stream(sg.stream):
        for it in range(steps):
            picks = []
            for _ in range(batch_frames):
                r = int(rng.integers(len(trajs)))
                k = int(rng.integers(1, trajs[r][0].shape[0] - 1))
                picks.append((r, k))
            prev, cur, nxt, rad, frame = batch(trajs, picks, dev)
            lr = lr0 * (lr1 / lr0) ** (it / max(steps - 1, 1))
            loss = sg.train_step(prev, cur, nxt, rad, frame, batch_frames, noise=noise, seed=seed * 1000003 + it, lr=lr)
            losses.append(loss)
            if log_every and it % log_every == 0:
                print("step %d loss %.4g lr %.3g" % (it, loss, lr), flush=True)
    return losses


# ---------------------------------------------------------------------------------------
# observables judged against DEM
# ---------------------------------------------------------------------------------------
def runout_front(x, q=0.999):
    """Runout front: the q-quantile of the particles' x (robust to a few outliers)."""
    return float(np.quantile(np.asarray(x)[:, 0], q))


def depth_profile(x, rad, length, bins=400, packing=0.85):
    """Deposit depth from mass: disk area in each of `bins` columns over [0, length] divided by
    the column width and a packing fraction (insensitive to a few isolated particles)."""
    x = np.asarray(x)
    r = np.asarray(rad)
    w = length / bins
    idx = np.clip((x[:, 0] / length * bins).astype(int), 0, bins - 1)
    a = np.zeros(bins)
    np.add.at(a, idx, np.pi * r * r)
    return a / (w * packing)


def pile_profile(x, rad, length, bins=400):
    """Height of the deposit (max y + r) in `bins` columns over [0, length]."""
    x = np.asarray(x)
    idx = np.clip((x[:, 0] / length * bins).astype(int), 0, bins - 1)
    h = np.zeros(bins)
    np.maximum.at(h, idx, x[:, 1] + np.asarray(rad))
    return h


def prm_dict(p: SurrogateParams) -> dict:
    """The feature parameters as a plain dict (for the CPU restatement of the network)."""
    return dict(radius_graph=p.radius_graph, sigma_d=p.sigma_d, sigma_a=p.sigma_a, r_mean=p.r_mean, r_std=p.r_std,
                wall_clip=p.wall_clip,
                walls=[(tuple(p.wall_x[w]), tuple(p.wall_n[w])) for w in range(p.nwalls)])


def load(ctx: api.Context, path: str, sc, max_nodes=None, **kw) -> Surrogate:
    """A surrogate for scenario `sc` with the weights and feature scales saved by
    train_surrogate."""
    import json
    z = np.load(path)
    meta = json.loads(str(z["meta"]))
    prm = params_for(sc, sigma_a=meta["sigma_a"], max_nodes=max_nodes or sc.state.n, max_frames=1,
                     radius_graph=meta["radius_graph"], sigma_d=meta["sigma_d"], wall_clip=meta["wall_clip"], **kw)
    sg = Surrogate(ctx, prm)
    sg.set_params(z["params"])
    return sg


def evaluate(sg: Surrogate, make_scenario, seconds: float, ctx: api.Context) -> dict:
    """Full DEM rollout vs surrogate rollout (DEM fallback on) from the same initial state:
    wall-clock of each, fallback statistics, runout front and deposit profile errors."""
    sc = make_scenario()
    strides = int(round(seconds / (STRIDE * sc.dt)))
    a = api.from_scenario(sc, ctx=ctx)
    ctx.sync()
    t0 = time.perf_counter()
    a.run_steps(strides * STRIDE)
    ctx.sync()
    t_dem = time.perf_counter() - t0
    xa = a.particles.get("x")
    a.close()
    a.particles.close()
    b = api.from_scenario(make_scenario(), ctx=ctx)
    ctx.sync()
    t0 = time.perf_counter()
    st = sg.rollout(b, strides, use_network=True)
    ctx.sync()
    t_sur = time.perf_counter() - t0
    xb = b.particles.get("x")
    b.close()
    b.particles.close()
    x0 = sc.state.x
    fa, fb, f0 = runout_front(xa), runout_front(xb), runout_front(x0)
    length = sc.extra.get("length", float(max(xa[:, 0].max(), xb[:, 0].max())))
    ha, hb = pile_profile(xa, sc.state.rad, length), pile_profile(xb, sc.state.rad, length)
    da, db = depth_profile(xa, sc.state.rad, length), depth_profile(xb, sc.state.rad, length)
    n = sc.state.n
    return dict(n=n, seconds=seconds, strides=strides, dem_wall_s=t_dem, surrogate_wall_s=t_sur,
                speedup=t_dem / t_sur, dem_particle_steps_per_s=n * strides * STRIDE / t_dem,
                surrogate_particle_steps_per_s=n * strides * STRIDE / t_sur,
                front_dem=fa, front_surrogate=fb, front_initial=f0,
                front_error=abs(fb - fa) / fa, runout_error=abs(fb - fa) / max(fa - f0, 1e-30),
                profile_error=float(np.abs(ha - hb).mean() / max(ha.max(), 1e-30)),
                depth_error=float(np.abs(da - db).mean() / max(da.max(), 1e-30)),
                max_height_dem=float(ha.max()), max_height_surrogate=float(hb.max()), **st)
