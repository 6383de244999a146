"""Slab decomposition of one scene over the ranks of a torch.distributed group.

The reference computes full-list per-particle forces (src/CabanaDEM_Force.hpp:334-339, the
neighbour loop over i's own list): every particle sums its own pair terms and writes only its
own tangential history.  So a rank that owns a slab of the domain, and holds copies ("ghosts")
of every particle within contact reach of its slab, computes its particles' forces exactly.
No force is sent back, and history stays with the particle's owner.  One step on every rank:

1. migration: owned particles whose position left the slab go to the neighbouring slab's rank;
2. ghost exchange: owned particles within `halo` of a slab face are copied to the rank beyond;
3. the local set (owned and ghosts, ascending global id) takes one step, through `step_fn`;
4. the owned rows are kept, with their contact partners stored as global ids.  The ghosts'
   own results are dropped: their neighbourhood is incomplete.

Each owned particle then sums the same partners in the same order as the undecomposed run.
The local set is in global-id order, and it holds every particle that can touch an owned one.
So the decomposed run is bit-identical to the single-domain run; the CPU tests check this.
`halo` must cover the contact range after the step's drift: halo >= 2 r_max + 2 x (largest
displacement in one step).  The check after every step raises DemError when a particle moved
further than that margin allows.  Slabs are at least `halo` wide, so ghosts come from the two
neighbouring slabs only.

Exchanges are point-to-point (`batch_isend_irecv`: counts, then rows) between neighbouring
ranks only.  They are float64 tensors on `device`: the CPU for gloo, the rank's GPU for NCCL
(set it with torch.cuda.set_device first).  Every step starts with an all-reduce on all
ranks, so the group's first collective involves every rank, as NCCL requires before
point-to-point batches.
A particle's row carries its global id, every per-particle field of the reference's Particles
(src/CabanaDEM_Particles.hpp:349-370) and its history with partners as global ids.

This is the host-side plan of the decomposition: one host round trip per step.  Bonds and
triangle meshes are not decomposed (a bond partner may leave the halo); `step_fn` sees plane
walls only."""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist

from ._lib import DemError
from .state import ParticleState, WallState

_VEC = ("x", "u", "omega", "force", "torque")
_SCAL = ("m", "rho", "rad", "I", "E", "nu", "G")


def _layout(mc: int, mw: int):
    """Column ranges of one particle row: name -> (first column, width)."""
    cols, at = {}, 0
    for name, w in (("gid", 1), *((v, 3) for v in _VEC), *((s, 1) for s in _SCAL), ("tng_count", 1),
                    ("tng_idx", mc), ("tng_ss_x", mc), ("tng_ss_y", mc), ("tng_ss_z", mc),
                    ("tng_sw_x", mw), ("tng_sw_y", mw), ("tng_sw_z", mw)):
        cols[name] = (at, w)
        at += w
    return cols, at


class SlabDecomposition:
    """Slabs of equal width along `axis` over [lo, hi]; rank r owns lo + r w <= x < lo + (r+1) w
    (the end slabs also own what lies beyond lo and hi)."""

    def __init__(self, axis: int, lo: float, hi: float, halo: float, max_cnts: int, max_walls: int,
                 group=None, device="cpu"):
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.axis, self.lo, self.hi, self.halo = int(axis), float(lo), float(hi), float(halo)
        self.width = (self.hi - self.lo) / self.world
        if not (self.width > 0.0 and self.halo >= 0.0):
            raise DemError("SlabDecomposition: hi > lo and halo >= 0 required")
        if self.world > 1 and self.halo > self.width:
            raise DemError("SlabDecomposition: slab width %.6g below halo %.6g" % (self.width, self.halo))
        self.mc, self.mw = int(max_cnts), max(int(max_walls), 1)
        self.cols, self.ncols = _layout(self.mc, self.mw)
        self.device = torch.device(device)
        self.slab_lo = self.lo + self.rank * self.width
        self.slab_hi = self.lo + (self.rank + 1) * self.width
        self.peers = [p for p in (self.rank - 1, self.rank + 1) if 0 <= p < self.world]
        self.rows = np.zeros((0, self.ncols))
        self.migrated = 0      # particles this rank sent to a neighbour, since creation
        self.ghosts = 0        # ghost rows this rank received at the last step

    # ---- ownership
    def owner(self, coord: np.ndarray) -> np.ndarray:
        return np.clip(np.floor((coord - self.lo) / self.width), 0, self.world - 1).astype(np.int64)

    def scatter(self, state: ParticleState):
        """Take this rank's rows of a global state known to every rank (global id = index)."""
        if state.max_cnts != self.mc or state.tng_sw_x.shape[1] != self.mw:
            raise DemError("scatter: MaxCnts / MaxNoWalls differ from the decomposition's")
        own = self.owner(state.x[:, self.axis]) == self.rank
        self.rows = self._pack(state, np.flatnonzero(own), np.arange(state.n, dtype=np.int64))

    # ---- rows <-> ParticleState
    def _col(self, rows, name):
        a, w = self.cols[name]
        return rows[:, a:a + w]

    def _pack(self, st: ParticleState, idx: np.ndarray, gid_of: np.ndarray) -> np.ndarray:
        """Rows of particles idx of st; gid_of maps st's indices (and history partners) to global ids."""
        rows = np.empty((len(idx), self.ncols))
        self._col(rows, "gid")[:, 0] = gid_of[idx]
        for f in _VEC:
            self._col(rows, f)[:] = getattr(st, f)[idx]
        for f in _SCAL:
            self._col(rows, f)[:, 0] = getattr(st, f)[idx]
        cnt = st.tng_count[idx].astype(np.int64)
        self._col(rows, "tng_count")[:, 0] = cnt
        live = np.arange(self.mc)[None, :] < cnt[:, None]
        part = st.tng_idx[idx].astype(np.int64)
        self._col(rows, "tng_idx")[:] = np.where(live, gid_of[np.where(live, part, 0)], -1)
        for c in "xyz":
            self._col(rows, "tng_ss_" + c)[:] = getattr(st, "tng_ss_" + c)[idx]
            self._col(rows, "tng_sw_" + c)[:] = getattr(st, "tng_sw_" + c)[idx]
        return rows

    def _unpack(self, rows: np.ndarray, owned: np.ndarray) -> ParticleState:
        """ParticleState of rows sorted by global id; history partners (global ids) become
        local indices for owned rows; ghosts carry no history (their results are dropped)."""
        n = rows.shape[0]
        st = ParticleState.create(n, self.mc, self.mw)
        for f in _VEC:
            getattr(st, f)[:] = self._col(rows, f)
        for f in _SCAL:
            getattr(st, f)[:] = self._col(rows, f)[:, 0]
        gid = self._col(rows, "gid")[:, 0].astype(np.int64)
        cnt = np.where(owned, self._col(rows, "tng_count")[:, 0], 0).astype(np.int32)
        live = np.arange(self.mc)[None, :] < cnt[:, None]
        part = self._col(rows, "tng_idx").astype(np.int64)
        loc = np.searchsorted(gid, np.where(live, part, gid[0] if n else 0))
        found = (loc < n) & (gid[np.minimum(loc, max(n - 1, 0))] == part)
        if n and not np.all(found | ~live):
            raise DemError("slab step: a tracked contact partner is outside the halo")
        st.tng_idx[:] = np.where(live, loc, -1).astype(np.int32)
        st.tng_count[:] = cnt
        for c in "xyz":
            getattr(st, "tng_ss_" + c)[:] = np.where(live, self._col(rows, "tng_ss_" + c), 0.0)
            getattr(st, "tng_sw_" + c)[:] = self._col(rows, "tng_sw_" + c)
        return st

    # ---- point-to-point exchange with the neighbouring slabs
    def _exchange(self, out: dict) -> list:
        """Send out[p] (rows, possibly none) to each neighbour p; return the rows received."""
        if not self.peers:
            return []
        dev = self.device
        sc = {p: torch.tensor([len(out.get(p, ()))], dtype=torch.int64, device=dev) for p in self.peers}
        rc = {p: torch.zeros(1, dtype=torch.int64, device=dev) for p in self.peers}
        ops = []
        for p in self.peers:
            ops.append(dist.P2POp(dist.isend, sc[p], p, self.group))
            ops.append(dist.P2POp(dist.irecv, rc[p], p, self.group))
        for w in dist.batch_isend_irecv(ops):
            w.wait()
        ops, recv, keep = [], {}, []
        for p in self.peers:
            k = int(len(out.get(p, ())))
            if k:
                t = torch.from_numpy(np.ascontiguousarray(out[p], dtype=np.float64)).to(dev)
                keep.append(t)
                ops.append(dist.P2POp(dist.isend, t, p, self.group))
            r = int(rc[p].item())
            if r:
                recv[p] = torch.empty((r, self.ncols), dtype=torch.float64, device=dev)
                ops.append(dist.P2POp(dist.irecv, recv[p], p, self.group))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        return [recv[p].cpu().numpy() for p in self.peers if p in recv]

    # ---- one step
    def _agree(self, err: str):
        """Collective check: every rank raises when any rank met an error, so that no rank is
        left waiting in the next exchange."""
        flag = torch.tensor([1 if err else 0], dtype=torch.int64, device=self.device)
        dist.all_reduce(flag, op=dist.ReduceOp.MAX, group=self.group)
        if int(flag.item()):
            raise DemError(err or "slab step: another rank failed")

    def step(self, step_fn):
        """Migrate, exchange ghosts, step the local set once with step_fn(ParticleState) (in
        place), keep the owned rows."""
        coord = self._col(self.rows, "x")[:, self.axis]
        dest = self.owner(coord)
        self._agree("slab step: a particle moved past a whole slab in one step"
                    if np.any(np.abs(dest - self.rank) > 1) else "")
        out = {p: self.rows[dest == p] for p in self.peers}
        self.migrated += sum(len(v) for v in out.values())
        got = self._exchange(out)
        self.rows = np.vstack([self.rows[dest == self.rank], *got])
        coord = self._col(self.rows, "x")[:, self.axis]
        gout = {}
        if self.rank - 1 in self.peers:
            gout[self.rank - 1] = self.rows[coord < self.slab_lo + self.halo]
        if self.rank + 1 in self.peers:
            gout[self.rank + 1] = self.rows[coord >= self.slab_hi - self.halo]
        ghosts = self._exchange(gout)
        self.ghosts = sum(len(g) for g in ghosts)
        local = np.vstack([self.rows, *ghosts])
        owned = np.zeros(len(local), dtype=bool)
        owned[: len(self.rows)] = True
        order = np.argsort(self._col(local, "gid")[:, 0], kind="stable")
        local, owned = local[order], owned[order]
        err, st = "", None
        try:
            st = self._unpack(local, owned)
        except DemError as e:
            err = str(e)
        self._agree(err)
        x0 = st.x[owned, self.axis].copy()
        try:
            if owned.any():      # a rank with an empty slab (or ghosts only) has nothing to step
                step_fn(st)
        except DemError as e:
            err = "slab step: " + str(e)
        if not err and self.world > 1 and st.n:
            margin = max(self.halo - 2.0 * float(st.rad.max()), 0.0) / 2.0
            if np.any(np.abs(st.x[owned, self.axis] - x0) > margin):
                err = "slab step: a particle moved more than (halo - 2 r_max) / 2 in one step"
        self._agree(err)
        gid = self._col(local, "gid")[:, 0].astype(np.int64)
        self.rows = self._pack(st, np.flatnonzero(owned), gid)

    def run(self, step_fn, nsteps: int):
        for _ in range(int(nsteps)):
            self.step(step_fn)

    # ---- results
    def kinetic_energy(self) -> float:
        """Total translational + rotational kinetic energy of the scene (collective: every rank
        calls it and gets the same value), summed per rank over its own particles in global-id
        order, then over the ranks in rank order.  The rank sums are gathered rather than
        all-reduced so that every rank adds them in the same order."""
        gid = self._col(self.rows, "gid")[:, 0]
        rows = self.rows[np.argsort(gid, kind="stable")]
        u, w = self._col(rows, "u"), self._col(rows, "omega")
        m, inertia = self._col(rows, "m")[:, 0], self._col(rows, "I")[:, 0]
        e = 0.0
        for k in range(len(rows)):
            e += 0.5 * m[k] * (u[k, 0] * u[k, 0] + u[k, 1] * u[k, 1] + u[k, 2] * u[k, 2]) + \
                0.5 * inertia[k] * (w[k, 0] * w[k, 0] + w[k, 1] * w[k, 1] + w[k, 2] * w[k, 2])
        mine = torch.tensor([e], dtype=torch.float64, device=self.device)
        parts = [torch.zeros(1, dtype=torch.float64, device=self.device) for _ in range(self.world)]
        dist.all_gather(parts, mine, group=self.group)
        total = 0.0
        for p in parts:
            total += float(p.item())
        return total

    def gather(self) -> ParticleState | None:
        """The global state on rank 0 (particles in global-id order, history partners as global
        ids), None on the other ranks."""
        parts = [None] * self.world if self.rank == 0 else None
        dist.gather_object(self.rows, parts, dst=0, group=self.group)
        if self.rank != 0:
            return None
        rows = np.vstack(parts)
        rows = rows[np.argsort(self._col(rows, "gid")[:, 0], kind="stable")]
        gid = self._col(rows, "gid")[:, 0].astype(np.int64)
        if not np.array_equal(gid, np.arange(len(gid))):
            raise DemError("gather: global ids are not 0..n-1 exactly once")
        n = len(gid)
        st = ParticleState.create(n, self.mc, self.mw)
        for f in _VEC:
            getattr(st, f)[:] = self._col(rows, f)
        for f in _SCAL:
            getattr(st, f)[:] = self._col(rows, f)[:, 0]
        st.tng_count[:] = self._col(rows, "tng_count")[:, 0].astype(np.int32)
        st.tng_idx[:] = self._col(rows, "tng_idx").astype(np.int32)
        for c in "xyz":
            getattr(st, "tng_ss_" + c)[:] = self._col(rows, "tng_ss_" + c)
            getattr(st, "tng_sw_" + c)[:] = self._col(rows, "tng_sw_" + c)
        return st


class DeviceStep:
    """step_fn on this rank's GPU through the public API: upload the local set, one step of the
    device solver, download.  Plane walls keep their positions across calls (kinematic walls
    advance inside the solver)."""

    def __init__(self, walls: WallState | None, params: dict, dt: float, skin: float = 0.0, delta: float = 0.0,
                 gravity=(0.0, 0.0, 0.0), ctx=None, api=None):
        if api is None:      # the device library's Python API (a stand-in with the same calls in tests)
            from . import api
        self.api = api
        self.walls = walls.copy() if walls is not None and walls.n > 0 else None
        self.force = api.Force(params["cor_pp"], params["cor_pw"], params["mu_pp"], params["mu_pw"],
                               params.get("quirks", api.REF_COMPAT))
        self.dt, self.skin, self.delta, self.gravity = float(dt), float(skin), float(delta), tuple(gravity)
        self.ctx = ctx or api.default_context()

    def __call__(self, st: ParticleState):
        api = self.api
        nw = self.walls.n if self.walls is not None else 0
        p = api.Particles(st.n, st.max_cnts, nw, ctx=self.ctx)
        w = s = None
        try:
            p.upload(st)
            if self.walls is not None:
                w = api.Wall(nw, ctx=self.ctx)
                w.upload(self.walls)
            s = api.SolverDEM(p, w, self.force, self.dt, delta=self.delta, skin=self.skin, gravity=self.gravity)
            s.run_steps(1)
            if self.walls is not None:
                self.walls.x[:] = s.wall_positions()
            out = p.download()
        finally:      # the solver before the particles and walls it refers to
            if s is not None:
                s.close()
            if w is not None:
                w.close()
            p.close()
        for k, v in out.arrays().items():
            a = getattr(st, k)
            if k.startswith("tng_sw_"):      # the device holds one column per wall
                c = min(a.shape[1], v.shape[1])
                a[:, :c] = v[:, :c]
            else:
                a[...] = v
