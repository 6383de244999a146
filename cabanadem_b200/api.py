"""Python mirror of the reference's operator interface, running on libb200dem.so.

Names, argument meaning and step semantics follow the reference:

=========================================  ================================================
reference (file:line)                      here
=========================================  ================================================
Particles<Mem,3,MaxCnts,MaxNoWalls>        :class:`Particles` (capacities at run time)
  (src/CabanaDEM_Particles.hpp:22-71)
  slicePosition() ... (:99-271)            ``slicePosition()`` ... (host copies),
                                           ``set(field, array)`` / ``get(field)``
  updateParticles(exec, functor) (:91-97)  ``updateParticles(functor)`` (host functor on a
                                           ParticleState, then upload)
Wall<Mem,3> (src/CabanaDEM_Wall.hpp:22)    :class:`Wall`
Force(cor_pp, cor_pw, mu_pp, mu_pw)        :class:`Force`
  (src/CabanaDEM_Force.hpp:23-35)
Integrator(dt).stage1/2/3                  :class:`Integrator` (bound to a solver)
  (src/CabanaDEM_Integrator.hpp:16-102)
computeForceParticleParticleInfiniteWall   :func:`computeForceParticleParticleInfiniteWall`
  (src/CabanaDEM_Force.hpp:700-710)
createSolverDEM / SolverDEM::run           :func:`createSolverDEM`, :meth:`SolverDEM.run`
  (src/CabanaDEM_Solver.hpp:66-138)        (num_steps + 1 steps, as the reference loop)
=========================================  ================================================
"""
from __future__ import annotations

import ctypes as C
import os
import weakref

import numpy as np

from . import _lib
from ._lib import DemError, F, W, check, lib
from .inputs import Inputs
from .state import ParticleState, WallState

REF_COMPAT = 0x3F

_F_DTYPE = {"tng_idx": np.int32, "tng_count": np.int32, "fix": np.uint8, "scene": np.int32}


def _shape(field, n, mc, mw):
    if field in ("x", "u", "omega", "force", "torque", "ext_force"):
        return (n, 3)
    if field in ("tng_idx", "tng_ss_x", "tng_ss_y", "tng_ss_z"):
        return (n, mc)
    if field in ("tng_sw_x", "tng_sw_y", "tng_sw_z"):
        return (n, mw)
    return (n,)


class Context:
    """One device + one CUDA stream (dem_ctx)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        st = lib().dem_ctx_create(int(device), C.byref(h))
        if st:
            raise DemError("dem_ctx_create failed (status %d): no usable CUDA device" % st)
        self.h = h
        self._children = []   # weak references to objects created on this context, in order

    def adopt(self, obj):
        """Register an object created on this context; close() closes it first."""
        self._children.append(weakref.ref(obj))

    def sync(self):
        check(lib().dem_ctx_sync(self.h), self.h, "dem_ctx_sync")

    def stream_ptr(self) -> int:
        """cudaStream_t of this context (for CUDA events on the library's stream)."""
        return int(lib().dem_ctx_stream(self.h) or 0)

    def close(self):
        """Destroy the context after closing every object created on it (newest first)."""
        if self.h:
            for r in reversed(self._children):
                o = r()
                if o is not None:
                    o.close()
            self._children = []
            lib().dem_ctx_destroy(self.h)
            self.h = None

    @property
    def alive(self) -> bool:
        return bool(self.h)


_default_ctx = None


def default_context():
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


class Particles:
    output_folder = ""      # Particles(exec, n, output_folder) of the reference; "" writes nothing
    output_format = None    # "csv", "xdmf" or "both"; None: $CABANADEM_OUTPUT_FORMAT, else "csv"

    def __init__(self, n: int, max_cnts: int = 6, max_walls: int = 1, ctx: Context | None = None,
                 output_folder: str = ""):
        self.ctx = ctx or default_context()
        self.n, self.max_cnts, self.max_walls = int(n), int(max_cnts), int(max_walls)
        h = C.c_void_p()
        check(lib().dem_particles_create(self.ctx.h, self.n, self.max_cnts, self.max_walls, C.byref(h)),
              self.ctx.h, "dem_particles_create")
        self.h = h
        self.ctx.adopt(self)
        if output_folder:      # Particles.hpp:53-61: created if it does not exist
            os.makedirs(output_folder, exist_ok=True)
            self.output_folder = str(output_folder)

    # ---- output and resize (Particles.hpp:273-346)
    def setOutputFormat(self, fmt: str):
        if fmt not in ("csv", "xdmf", "both"):
            raise DemError("setOutputFormat: csv, xdmf or both")
        self.output_format = fmt

    def output(self, output_step: int, output_time: float):
        """One snapshot of the current state in the output folder (Particles.hpp:299-346):
        particles_<step>.csv and/or particles_<step>.xmf + .bin, as the C++ interface writes them."""
        if not self.output_folder:
            return
        from . import snapshots
        fmt = self.output_format or os.environ.get("CABANADEM_OUTPUT_FORMAT", "csv")
        if fmt not in ("csv", "xdmf", "both"):
            raise DemError("output format: csv, xdmf or both, got %r" % fmt)
        st = self.download()
        if fmt != "xdmf":
            snapshots.write_csv(self.output_folder, int(output_step), float(output_time), st)
        if fmt != "csv":
            snapshots.write_xdmf(self.output_folder, int(output_step), float(output_time), st)

    def resize(self, n: int):
        """Particles::resize(n) (Particles.hpp:273-297): the first min(n, size) particles keep
        their values, added ones start zeroed with empty contact slots.  The device set is
        re-created, so no solver may use it (create solvers after the last resize); external
        forces and fix flags are reset."""
        for r in self.ctx._children:
            o = r()
            if o is not None and o is not self and getattr(o, "particles", None) is self and getattr(o, "h", None):
                raise DemError("Particles.resize: a solver is attached to this particle set")
        st = self.download().resized(int(n))
        h = C.c_void_p()
        check(lib().dem_particles_create(self.ctx.h, int(n), self.max_cnts, self.max_walls, C.byref(h)),
              self.ctx.h, "dem_particles_create")
        lib().dem_particles_destroy(self.h)
        self.h, self.n = h, int(n)
        self.upload(st)

    # ---- field access
    def set(self, field: str, arr):
        """Upload a field in caller order.  From page-locked (pinned) memory the copy is queued
        on the context's stream: keep `arr` unchanged until a call that synchronises (get, a
        run, Context.sync); other arrays are read before set returns."""
        dt = _F_DTYPE.get(field, np.float64)
        a = np.ascontiguousarray(arr, dtype=dt)
        exp = _shape(field, self.n, self.max_cnts, self.max_walls)
        if a.size != int(np.prod(exp)):
            raise DemError("set(%s): expected shape %s, got %s" % (field, exp, a.shape))
        check(lib().dem_particles_set(self.h, F[field], a.ctypes.data, a.size), self.ctx.h, "set " + field)

    def get(self, field: str, out=None):
        """Host copy of a field in caller order; `out` (a C-contiguous array of the field's
        dtype and size, e.g. in pinned memory) receives it instead of a new array."""
        dt = _F_DTYPE.get(field, np.float64)
        shape = _shape(field, self.n, self.max_cnts, self.max_walls)
        if out is None:
            a = np.empty(shape, dtype=dt)
        else:
            a = out
            if a.dtype != dt or a.size != int(np.prod(shape)) or not a.flags["C_CONTIGUOUS"]:
                raise DemError("get(%s): out must be C-contiguous %s of %d elements" % (field, np.dtype(dt).name,
                                                                                         int(np.prod(shape))))
        check(lib().dem_particles_get(self.h, F[field], a.ctypes.data, a.size), self.ctx.h, "get " + field)
        return a

    def get_device(self, field: str, out):
        """Copy a field in caller order into the device buffer `out` (a torch tensor of the
        field's element count, e.g. float64 [n, 3] for "x"), queued on this context's stream."""
        check(lib().dem_particles_get_device(self.h, F[field], C.c_void_p(out.data_ptr()), out.numel()), self.ctx.h,
              "get_device " + field)

    def save(self, path: str):
        """Checkpoint every field (caller order) to `path` (dem_checkpoint_save)."""
        check(lib().dem_checkpoint_save(self.h, str(path).encode()), self.ctx.h, "dem_checkpoint_save")

    def load(self, path: str):
        """Restore a checkpoint written by save() (same n, MaxCnts, MaxNoWalls)."""
        check(lib().dem_checkpoint_load(self.h, str(path).encode()), self.ctx.h, "dem_checkpoint_load")

    def clear_contacts(self):
        """Contact counts 0, slot partners -1, slot and wall history 0, on the device
        (dem_particles_clear_contacts): a fresh start without uploading zero history."""
        check(lib().dem_particles_clear_contacts(self.h), self.ctx.h, "dem_particles_clear_contacts")

    def clear_forces(self):
        """Force and torque zero on the device (dem_particles_clear_forces), as new particles have
        them: with clear_contacts, a fresh start from uploaded positions and velocities."""
        check(lib().dem_particles_clear_forces(self.h), self.ctx.h, "dem_particles_clear_forces")

    def upload(self, s: ParticleState):
        for f in ("rad", "x", "u", "omega", "force", "torque", "m", "I", "rho", "E", "nu", "G",
                  "tng_idx", "tng_ss_x", "tng_ss_y", "tng_ss_z", "tng_count"):
            self.set(f, getattr(s, f))
        if self.max_walls > 0:
            for f in ("tng_sw_x", "tng_sw_y", "tng_sw_z"):
                self.set(f, getattr(s, f)[:, : self.max_walls])

    def download(self) -> ParticleState:
        s = ParticleState.create(self.n, self.max_cnts, max(self.max_walls, 1))
        for f in ("x", "u", "omega", "force", "torque", "m", "I", "rho", "rad", "E", "nu", "G",
                  "tng_idx", "tng_ss_x", "tng_ss_y", "tng_ss_z", "tng_count"):
            setattr(s, f, self.get(f))
        if self.max_walls > 0:
            for f in ("tng_sw_x", "tng_sw_y", "tng_sw_z"):
                setattr(s, f, self.get(f))
        return s

    def updateParticles(self, functor):
        """Run a host functor over a ParticleState copy, then upload it."""
        s = self.download()
        for pid in range(self.n):
            functor(s, pid)
        self.upload(s)

    # reference-named accessors (host copies)
    def slicePosition(self): return self.get("x")
    def sliceVelocity(self): return self.get("u")
    def sliceOmega(self): return self.get("omega")
    def sliceForce(self): return self.get("force")
    def sliceTorque(self): return self.get("torque")
    def sliceMass(self): return self.get("m")
    def sliceDensity(self): return self.get("rho")
    def sliceRadius(self): return self.get("rad")
    def sliceMomentOfInertia(self): return self.get("I")
    def sliceYoungsMod(self): return self.get("E")
    def slicePoissonsRatio(self): return self.get("nu")
    def sliceShearMod(self): return self.get("G")
    def sliceTangentialDispIdx(self): return self.get("tng_idx")
    def sliceTangentialDispSSx(self): return self.get("tng_ss_x")
    def sliceTangentialDispSSy(self): return self.get("tng_ss_y")
    def sliceTangentialDispSSz(self): return self.get("tng_ss_z")
    def sliceTotalNoTangentialContacts(self): return self.get("tng_count")
    def sliceTangentialDispSWx(self): return self.get("tng_sw_x")
    def sliceTangentialDispSWy(self): return self.get("tng_sw_y")
    def sliceTangentialDispSWz(self): return self.get("tng_sw_z")

    def close(self):
        if self.h and self.ctx.alive:   # a closed context has closed this object already
            lib().dem_particles_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Wall:
    def __init__(self, n: int, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self.n = int(n)
        h = C.c_void_p()
        check(lib().dem_walls_create(self.ctx.h, self.n, C.byref(h)), self.ctx.h, "dem_walls_create")
        self.h = h
        self.ctx.adopt(self)

    def set(self, field, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        check(lib().dem_walls_set(self.h, W[field], a.ctypes.data, a.size), self.ctx.h, "wall set " + field)

    def upload(self, w: WallState):
        for f in ("x", "u", "omega", "normal", "E", "nu", "G"):
            self.set(f, getattr(w, f))

    def close(self):
        if self.h and self.ctx.alive:
            lib().dem_walls_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Force:
    """Force(cor_pp, cor_pw, friction_pp, friction_pw) (src/CabanaDEM_Force.hpp:23-35)."""

    def __init__(self, cor_pp, cor_pw, friction_pp, friction_pw, quirks=REF_COMPAT):
        self.cor_pp, self.cor_pw = float(cor_pp), float(cor_pw)
        self.friction_pp, self.friction_pw = float(friction_pp), float(friction_pw)
        self.quirks = int(quirks)

    def params(self):
        return _lib.ForceParams(self.cor_pp, self.cor_pw, self.friction_pp, self.friction_pw, self.quirks)


class SolverDEM:
    """SolverDEM (src/CabanaDEM_Solver.hpp:13-122) on the device."""

    def __init__(self, particles: Particles, wall: Wall | None, force: Force, dt: float, delta: float = 0.0,
                 skin: float = 0.0, rebuild_every_step: bool = False, gravity=(0.0, 0.0, 0.0),
                 precision: int = _lib.DEM_FP64, num_steps: int = 0, output_frequency: int = 0,
                 max_neighbors: int = 0, steps_per_launch: int = 0, stream_block: int = 0,
                 contact_lanes: int = 0, stream_split: int = 0, dense_form: int = 0, scene_kernel: int = 0,
                 launch_overlap: int = 0, cooperative_loop: int = 0):
        self.particles, self.wall, self.force = particles, wall, force
        self.dt, self.num_steps, self.output_frequency = float(dt), int(num_steps), int(output_frequency)
        sp = _lib.SolverParams()
        sp.dt, sp.delta, sp.skin = float(dt), float(delta), float(skin)
        sp.rebuild_every_step = 1 if rebuild_every_step else 0
        sp.precision = int(precision)
        sp.gravity = (C.c_double * 3)(*gravity)
        sp.max_neighbors = int(max_neighbors)
        sp.steps_per_launch = int(steps_per_launch)
        sp.stream_block = int(stream_block)
        sp.contact_lanes = int(contact_lanes)
        sp.stream_split = int(stream_split)
        sp.dense_form = int(dense_form)
        sp.scene_kernel = int(scene_kernel)
        sp.launch_overlap = int(launch_overlap)
        sp.cooperative_loop = int(cooperative_loop)
        fp = force.params()
        h = C.c_void_p()
        check(lib().dem_solver_create(particles.ctx.h, particles.h, wall.h if wall else None, C.byref(fp),
                                      C.byref(sp), C.byref(h)), particles.ctx.h, "dem_solver_create")
        self.h = h
        particles.ctx.adopt(self)
        self.integrator = Integrator(self)
        self.last_status = 0

    def run(self):
        """Reference loop: for step in 0..num_steps inclusive (Solver.hpp:79)."""
        return self.run_steps(self.num_steps + 1)

    def run_steps(self, nsteps: int, allow=_lib.DEM_ERR_CONTACT_OVERFLOW):
        st = lib().dem_solver_run(self.h, int(nsteps))
        self.last_status = st
        return check(st, self.particles.ctx.h, "dem_solver_run", allow=allow)

    def set_mesh(self, tri, E, nu, G, velocity=None, max_contacts=8):
        """Triangle-mesh wall: tri [nt, 3, 3] vertex coordinates, one material, optional
        translation velocity (applied when the force's DEM_Q6_WALL_STATIC bit is clear)
        (dem_solver_set_mesh)."""
        t = np.ascontiguousarray(tri, dtype=np.float64).reshape(-1, 9)
        v = None if velocity is None else np.ascontiguousarray(velocity, dtype=np.float64)
        check(lib().dem_solver_set_mesh(self.h, t.ctypes.data if t.size else None, t.shape[0], float(E), float(nu),
                                        float(G), v.ctypes.data if v is not None else None, int(max_contacts)),
              self.particles.ctx.h, "dem_solver_set_mesh")

    def mesh_translation(self):
        out = np.zeros(3)
        check(lib().dem_solver_mesh_translation(self.h, out.ctypes.data), self.particles.ctx.h,
              "dem_solver_mesh_translation")
        return out

    def wall_positions(self):
        """Current positions [nw, 3] of the solver's walls: walls with a velocity move by
        dt * u each step when the force's DEM_Q6_WALL_STATIC bit is clear."""
        nw = self.wall.n if self.wall is not None else 0
        out = np.zeros((nw, 3))
        check(lib().dem_solver_wall_positions(self.h, out.ctypes.data, out.size), self.particles.ctx.h,
              "dem_solver_wall_positions")
        return out

    def stats(self):
        s = _lib.RunStats()
        check(lib().dem_solver_stats(self.h, C.byref(s)), self.particles.ctx.h, "dem_solver_stats")
        return {k: getattr(s, k) for k, _ in s._fields_}

    def set_scenes(self, params, walls_per_scene: int):
        """Batched independent scenes: params is a sequence of (cor_pp, cor_pw, mu_pp, mu_pw)
        per scene; the particles' "scene" field assigns them (dem_solver_set_scenes)."""
        arr = (_lib.SceneParams * len(params))(*[_lib.SceneParams(*map(float, p)) for p in params])
        check(lib().dem_solver_set_scenes(self.h, arr, len(params), int(walls_per_scene)), self.particles.ctx.h,
              "dem_solver_set_scenes")

    def profile_steps(self, nsteps: int) -> float:
        """Run nsteps fused steps launched one by one between CUDA events; returns the
        mean duration (ms) of one fused step launch."""
        ms = C.c_double(0.0)
        check(lib().dem_solver_profile(self.h, int(nsteps), C.byref(ms)), self.particles.ctx.h,
              "dem_solver_profile", allow=_lib.DEM_ERR_CONTACT_OVERFLOW)
        return ms.value

    def build_neighbors(self):
        check(lib().dem_build_neighbors(self.h), self.particles.ctx.h, "dem_build_neighbors")

    def rebuild(self):
        """The time loop's rebuild, now: Morton re-sort, new list, displacement bound reset
        (dem_solver_rebuild)."""
        check(lib().dem_solver_rebuild(self.h), self.particles.ctx.h, "dem_solver_rebuild")

    def compute_force(self):
        return check(lib().dem_compute_force(self.h), self.particles.ctx.h, "dem_compute_force",
                     allow=_lib.DEM_ERR_CONTACT_OVERFLOW)

    def neighbors(self):
        n = self.particles.n
        off = np.zeros(n + 1, dtype=np.int32)
        tot = C.c_long(0)
        check(lib().dem_neighbors_get(self.h, off.ctypes.data, None, C.byref(tot)), self.particles.ctx.h, "nbr")
        idx = np.zeros(max(tot.value, 1), dtype=np.int32)
        check(lib().dem_neighbors_get(self.h, off.ctypes.data, idx.ctypes.data, C.byref(tot)),
              self.particles.ctx.h, "nbr")
        return off, idx[: tot.value]

    def energy(self):
        out = (C.c_double * 4)()
        check(lib().dem_energy(self.h, out), self.particles.ctx.h, "dem_energy")
        return np.array(out[:])

    def close(self):
        if self.h and self.particles.ctx.alive:
            lib().dem_solver_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Integrator:
    """Integrator::stage1/2/3 (src/CabanaDEM_Integrator.hpp:31-102) on a solver's particles."""

    def __init__(self, solver: SolverDEM):
        self._s = solver

    def stage1(self, particles=None):
        check(lib().dem_stage1(self._s.h), self._s.particles.ctx.h, "stage1")

    def stage2(self, particles=None):
        check(lib().dem_stage2(self._s.h), self._s.particles.ctx.h, "stage2")

    def stage3(self, particles=None):
        check(lib().dem_stage3(self._s.h), self._s.particles.ctx.h, "stage3")


def computeForceParticleParticleInfiniteWall(solver: SolverDEM):
    """src/CabanaDEM_Force.hpp:700-710: zero, compact contacts, pp force, wall force."""
    return solver.compute_force()


def createSolverDEM(inputs: Inputs, particles: Particles, wall: Wall, force: Force, delta: float, **kw):
    """createSolverDEM<Mem>(inputs, particles, wall, force, delta) (src/CabanaDEM_Solver.hpp:129-138).
    The reference rebuilds the list every step with cutoff delta; that is the default here."""
    kw.setdefault("rebuild_every_step", True)
    return SolverDEM(particles, wall, force, float(inputs["timestep"]), delta=delta,
                     num_steps=int(inputs["num_steps"]), output_frequency=int(inputs["output_frequency"]), **kw)


def from_scenario(sc, ctx: Context | None = None, rebuild_every_step=False, precision=_lib.DEM_FP64,
                  steps_per_launch=0, max_neighbors=0, stream_block=0, contact_lanes=0, stream_split=0,
                  dense_form=0, scene_kernel=0, launch_overlap=0, cooperative_loop=0):
    """Particles + Wall + SolverDEM on the device for a scenarios.Scenario."""
    st = sc.state
    nwalls = sc.walls.n if sc.walls is not None else 0
    if sc.extra.get("scene") is not None:
        nwalls = sc.extra["walls_per_scene"]
    p = Particles(st.n, st.max_cnts, nwalls, ctx=ctx)
    p.upload(st)
    w = None
    if sc.walls is not None and sc.walls.n > 0:
        w = Wall(sc.walls.n, ctx=p.ctx)
        w.upload(sc.walls)
    prm = sc.params
    f = Force(prm["cor_pp"], prm["cor_pw"], prm["mu_pp"], prm["mu_pw"], prm.get("quirks", REF_COMPAT))
    s = SolverDEM(p, w, f, sc.dt, delta=sc.delta, skin=sc.skin, rebuild_every_step=rebuild_every_step,
                  gravity=sc.gravity, precision=precision, steps_per_launch=steps_per_launch,
                  max_neighbors=max_neighbors, stream_block=stream_block, contact_lanes=contact_lanes,
                  stream_split=stream_split, dense_form=dense_form, scene_kernel=scene_kernel,
                  launch_overlap=launch_overlap, cooperative_loop=cooperative_loop)
    if sc.extra.get("scene") is not None:
        p.set("scene", sc.extra["scene"])
        s.set_scenes(sc.extra["scene_params"], sc.extra["walls_per_scene"])
    m = sc.extra.get("mesh")
    if m is not None:
        s.set_mesh(m.tri, m.E, m.nu, m.G, velocity=m.u, max_contacts=m.max_contacts)
    return s


class BatchRunner:
    """Independent scenes of a batched set (scenarios.batched_scenes) grouped by scene size
    (scenarios.split_scenes): each size bucket is one solver, with the launch settings tuned for
    that bucket (`configs[bucket]`; else autotune.tune on the bucket's scenes when `tune`; else
    the B200 settings shipped with the package for that bucket, autotune.packaged, or the
    defaults), on a context of its own, so on a CUDA stream of its own.  run_steps advances every bucket at once: one host
    thread per bucket, each a graph-looped run of its solver, the buckets' kernels running
    concurrently on the GPU.  Scenes never interact, so every scene evolves as it does alone."""

    def __init__(self, sc, precision=_lib.DEM_FP64, configs=None, tune=False, device=0, tune_steps=300):
        from . import autotune, scenarios as S
        self.n = sc.state.n
        self.parts = []
        buckets = list(S.split_scenes(sc))
        # the buckets' solvers run concurrently on their own streams: no dependent launches, whose
        # early-resident waiting blocks would hold SM resources the other buckets' kernels use
        # (1,024-scene batch: 73.2 against 77.8 us per step)
        overlap = 2 if len(buckets) > 1 else 0
        for b, sub, ids in buckets:
            cfg = (configs or {}).get(b)
            if cfg is None and tune:
                # long enough trials to see the rebuild cadence each skin gives (a rebuild every
                # 50-100 steps in the fired clusters)
                cfg = autotune.tune(sub, precision=precision, warmup=20, steps=tune_steps)
            elif cfg is None:
                cfg = autotune.packaged(sub, precision)   # B200 settings shipped with the package
            cfg = dict(autotune.DEFAULTS, **(cfg or {}))
            kw = autotune.apply(sub, cfg)
            ctx = Context(device)
            self.parts.append(dict(bucket=b, scenario=sub, scenes=ids, ctx=ctx, config=cfg,
                                   solver=from_scenario(sub, ctx=ctx, precision=precision, launch_overlap=overlap,
                                                        **kw)))

    def run_steps(self, nsteps: int):
        import threading
        errors = []

        def work(s):
            try:
                s.run_steps(nsteps)
            except Exception as e:   # re-raised on the calling thread
                errors.append(e)
        threads = [threading.Thread(target=work, args=(p["solver"],)) for p in self.parts]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if errors:
            raise errors[0]

    def download(self) -> ParticleState:
        """The whole batch's state in the original particle order."""
        parts = [(p["scenario"].extra["rows"], p["solver"].particles.download()) for p in self.parts]
        first = parts[0][1]
        out = ParticleState.create(self.n, max_cnts=first.max_cnts, max_walls=first.max_walls)
        for rows, st in parts:
            for f, v in st.arrays().items():
                getattr(out, f)[rows] = v
        return out

    def stats(self):
        return [dict(bucket=p["bucket"], config=p["config"], **p["solver"].stats()) for p in self.parts]

    def close(self):
        for p in self.parts:
            p["solver"].close()
            p["ctx"].close()
        self.parts = []


class Bonds:
    """ParticlesBondedDEM's bond slots (src/CabanaBondedDEM_Particles.hpp:29-293) on a solver's
    particles, with setupBonds (:86-171) and the bonded loop (tst_01_BDEM:295-306)."""

    def __init__(self, solver: SolverDEM, max_bonds: int, quirks=0x07, beta=0.1, radius_factor=1.0, kn=0.0,
                 kt=0.0, break_strain=0.0):
        self.solver = solver
        self.max_bonds = int(max_bonds)
        bp = _lib.BondParams(int(quirks), float(beta), float(radius_factor), float(kn), float(kt),
                             float(break_strain))
        h = C.c_void_p()
        check(lib().dem_bonds_create(solver.h, self.max_bonds, C.byref(bp), C.byref(h)), solver.particles.ctx.h,
              "dem_bonds_create")
        self.h = h
        solver.particles.ctx.adopt(self)

    def setupBonds(self, factor=3.0, search_cutoff=0.0):
        check(lib().dem_bonds_setup(self.h, float(factor), float(search_cutoff)), self.solver.particles.ctx.h,
              "dem_bonds_setup")

    def get(self, field):
        n = self.solver.particles.n
        if field == "count":
            a = np.empty(n, dtype=np.int32)
        elif field == "idx":
            a = np.empty((n, self.max_bonds), dtype=np.int32)
        elif field == "broken":
            a = np.empty((n, self.max_bonds), dtype=np.uint8)
        else:
            a = np.empty((n, self.max_bonds))
        check(lib().dem_bonds_get(self.h, _lib.BFIELD[field], a.ctypes.data, a.size), self.solver.particles.ctx.h,
              "dem_bonds_get " + field)
        return a

    def set(self, field, arr):
        """Upload a bond slice (dem_bonds_set): idx in caller indices (-1 empty), count,
        init_len, the history fields (ft_*, mn_*, mt_*) or broken, shaped as get() returns."""
        dt = {"count": np.int32, "idx": np.int32, "broken": np.uint8}.get(field, np.float64)
        a = np.ascontiguousarray(arr, dtype=dt)
        check(lib().dem_bonds_set(self.h, _lib.BFIELD[field], a.ctypes.data, a.size), self.solver.particles.ctx.h,
              "dem_bonds_set " + field)

    # ---- the bonded loop phase by phase (tst_01_BDEM:295-306)
    def resetForcesAndTorques(self):
        """CabanaBondedDEM::resetForcesAndTorques (src/CabanaBondedDEM_Force.hpp:16-50): F = tau = 0."""
        check(lib().dem_bonded_reset(self.h), self.solver.particles.ctx.h, "dem_bonded_reset")

    def applyExternalForce(self):
        """F += the external force (the example's applyTensileForce, tst_01_BDEM:70-117)."""
        check(lib().dem_apply_external_force(self.solver.h), self.solver.particles.ctx.h, "dem_apply_external_force")

    def computeBondedForce(self, dt: float):
        """CabanaBondedDEM::computeBondedForce(particles, dt) (src/CabanaBondedDEM_Force.hpp:53-348)."""
        return check(lib().dem_bonded_force(self.h, float(dt)), self.solver.particles.ctx.h, "dem_bonded_force")

    def applyBoundaryConditions(self):
        """Gravity, then the fix flags (the example's applyBoundaryConditions, tst_01_BDEM:19-67)."""
        check(lib().dem_apply_boundary_conditions(self.solver.h), self.solver.particles.ctx.h,
              "dem_apply_boundary_conditions")

    def broken(self) -> int:
        """Broken bond ends (each bond of a symmetric pair is counted at both particles)."""
        c = C.c_long(0)
        check(lib().dem_bonds_broken(self.h, C.byref(c)), self.solver.particles.ctx.h, "dem_bonds_broken")
        return c.value

    def run_steps(self, nsteps: int):
        return check(lib().dem_bonded_run(self.h, int(nsteps)), self.solver.particles.ctx.h, "dem_bonded_run")

    def close(self):
        if self.h and self.solver.particles.ctx.alive:
            lib().dem_bonds_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bonded_from_case(case: dict, ctx: Context | None = None, steps_per_launch=0, precision=_lib.DEM_FP64,
                     launch_overlap=0):
    """Particles + SolverDEM + Bonds on the device for a scenarios.bonded_bar /
    bdem_two_particles case (bonds set up).  precision DEM_MIXED keeps the bond
    force/moment history in FP32 (strain, geometry and integration stay FP64)."""
    st = case["state"]
    p = Particles(st.n, max(st.max_cnts, 1), 0, ctx=ctx)
    p.upload(st)
    if case.get("ext_force") is not None:
        p.set("ext_force", case["ext_force"])
    if case.get("fix_flags") is not None:
        p.set("fix", case["fix_flags"])
    s = SolverDEM(p, None, Force(1.0, 1.0, 0.0, 0.0), case["dt"], skin=0.0, steps_per_launch=steps_per_launch,
                  precision=precision, launch_overlap=launch_overlap)
    bp = case["bparams"]
    b = Bonds(s, case["bonds"].max_bonds, quirks=bp["quirks"], beta=bp["beta"], radius_factor=bp["radius_factor"],
              kn=bp["kn"], kt=bp["kt"], break_strain=bp["break_strain"])
    b.setupBonds(case["bond_factor"], case["search_cutoff"])
    return b
