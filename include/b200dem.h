/*
 * b200dem.h -- C ABI of the B200-native DEM contact step (libb200dem.so).
 *
 * The library replaces the Kokkos/Cabana path of CabanaDEM on one GPU: particle storage
 * (Particles.hpp), walls (Wall.hpp), the Hertz-Mindlin force (Force.hpp), the
 * velocity-Verlet integrator (Integrator.hpp), the Verlet neighbour list and the time loop
 * (Solver.hpp), and the bonded-DEM force (CabanaBondedDEM_*.hpp).  Each declaration cites
 * the reference interface it stands in for (paths relative to the reference repository).
 *
 * Conventions
 *  - Every call returns an int status: 0 (DEM_OK) or DEM_ERR_* bits.  Nothing aborts or
 *    traps; dem_last_error() returns a message for the last failure on a context.
 *  - The library owns all device memory.  Host arrays are caller-owned and copied.
 *  - Host arrays use the reference's layout and particle order: vectors [n][3],
 *    tangential history [n][MaxCnts], wall history [n][MaxNoWalls]; contact partner ids
 *    are the caller's particle indices.  Internally particles are re-ordered along a
 *    Morton curve; that order never shows through this interface.
 *  - One dem_ctx owns one CUDA stream; calls on it are stream-ordered, *_get and
 *    dem_ctx_sync synchronise.  A context is used by one host thread at a time.
 *  - dem_particles_set reads a pageable host array before it returns.  From page-locked
 *    (pinned) host memory the copy is queued on the context's stream instead, so that
 *    several uploads overlap: keep such an array unchanged until a call that synchronises
 *    (any *_get, dem_solver_run, dem_ctx_sync).
 */
#ifndef B200DEM_H
#define B200DEM_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status bits --------------------------------------------------------------- */
#define DEM_OK                    0
#define DEM_ERR_INVALID           0x001 /* bad argument                                  */
#define DEM_ERR_CUDA              0x002 /* CUDA runtime error                             */
#define DEM_ERR_CONTACT_OVERFLOW  0x004 /* more than MaxCnts contacts (ref: OOB write)    */
#define DEM_ERR_NEIGHBOR_OVERFLOW 0x008 /* neighbour list capacity exceeded (internal)    */
#define DEM_ERR_NAN               0x010 /* non-finite state detected                      */
#define DEM_ERR_TIMEOUT           0x020 /* bounded device wait gave up                    */
#define DEM_ERR_BOND_OVERFLOW     0x040 /* more than MaxBonds bonds                       */
#define DEM_ERR_NOMEM             0x080 /* device allocation failed                       */
#define DEM_ERR_UNSUPPORTED       0x100 /* option not supported                           */
#define DEM_ERR_MESH_OVERFLOW     0x200 /* more than 32 mesh triangles near one particle  */

/* ---- reference behaviours (bit set = reproduce the reference) ------------------ */
#define DEM_Q1_VELJ_USES_UI  0x01u /* src/CabanaDEM_Force.hpp:133-137                    */
#define DEM_Q2_ETA_T_ZERO    0x02u /* src/CabanaDEM_Force.hpp:224, :618.  Clear: eta_t > 0,
                                    * and the wall law applies its Coulomb-limited force (the
                                    * reference adds eta_t v_t back to it, :640-643, harmless
                                    * only with its eta_t = 0); the damping then only resets
                                    * the spring, as the reference's reset does.            */
#define DEM_Q3_NO_PP_TORQUE  0x04u /* src/CabanaDEM_Force.hpp:324-326                    */
#define DEM_Q4_UNIT_HISTORY  0x08u /* src/CabanaDEM_Force.hpp:310-319                    */
#define DEM_Q5_WALL_FT_TYPO  0x10u /* src/CabanaDEM_Force.hpp:624                        */
#define DEM_Q6_WALL_STATIC   0x20u /* src/CabanaDEM_Force.hpp:529: wall velocity ignored;
                                    * clear: walls move with their velocity (x += dt u each
                                    * step, with the particles' drift) and the wall contact uses
                                    * the relative velocity                                  */
#define DEM_REF_COMPAT       0x3Fu

/* ---- particle fields for dem_particles_set/get (Particles.hpp:99-271) ------------ */
enum dem_field {
    DEM_F_X = 0,        /* double [n][3]  slicePosition          */
    DEM_F_U,            /* double [n][3]  sliceVelocity          */
    DEM_F_OMEGA,        /* double [n][3]  sliceOmega             */
    DEM_F_FORCE,        /* double [n][3]  sliceForce             */
    DEM_F_TORQUE,       /* double [n][3]  sliceTorque            */
    DEM_F_M,            /* double [n]     sliceMass              */
    DEM_F_RHO,          /* double [n]     sliceDensity           */
    DEM_F_RAD,          /* double [n]     sliceRadius            */
    DEM_F_I,            /* double [n]     sliceMomentOfInertia   */
    DEM_F_E,            /* double [n]     sliceYoungsMod         */
    DEM_F_NU,           /* double [n]     slicePoissonsRatio     */
    DEM_F_G,            /* double [n]     sliceShearMod          */
    DEM_F_TNG_IDX,      /* int    [n][MaxCnts]    sliceTangentialDispIdx          */
    DEM_F_TNG_SS_X,     /* double [n][MaxCnts]    sliceTangentialDispSSx          */
    DEM_F_TNG_SS_Y,
    DEM_F_TNG_SS_Z,
    DEM_F_TNG_COUNT,    /* int    [n]             sliceTotalNoTangentialContacts  */
    DEM_F_TNG_SW_X,     /* double [n][MaxNoWalls] sliceTangentialDispSWx          */
    DEM_F_TNG_SW_Y,
    DEM_F_TNG_SW_Z,
    DEM_F_FIX,          /* uint8  [n]  DEM_FIX_* flags (boundary-condition hook)      */
    DEM_F_EXT_FORCE,    /* double [n][3] external force added before the pair forces  */
    DEM_F_SCENE,        /* int    [n]  scene index for batched independent scenes      */
    DEM_F_COUNT_
};
#define DEM_FIX_FORCE  0x1 /* zero F after the force pass (tst_01_BDEM:19-67)           */
#define DEM_FIX_TORQUE 0x2 /* zero torque after the force pass                          */

enum dem_wall_field { DEM_W_X = 0, DEM_W_U, DEM_W_OMEGA, DEM_W_NORMAL, DEM_W_E, DEM_W_NU, DEM_W_G };

enum dem_precision { DEM_FP64 = 0, DEM_MIXED = 1 };

typedef struct dem_ctx dem_ctx;
typedef struct dem_particles dem_particles;
typedef struct dem_walls dem_walls;
typedef struct dem_solver dem_solver;
typedef struct dem_bonds dem_bonds;

/* Force model, replaces Force(cor_pp, cor_pw, friction_pp, friction_pw)
 * (src/CabanaDEM_Force.hpp:23-35) plus the quirk selection. */
typedef struct dem_force_params {
    double cor_pp, cor_pw, mu_pp, mu_pw;
    unsigned quirks;
} dem_force_params;

/* Solver options, replaces SolverDEM's inputs (timestep) and the hard-coded neighbour
 * settings (delta, cell_ratio; src/CabanaDEM_Solver.hpp:43-63). */
typedef struct dem_solver_params {
    double dt;
    double delta;          /* > 0: uniform cutoff as the reference (3 r); 0: r_i + r_j + skin */
    double skin;           /* Verlet skin (used when delta == 0)                              */
    int rebuild_every_step;/* 1: rebuild before every force pass (Solver.hpp:87-88)           */
    int precision;         /* DEM_FP64 or DEM_MIXED                                           */
    double gravity[3];     /* body acceleration, added after the pair forces                 */
    int max_neighbors;     /* initial neighbour-list capacity per particle (0 = 32)          */
    int steps_per_launch;  /* fused steps per captured graph (0 = 32)                        */
    int stream_block;      /* streaming-kernel block size: 64, 128 or 256 (0 = 128)          */
    int contact_lanes;     /* 0 = automatic: while few particles are in contact, a streaming,
                            * a cooperative contact (8 lanes per particle, MaxCnts <= 32) and
                            * an apply kernel per step; while most are, one kernel over every
                            * particle.  1, 4 or 8: always the three-kernel step, its contact
                            * kernel with that many lanes per particle.  Same results.        */
    int stream_split;      /* streaming pass of the three-kernel step: 0 = automatic (4), 1 one
                            * kernel over every particle, 2 the particles without listed
                            * neighbours and the rest in two kernels, 3 the same two kernels as
                            * concurrent branches, 4 one persistent kernel whose tiles of
                            * particles are staged in shared memory by bulk asynchronous
                            * copies.  Same results.                                           */
    int dense_form;        /* step of a dense flow (most particles in contact, contact_lanes 0):
                            * 0 = automatic (2 above 65,536 particles, else 1), 1 one kernel
                            * with a thread per particle, 2 three kernels: contact search per
                            * particle, the pair law per contact, sums and integration per
                            * particle; 2 is also used at every density.  Same results.         */
    int scene_kernel;      /* batched scenes (dem_solver_set_scenes) of at most 64 particles each:
                            * 0 = automatic (a run is one persistent launch, a block per scene,
                            * every step inside it; with the Verlet-skin mode, static walls, no
                            * mesh, contact_lanes and dense_form 0), 1 = the per-step kernels.
                            * Same results.                                                    */
    int launch_overlap;    /* 0 = automatic (on), 1 on: each kernel of a step is launched as the
                            * programmatic dependent of the kernel before it, so that its launch
                            * overlaps that kernel's tail (it waits for that kernel's completion
                            * before it touches any state); 2 off: plain stream order.  Same
                            * results.                                                         */
    int cooperative_loop;  /* 0 = automatic (on), 1 on: while the step is one kernel over every
                            * particle (at most 65,536 particles, Verlet-skin mode, the graph
                            * while-loop, steps_per_launch 0), a run's steps between neighbour
                            * builds are one cooperative launch with a grid barrier between
                            * steps instead of a graph replay of per-step kernels; 2 off.  Same
                            * results.                                                         */
} dem_solver_params;

typedef struct dem_run_stats {
    long steps;            /* fused steps executed since creation          */
    long rebuilds;         /* neighbour builds since creation              */
    int max_neighbors;     /* largest list length at the last build        */
    int neighbor_capacity; /* current per-particle capacity                */
    int status;            /* sticky DEM_ERR_* bits seen on the device     */
    double disp_bound;     /* displacement bound since the last build (m)  */
    long launches;         /* kernels launched by this solver (graph nodes counted per replay) */
    double graph_ms;       /* device time of the step graphs replayed by dem_solver_run (CUDA
                            * events around each replay; host gaps and rebuilds excluded)  */
    long graph_steps;      /* fused steps those replays advanced                          */
    int launch_overlap;    /* 1: the step kernels are launched as programmatic dependents      */
    int cooperative_loop;  /* 1: the last run's steps ran in cooperative launches             */
} dem_run_stats;

/* ---- context ------------------------------------------------------------------- */
int dem_ctx_create(int device, dem_ctx **out);
int dem_ctx_destroy(dem_ctx *ctx);
int dem_ctx_sync(dem_ctx *ctx);
const char *dem_last_error(dem_ctx *ctx);
int dem_version(void);
/* The context's CUDA stream (cudaStream_t), so that callers can order their own work
 * after the library's and time it with CUDA events (no reference counterpart). */
void *dem_ctx_stream(dem_ctx *ctx);

/* ---- particles: Particles<Mem,3,MaxCnts,MaxNoWalls>(exec, n, out) ----------------
 * (src/CabanaDEM_Particles.hpp:22-71; template parameters become runtime capacities) */
int dem_particles_create(dem_ctx *ctx, int n, int max_contacts, int max_walls, dem_particles **out);
int dem_particles_destroy(dem_particles *p);
/* slice*() + updateParticles (src/CabanaDEM_Particles.hpp:91-271): SoA upload/download.
 * count = number of elements in `host` (e.g. 3*n for DEM_F_X).  A set from pinned host
 * memory is asynchronous (see Conventions). */
int dem_particles_set(dem_particles *p, int field, const void *host, long count);
int dem_particles_get(dem_particles *p, int field, void *host, long count);
/* As dem_particles_get into device memory `dev` (same layout and caller order), queued on
 * the context's stream without a host synchronisation. */
int dem_particles_get_device(dem_particles *p, int field, void *dev, long count);
/* Forget every contact: the tangential contact counts become 0, slot partners -1, slot and
 * wall history 0 -- the values the reference's examples give every particle in their set-up
 * functors (examples/01_elastic_normal_impact_of_two_identical_particles.cpp:125-130).
 * Device-side, no host copy: a caller starting a new run from fresh positions and
 * velocities sets those fields and calls this instead of uploading zero history arrays. */
int dem_particles_clear_contacts(dem_particles *p);
/* Force and torque zero, on the device, as newly created particles have them (the reference's
 * AoSoA is zero-initialised, src/CabanaDEM_Particles.hpp:22-71): with dem_particles_clear_contacts
 * the fresh start of a new run from uploaded positions and velocities. */
int dem_particles_clear_forces(dem_particles *p);
int dem_particles_size(dem_particles *p);

/* ---- walls: Wall<Mem,3>(exec, n, out) (src/CabanaDEM_Wall.hpp:22-153) ------------- */
int dem_walls_create(dem_ctx *ctx, int n, dem_walls **out);
int dem_walls_destroy(dem_walls *w);
int dem_walls_set(dem_walls *w, int field, const double *host, long count);

/* ---- solver: createSolverDEM<Mem>(inputs, particles, wall, force, delta) ----------
 * (src/CabanaDEM_Solver.hpp:129-138; ctor :32-64) */
int dem_solver_create(dem_ctx *ctx, dem_particles *p, dem_walls *w, const dem_force_params *fp,
                      const dem_solver_params *sp, dem_solver **out);
int dem_solver_destroy(dem_solver *s);
/* SolverDEM::run() body for nsteps steps (src/CabanaDEM_Solver.hpp:79-97): fused
 * force + integration kernels, graph-captured, neighbour rebuild when the
 * displacement bound exceeds skin/2 (or every step when rebuild_every_step). */
int dem_solver_run(dem_solver *s, int nsteps);
int dem_solver_stats(dem_solver *s, dem_run_stats *out);
/* Change the time step of later steps and phases: the dt an Integrator / BondedDEMIntegrator
 * is constructed with (src/CabanaDEM_Integrator.hpp:22-27,
 * src/CabanaBondedDEM_Integrator.hpp:22-27), for callers whose integrator and solver are
 * set up apart. */
int dem_solver_set_timestep(dem_solver *s, double dt);
/* Current wall positions [nw][3] (moving walls advance by dt * u each step when
 * DEM_Q6_WALL_STATIC is clear; no reference counterpart: the reference's walls never move,
 * src/CabanaDEM_Force.hpp:529). */
int dem_solver_wall_positions(dem_solver *s, double *host, long count);
/* Triangle-mesh wall (no reference counterpart: the reference has a Python intersection
 * prototype only, examples/python/particle_single_trangle_intersection_test.py).
 * tri [nt][3][3]: vertex coordinates (nt <= 4096, 0 removes the mesh); one material (E, nu,
 * G) with the plane walls' force parameters (cor_pw, mu_pw); velocity [3] or NULL: the mesh
 * translates by dt * velocity each step when DEM_Q6_WALL_STATIC is clear.  A contact acts as
 * a plane through the triangle's closest point (normal from that point to the particle
 * centre); an edge or vertex shared with a triangle already in contact, or lying on a
 * triangle the particle touches by its face, makes no second contact.  Each particle tracks
 * up to max_contacts (<= 16) triangle contacts (more: DEM_ERR_CONTACT_OVERFLOW, the extra
 * contacts act without history); candidates are the triangles within the list cutoff at
 * each neighbour build (more than 32: DEM_ERR_MESH_OVERFLOW).  Not with batched scenes or
 * bonds.  The contacts are summed after the plane walls, in triangle order. */
int dem_solver_set_mesh(dem_solver *s, const double *tri, int nt, double E, double nu, double G,
                        const double *velocity, int max_contacts);
/* The mesh's current translation [3] (zero for a static mesh). */
int dem_solver_mesh_translation(dem_solver *s, double *host3);
/* Same steps as dem_solver_run, but each fused step kernel is launched on its own between
 * two CUDA events; *kernel_ms receives the mean duration of one fused step launch
 * (rebuilds excluded).  For roofline measurement; no reference counterpart. */
int dem_solver_profile(dem_solver *s, int nsteps, double *kernel_ms);

/* Batched independent scenes (no reference counterpart).  Each particle belongs to the scene
 * given by DEM_F_SCENE; particles of different scenes never interact, whatever their
 * coordinates (the neighbour grid is built per scene).  Scene k uses params[k] for its
 * restitution and friction and owns walls [k*walls_per_scene, (k+1)*walls_per_scene) of the
 * solver's wall set; walls_per_scene <= MaxNoWalls.  All scenes advance in the same launches. */
typedef struct dem_scene_params {
    double cor_pp, cor_pw, mu_pp, mu_pw;
} dem_scene_params;
int dem_solver_set_scenes(dem_solver *s, const dem_scene_params *params, int nscenes, int walls_per_scene);

/* Reference-order phases, one launch each, for callers that drive the loop themselves:
 * Integrator::stage1/2/3 (src/CabanaDEM_Integrator.hpp:31-102), neighbors->build
 * (src/CabanaDEM_Solver.hpp:87-88) and computeForceParticleParticleInfiniteWall
 * (src/CabanaDEM_Force.hpp:700-710: zero, compact contacts, pp force, wall force). */
int dem_stage1(dem_solver *s);
int dem_stage2(dem_solver *s);
int dem_stage3(dem_solver *s);
int dem_build_neighbors(dem_solver *s);
/* The rebuild dem_solver_run performs when the displacement bound reaches skin/2, done now:
 * storage re-sorted along the Morton curve (contact partners remapped), list rebuilt,
 * displacement bound reset.  Results of later steps are unchanged bit for bit (sums run in
 * caller order); for callers that want a rebuild at a point of their choice, e.g. after
 * moving particles themselves.  No reference counterpart beyond neighbors->build
 * (src/CabanaDEM_Solver.hpp:87-88), which this extends with the re-sort. */
int dem_solver_rebuild(dem_solver *s);
int dem_compute_force(dem_solver *s);

/* Neighbour list of the last build in caller order, CSR: offsets[n+1], idx[total]
 * (ascending partner id).  Pass idx=NULL to get the total in *total. */
int dem_neighbors_get(dem_solver *s, int *offsets, int *idx, long *total);

/* ---- bonded DEM: ParticlesBondedDEM<Mem,Dim,MaxBonds> bond slots ---------------------
 * (src/CabanaBondedDEM_Particles.hpp:29-293) and computeBondedForce
 * (src/CabanaBondedDEM_Force.hpp:53-348).  Reference behaviours, bit set = reproduce: */
#define DEM_BQ10_INDEX_BY_J   0x01u /* history indexed by partner id (BondedDEM_Force.hpp:207, :231-322) */
#define DEM_BQ11_HARDCODED_K  0x02u /* stiffness from E, G, bond area (BondedDEM_Force.hpp:186-198)     */
#define DEM_BQ1_VELJ_USES_UI  0x04u /* vel_j y,z use u(i,.) (BondedDEM_Force.hpp:142-146)               */
#define DEM_BOND_REF_COMPAT   0x07u

typedef struct dem_bond_params {
    unsigned quirks;
    double beta;           /* sign-damping factor (reference: 0.1, BondedDEM_Force.hpp:186)   */
    double radius_factor;  /* bond radius = min(r_i, r_j) * factor (reference: 1, :187)        */
    double kn, kt;         /* explicit normal / shear stiffness, used when BQ11 is clear       */
    double break_strain;   /* > 0: a bond breaks once (rij - L0) / L0 exceeds it (no reference
                              counterpart)                                                    */
} dem_bond_params;

enum dem_bond_field {
    DEM_B_IDX = 0,     /* int    [n][MaxBonds] sliceBondIdx (caller indices, -1 empty) */
    DEM_B_INIT_LEN,    /* double [n][MaxBonds] sliceBondInitLen                       */
    DEM_B_COUNT,       /* int    [n]           sliceTotalNoBonds                      */
    DEM_B_FT_X, DEM_B_FT_Y, DEM_B_FT_Z,   /* double [n][MaxBonds] sliceBondFt*        */
    DEM_B_MN_X, DEM_B_MN_Y, DEM_B_MN_Z,   /* double [n][MaxBonds] sliceBondMn*        */
    DEM_B_MT_X, DEM_B_MT_Y, DEM_B_MT_Z,   /* double [n][MaxBonds] sliceBondMt*        */
    DEM_B_BROKEN       /* uint8  [n][MaxBonds] 1 once the bond has broken             */
};

/* Bond storage for the solver's particles (ParticlesBondedDEM ctor, :52-60). */
int dem_bonds_create(dem_solver *s, int max_bonds, const dem_bond_params *bp, dem_bonds **out);
int dem_bonds_destroy(dem_bonds *b);
/* setupBonds<Exec>() (src/CabanaBondedDEM_Particles.hpp:86-171): bond every j != i with
 * rij < factor * rad(i) among the candidates within search_cutoff, in ascending j; rest
 * length = rij.  The reference uses factor 3 and search cutoff 4 rad(0). */
int dem_bonds_setup(dem_bonds *b, double factor, double search_cutoff);
int dem_bonds_get(dem_bonds *b, int field, void *host, long count);
int dem_bonds_broken(dem_bonds *b, long *count);
/* nsteps of the bonded loop (tst_01_BDEM:295-306): stage1, stage2, force reset, external
 * force (DEM_F_EXT_FORCE), computeBondedForce, boundary hook (DEM_F_FIX), stage3 -- fused
 * into one kernel per step, graph-captured. */
int dem_bonded_run(dem_bonds *b, int nsteps);
/* Upload of a bond slice (the reference's slices are writable views,
 * src/CabanaBondedDEM_Particles.hpp:187-201): DEM_B_IDX in caller indices (-1 empty),
 * DEM_B_COUNT, DEM_B_INIT_LEN, the history fields and DEM_B_BROKEN, in the layout of
 * dem_bonds_get.  Bonds set this way fix the particle order as dem_bonds_setup does. */
int dem_bonds_set(dem_bonds *b, int field, const void *host, long count);

/* The bonded loop phase by phase, for callers that drive it themselves (the reference's
 * loop, tst_01_BDEM:295-306):
 *   stage1, stage2            BondedDEMIntegrator::stage1/2 (src/CabanaBondedDEM_Integrator.hpp:
 *                             31-74): dem_stage1 / dem_stage2 on the solver the bonds belong to
 *                             (the same arithmetic as Integrator::stage1/2)
 *   dem_bonded_reset          resetForcesAndTorques (src/CabanaBondedDEM_Force.hpp:16-50): F = tau = 0
 *   dem_apply_external_force  F += DEM_F_EXT_FORCE, in the position of the example's
 *                             applyTensileForce (tst_01_BDEM:70-117); no-op without it
 *   dem_bonded_force          computeBondedForce(particles, dt) (src/CabanaBondedDEM_Force.hpp:
 *                             53-348): F and tau += every bond's force and moment in slot order,
 *                             bond history updated, bonds past the breakage strain broken;
 *                             returns DEM_ERR_BOND_OVERFLOW as dem_bonded_run does
 *   dem_apply_boundary_conditions  gravity (m g), then the DEM_F_FIX flags zero F and/or tau, in
 *                             the position of the example's applyBoundaryConditions (tst_01_BDEM:19-67)
 *   stage3                    BondedDEMIntegrator::stage3 (:77-102): dem_stage3
 * The phases in this order give the fused dem_bonded_run's results bit for bit. */
int dem_bonded_reset(dem_bonds *b);
int dem_apply_external_force(dem_solver *s);
int dem_bonded_force(dem_bonds *b, double dt);
int dem_apply_boundary_conditions(dem_solver *s);

/* ---- neighbour list without allocation ---------------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device memory at the
 * point where they need a neighbour list: code whose device memory belongs to another
 * allocator (a framework's caching pool, a budget fixed up front), code in a time loop that
 * must not stall the GPU (cudaMalloc and cudaFree can synchronise the device), and code that
 * may not call an allocation API at all.  Builds the list dem_build_neighbors builds, for
 * particles held in the caller's device arrays, with its scratch taken from a fixed array
 * inside the library (about 2.4 MB on every GPU that loads it, held until the process exits).
 *   x[n][3], rad[n]               device inputs: positions and radii
 *   delta > 0: uniform cutoff; otherwise cutoff r_i + r_j + skin
 *   nn[n], idx[max_neighbors][n]  device outputs: list length, partner indices in ascending
 *                                 order, slot-major (partner k of particle i at idx[k*n + i])
 *   stream                        cudaStream_t (NULL: default stream); synchronised on return
 * Returns DEM_ERR_INVALID when n > DEM_NOALLOC_MAX_PARTICLES or max_neighbors >
 * DEM_NOALLOC_MAX_NEIGHBORS, DEM_ERR_NEIGHBOR_OVERFLOW when a particle has more than
 * max_neighbors partners (its list is cut at max_neighbors), and DEM_ERR_NAN when a position
 * or radius is not finite (every list is then empty).
 * All calls share the scratch array and it keeps the last call's contents: calls that could
 * overlap on the GPU race and must be ordered by the caller.  The first call on a device looks
 * up the array's address (with that device current) and keeps it for the life of the
 * process; make that call before any stream capture, and do not call this function again on
 * a device after a cudaDeviceReset of it (the kept address is then stale). */
#define DEM_NOALLOC_MAX_PARTICLES 32768
#define DEM_NOALLOC_MAX_NEIGHBORS 128
int dem_neighbor_list_noalloc(const double *x, const double *rad, int n, double delta, double skin,
                              int max_neighbors, int *nn, int *idx, void *stream);

/* Checkpoint of every particle field (caller order) to a file and back; the neighbour list
 * is rebuilt after a load, so a restarted run continues bit for bit.  The particles object
 * given to load must have the same n, MaxCnts and MaxNoWalls.  Load reads and checks the
 * whole file before it changes anything: on DEM_ERR_INVALID (unreadable, truncated or
 * mismatched file) the particles keep their previous state. */
int dem_checkpoint_save(dem_particles *p, const char *path);
int dem_checkpoint_load(dem_particles *p, const char *path);

/* Energy totals (no reference counterpart): out[0] translational kinetic, out[1]
 * rotational kinetic, out[2] Hertz elastic energy of pp contacts, out[3] of wall
 * contacts.  Fixed-order reduction, so repeated calls are bitwise identical. */
int dem_energy(dem_solver *s, double out[4]);

/* ---- Learned surrogate: dense layers on the tensor cores -----------------------------
 * A two-layer perceptron over rows, y = W2 relu(W1 x + b1) + b2 (+ residual), hidden width
 * 128, BF16 operands and FP32 accumulation (tcgen05 MMA, TMEM accumulators).  All pointers
 * are device pointers; rows are row-major.  Shapes (kin, nout): (16,128), (128,128),
 * (256,128), (384,128), (128,16).  Work is queued on the context's stream. */
typedef struct {
    const void *data;    /* bf16 [*][width] */
    const int *index;    /* row r of the input takes row index[r] of data (null: row r) */
    int width;           /* features taken from this source (multiple of 8) */
} dem_nn_rows;

typedef struct {
    int kin, nout;
    const void *w1t;     /* bf16 [128][kin]   W1 as out x in (forward) */
    const void *w1;      /* bf16 [kin][128]   W1 as in x out (backward) */
    const float *b1;     /* [128] */
    const void *w2t;     /* bf16 [nout][128] */
    const void *w2;      /* bf16 [128][nout] */
    const float *b2;     /* [nout] */
} dem_nn_mlp;

/* Input = the concatenation of up to 3 gathered sources (widths sum to kin).  Outputs that
 * are null are not written: out (bf16), out_f32, h1 (bf16 [rows][128] hidden activations,
 * needed by the backward pass). */
int dem_nn_mlp_forward(dem_ctx *ctx, const dem_nn_mlp *m, long rows, const dem_nn_rows *src, int nsrc,
                       const void *resid, void *out, float *out_f32, void *h1);
/* Backward of one forward call: dy (bf16 [rows][nout]) -> dz1 (bf16 [rows][128], written),
 * dx (fp32 [rows][kin], written; null skips it) and weight/bias gradients ADDED to g_w1t
 * [128][kin], g_b1 [128], g_w2t [nout][128], g_b2 [nout] (fixed-order sums: deterministic). */
int dem_nn_mlp_backward(dem_ctx *ctx, const dem_nn_mlp *m, long rows, const dem_nn_rows *src, int nsrc,
                        const void *dy, const void *h1, void *dz1, float *dx, float *g_w1t, float *g_b1,
                        float *g_w2t, float *g_b2);
/* The message (edge) layer in its factorised form: out = e + b2 + W2 relu(W1e e + b1 + P[recv]
 * + Q[send]) with PQ = [W1i h | W1j h] per node (bf16 [nodes][256]), e and out bf16
 * [rows][128], recv/send int [rows], w1e_t and w2t bf16 [128][128] (out x in), h1 (bf16
 * [rows][128], null: not written) the hidden activations.  form 0: the tile copies of e by the
 * tensor copy engine, one tile ahead, and the hidden tile in tensor memory (falls back to form
 * 1 when the driver cannot encode the tensor map); form 1: e staged by per-thread asynchronous
 * copies, the hidden tile in shared memory.  Same results.  Device pointers, the context's
 * stream (no reference counterpart). */
int dem_nn_edge_forward(dem_ctx *ctx, long rows, const void *e, const void *pq, const int *recv, const int *send,
                        const void *w1e_t, const float *b1, const void *w2t, const float *b2, void *out, void *h1,
                        int form);
/* Device error word of the context's tensor-core kernels (DEM_ERR_TIMEOUT when a bounded
 * wait gave up); synchronises, returns it in *status and clears it. */
int dem_nn_status(dem_ctx *ctx, int *status);
/* Bounds of the tensor-core kernels' waits, for testing that a wait which runs out is
 * reported and leaves the context usable (no reference counterpart).  poll_limit: polls of
 * the MMA-completion barrier per wait (0 = the default, about 4 million, seconds of waiting);
 * drop_mma != 0: the kernels issue no MMA and no commit, so every wait runs out with nothing
 * in flight (their outputs are then not written).  A block whose wait ran out waits once more,
 * with the same bound, for the MMA batch it was waiting on before it frees its tensor memory,
 * and sets DEM_ERR_TIMEOUT in the word dem_nn_status returns.  The setting is per device and
 * process-wide; it takes effect for kernels queued after the call. */
int dem_nn_debug_waits(dem_ctx *ctx, int poll_limit, int drop_mma);
/* Bounds of the staged streaming kernel's waits (stream_split 4), for testing that a wait which
 * runs out stops the run with DEM_ERR_TIMEOUT and leaves the context usable (no reference
 * counterpart).  poll_limit: polls of a tile's copy barrier per wait (0 = the default, about
 * 260,000); drop_copies != 0: the kernel arms its barriers but issues no copy, so every wait
 * runs out with nothing in flight.  A run then returns DEM_ERR_TIMEOUT with its step
 * unfinished (the particle state must be set again).  Calling with drop_copies = 0 also clears
 * the DEM_ERR_TIMEOUT bit of the solver's control word. */
int dem_solver_debug_stream_waits(dem_solver *s, int poll_limit, int drop_copies);

/* ---- Learned surrogate: message-passing network over the contact graph -------------------
 * Quasi-2D (x, y) particles.  One network stride replaces `steps_per_stride` DEM steps:
 * from the positions at the last two strides it predicts the change of the per-stride
 * displacement.  Graph: every pair closer than radius_graph (centre distance), per frame.
 * Network: node and edge encoders (16 -> 128 -> 128), three rounds of edge update
 * e += MLP[e, h_i, h_j] and node update h += MLP[h, sum_j e_ij], decoder 128 -> 128 -> 2;
 * dense layers as in dem_nn_mlp_*; aggregation in a fixed order (deterministic).
 * All position arrays are device pointers, double [n][3] in caller order (z ignored). */
typedef struct dem_surrogate dem_surrogate;

typedef struct {
    double radius_graph;     /* edge cutoff (m) */
    int steps_per_stride;    /* DEM steps per network stride (200) */
    double dt;               /* DEM time step (s); a stride lasts steps_per_stride * dt */
    double sigma_d;          /* scale of the per-stride displacement inputs (m) */
    double sigma_a;          /* scale of the predicted displacement change (m) */
    double r_mean, r_std;    /* radius normalisation */
    int nwalls;              /* planar walls (<= 4): feature distances and projection */
    double wall_x[4][3], wall_n[4][3];
    double wall_clip;        /* wall distance features saturate at this distance (m) */
    double gravity[3];       /* energy residual */
    double max_overlap;      /* fallback: any overlap above this fraction of the smaller radius */
    double energy_tol;       /* fallback: mechanical energy above its lowest value since the last
                              * DEM stride by more than energy_tol x total weight x r_mean, or
                              * the largest specific energy of one particle above its lowest
                              * value by more than the lift of one diameter (2 g r_mean) */
    int max_nodes;           /* capacity (particles per call, all frames together) */
    int max_frames;          /* capacity (independent frames per training batch) */
    int project_iters;       /* contact projection after a network stride: Jacobi sweeps (0: off) */
    double project_allow;    /* overlap left by the projection, fraction of the smaller radius */
} dem_surrogate_params;

typedef struct {
    long strides_network;    /* strides advanced by the network */
    long strides_dem;        /* strides advanced by DEM (fallback) */
    long fallback_overlap;   /* fallbacks caused by the overlap check */
    long fallback_energy;    /* fallbacks caused by the energy check */
    double max_overlap_seen; /* largest overlap fraction of an accepted network stride */
} dem_rollout_stats;

int dem_surrogate_create(dem_ctx *ctx, const dem_surrogate_params *prm, dem_surrogate **out);
int dem_surrogate_destroy(dem_surrogate *sg);
long dem_surrogate_num_params(dem_surrogate *sg);
/* FP32 master parameters, flat: for each layer (node enc, edge enc, 3 x (edge upd, node upd),
 * decoder) W1^T [128][kin], b1 [128], W2^T [nout][128], b2 [nout]. */
int dem_surrogate_get_params(dem_surrogate *sg, float *host, long n);
int dem_surrogate_set_params(dem_surrogate *sg, const float *host, long n);
int dem_surrogate_init_params(dem_surrogate *sg, unsigned long long seed);
/* Loss (mean squared error of the normalised displacement change) and its gradient for a
 * batch of frames: node i belongs to frame[i] (null: one frame); pos_prev, pos_cur,
 * pos_next: positions at strides k-1, k, k+1; Gaussian noise of std noise (m) is added to
 * the input positions (seeded).  grads_host (flat, like the parameters) may be null. */
int dem_surrogate_loss_grad(dem_surrogate *sg, int n, const double *pos_prev, const double *pos_cur,
                            const double *pos_next, const double *rad, const int *frame, int nframes,
                            double noise, unsigned long long seed, double *loss, float *grads_host);
/* loss_grad followed by one Adam step (lr, beta1 0.9, beta2 0.999, eps 1e-8). */
int dem_surrogate_train_step(dem_surrogate *sg, int n, const double *pos_prev, const double *pos_cur,
                             const double *pos_next, const double *rad, const int *frame, int nframes,
                             double noise, unsigned long long seed, double lr, double *loss);
/* One network stride: pos_next = pos_cur + (pos_cur - pos_prev) + sigma_a * net(...), then
 * projected out of the walls and, with project_iters > 0, out of overlaps larger than
 * project_allow (pairs of the graph, mass-weighted Jacobi sweeps). */
int dem_surrogate_predict(dem_surrogate *sg, int n, const double *pos_prev, const double *pos_cur,
                          const double *rad, const int *frame, int nframes, double *pos_next);
/* Hybrid rollout of a solver's particles (2D: z untouched) for nstrides strides: each stride
 * is a network stride unless its overlap or energy residual exceeds the thresholds, in
 * which case that stride is run by dem_solver_run from the state before it.  use_network = 0
 * runs every stride with DEM.  The solver's state is current on return. */
int dem_surrogate_rollout(dem_surrogate *sg, dem_solver *s, int nstrides, int use_network,
                          dem_rollout_stats *stats);

#ifdef __cplusplus
}
#endif
#endif
