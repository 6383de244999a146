// dem_internal.cuh -- device data layout and launcher declarations shared by the
// translation units of libb200dem.so.
//
// HBM layout (particles in Morton-sorted order, capacity `cap` = n):
//   pos[2]    double4 (x, y, z, r)      ping-pong (Ctl::cur); neighbour gathers read one 32 B sector
//   vel[2]    double  [3][cap]           SoA (ux | uy | uz); current buffer Ctl::vcur.  The
//   omg[2]    double  [3][cap]           contact step updates them in place (see dem_step.cu);
//                                        the bonded step and re-sorting use the second buffer
//   force, torque double [3][cap]        written by the last fused step / unfused force pass
//   mI        double2 (m, I)
//   mat       uint8 material id          (E, nu, G) deduplicated into pair tables
//   cstate    int: pp contact count (bits 0-7) | wall-history-active mask (bits 8-31)
//   tidx      int    [MaxCnts][cap]      partner (sorted index), slot-major
//   th        double [3][MaxCnts][cap]   tangential history x|y|z, slot-major
//   sw        double [3][MaxNoWalls][cap] wall tangential history
//   fix       uint8 flags, ext double [3][cap] (optional)
//   perm      sorted index -> caller index; rank: caller index -> sorted index
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "b200dem.h"

namespace b200dem {

constexpr int kMaxWalls = 24;
constexpr int kMaxMat = 32;

struct Ctl {
    int cur;                  // current position buffer
    int vcur;                 // current velocity / angular-velocity buffer
    int steps_done;           // fused steps executed in the current run
    int target;               // fused steps requested in the current run
    unsigned ticket;          // last-block election
    unsigned long long vmax2; // max |u|^2 of the drift in the running kernel (double bits)
    double disp;              // displacement bound since the last build
    double half_skin;         // stale threshold (list invalid once disp >= half_skin)
    int status;               // sticky DEM_ERR_* bits
    int max_nbr;              // longest neighbour list seen at the last build
    int ndefer;               // particles handed from the streaming to the contact kernel
    long long total_steps;
    long long rebuilds;
    int last_ndefer;          // deferred particles of the last completed fused step
    int nlone;                // particles [0, nlone) had no listed neighbour at the last build
                              // (placed first by the re-sort; 0 when the build did not re-sort)
    int nclear;               // particles [nlone, nlone + nclear): every listed neighbour's gap
                              // exceeded skin/2 at the last build (placed second)
    int npairs;               // contact work items of the current step (pair-parallel dense step)
    int loop_iter;            // iterations of the step loop in the current graph replay
    long long wfar_build;     // value of `rebuilds` when NbrList::wfar was last computed
    unsigned gen;             // step generation of the cooperative step loop (dem_persist.cuh)
};

struct Particles {
    int n, cap, mc, mw;
    double4 *pos[2];
    double *vel[2];
    double *omg[2];
    double *force, *torque;
    double *mI;    // [2][cap]: mass m (row 0) and moment of inertia I (row 1)
    uint8_t *mat;
    int *cstate;
    int *tidx;
    double *th;
    double *sw;
    uint8_t *fix;
    double *ext;   // may be null
    int *perm, *rank;
    unsigned long long *vslots;   // kVmaxSlots x 32 words: per-step max |u|^2, spread over L2 lines
    int *scene;                   // [cap] scene of each particle, null when all share scene 0
};

// (m, I) of particle i: two rows of one array, so that a kernel needing only m reads 8 bytes.
__host__ __device__ __forceinline__ double2 load_mI(const Particles &P, int i) {
    return make_double2(P.mI[i], P.mI[(long)P.cap + i]);
}

// Status bits that stop a run's steps (every gated kernel exits, the step loop ends): a list
// that overflowed (the host grows it and continues) and a bounded device wait that gave up (the
// run returns DEM_ERR_TIMEOUT).
constexpr int kStopBits = DEM_ERR_NEIGHBOR_OVERFLOW | DEM_ERR_TIMEOUT;
constexpr int kCoopSlots = 32;   // largest MaxCnts the cooperative contact kernel stages in shared memory
constexpr int kOneKernelMaxN = 65536;   // particle count up to which the step is always one kernel
constexpr int kVmaxSlots = 32;   // blocks fold their max into slot blockIdx % 32 (word 32 * slot)

struct PairConst {   // per (material a, material b) or (material a, wall w)
    double c_kn;     // 4./3. * E_eff            (Force.hpp:203, :568)
    double c_Sn;     // 2. * E_eff               (Force.hpp:211, :576)
    double c_kt;     // 8. * G_eff               (Force.hpp:222, :616)
    double pad;
};

struct WallGeom {
    double x[3];
    double n[3];
    double u[3];   // velocity (zero under DEM_Q6_WALL_STATIC): relative velocity of the contact
};

// Triangle-mesh wall on the device (one per solver).  Candidates: every triangle within the
// list cutoff of a particle at the last neighbour build, ascending id.
constexpr int kMeshCand = 32;      // candidate triangles per particle
constexpr int kMeshMaxTri = 4096;  // triangles per mesh (candidates are found by brute force)
constexpr int kMeshMaxContacts = 16;   // tracked triangle contacts per particle (upper bound)
struct MeshDev {
    int nt, mt;                    // triangles; tracked triangle contacts per particle
    const double *tri;             // [nt][9]: a, b, c at zero translation
    double *D;                     // [3] translation (advanced by the step finaliser when moving)
    double u[3];                   // velocity (zero for a static mesh)
    const struct PairConst *pm;    // [nmat] particle material against the mesh
    int *tid;                      // [mt][cap] triangle of each tracked contact
    double *th;                    // [3][mt][cap] tangential history
    unsigned char *cnt;            // [cap] tracked contacts
    int *cand;                     // [kMeshCand][cap]
    unsigned char *ncand;          // [cap]
};

struct ForceConsts {
    double K_n_pp, K_t_pp;     // eta = K * sqrt(S * m_eff)       (Force.hpp:215, :224)
    double K_n_pw, K_t_pw;     //                                  (Force.hpp:580, :618)
    double mu_pp, mu_pw;
    double dt, half_dt;
    double g[3];
    unsigned quirks;
    int nmat, nwall;
    int has_gravity;
    int has_ext;
    int has_fix;
    int mixed;                 // 1: FP32 contact forces (dem_mixed.cu)
    int wait_polls;            // polls per bounded wait of the staged streaming kernel (0: default)
    int drop_copies;           // testing only: the staged kernel arms its barriers but copies nothing
    int stream_block;          // k_stream block size: 64, 128 or 256
    int split;                 // streaming pass: 1 one kernel over every particle (k_stream);
                               // 2 the lone particles and the rest in two persistent kernels
                               // (k_stream_lone, k_stream_rest); 3 the same as concurrent branches;
                               // 4 one persistent kernel over bulk-staged tiles (k_stream_bulk)
    int dense;                 // 1: most particles are in contact -- contact kernels compiled for
                               // more resident blocks, wider apply grid (same arithmetic)
    int coop;                  // lanes per deferred particle in the contact kernel: 4 or 8
                               // (cooperative, MaxCnts <= kCoopSlots), 0: one thread each
    MeshDev mesh;              // triangle-mesh wall (nt == 0: none)
    int mesh_moving;           // the mesh translates each step (Q6 clear, nonzero velocity)
    struct WallGeom *mwalls;   // the device walls when some wall moves (Q6 clear, nonzero
                               // velocity): each step's finaliser advances x += dt u; else null
    int all;                   // 1: one kernel steps every particle (dense flows), no streaming
                               // or apply kernel; velocities ping-pong between their buffers;
                               // 2: the same step as three pair-parallel kernels (dem_pairs.cuh)
    const struct SceneConst *scenes;   // per-scene damping/friction, null: the scalars above
    int wps;                   // walls per scene (> 0 with scenes): scene s owns [s*wps, s*wps+wps)
    int pdl;                   // 1: the step kernels are launched with programmatic stream
                               // serialisation (launch_k), each the dependent of the one before
};

// ---- programmatic dependent launch ---------------------------------------------------
// A step kernel launched with programmatic stream serialisation may be scheduled while the
// kernel before it in the stream is still running, so that its launch overlaps that kernel's
// tail instead of following its completion.  Every kernel launched that way starts with
// grid_dep_wait(), which returns once the grids it depends on have completed and their memory
// operations are visible (at once for a kernel launched without the attribute), before it
// touches any device state; grid_dep_release() then lets the kernel after it be scheduled.
// A kernel whose blocks have all released (or exited) lets its dependent launch; that
// dependent's blocks wait in grid_dep_wait, so every grid waits only on grids whose blocks are
// all resident or done, and the chain always makes progress.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// One launch of `kernel` on stream s; with `overlap`, programmatic stream serialisation
// against the kernel before it (the kernel must begin with grid_dep_wait).
template <typename... KArgs, typename... Args>
inline cudaError_t launch_k(void (*kernel)(KArgs...), int grid, int block, size_t smem, cudaStream_t s, bool overlap,
                            Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = overlap ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// Per-scene force constants of batched independent scenes.
struct SceneConst {
    double K_n_pp, K_t_pp, K_n_pw, K_t_pw;
    double mu_pp, mu_pw;
};

struct NbrList {
    int *nn;     // [cap] list length
    int *idx;    // [maxnb][cap] sorted indices, ascending caller id
    int maxnb;
    int *nn_old, *idx_old;   // the lists of a re-sorting build in the old storage order ([cap],
                             // [maxnb][cap]), re-indexed into nn / idx after the permutation
    int *defer;  // [cap] particles deferred to the contact kernel in the current step
    double *defer_v, *defer_w;  // [3][cap] new u, omega of deferred particle t (slot t)
    // pair-parallel dense step (dem_pairs.cuh), allocated when that form is first used:
    int4 *pitem;     // [(maxnb + mw) * cap] contact work items: (i, j, history slot or -1, 0) or, for
                     // a wall, (i, -1 - wall, scene-local wall, wall history flag)
    double2 *pterm;  // [3][(maxnb + mw) * cap]: per item F (3) and tau (3) of particle i
    int4 *prec;      // [cap] first item, pair items, contact word at the step's start, wall items
    uint8_t *wfar;   // [cap] 1: at the last build every wall was farther than the stale threshold
                     // (valid while Ctl::wfar_build == Ctl::rebuilds and 2 disp < half_skin)
};

struct Grid {                 // one per scene, computed on the device at every build
    double lo[3];
    double cell, inv_cell;
    int dims[3];
    int bits;                 // Morton bits per axis (0: linear cell index)
    int ncodes;               // number of cell keys of this scene
    int base;                 // first key of this scene
    double rmax;
};

struct BuildBuffers {
    Grid *grid;               // device, [nscenes]
    int *total;               // device: total cell keys over all scenes
    int nscenes;              // scenes the grid array holds
    int *key;                 // [cap]
    int *cell_start;          // [cell_cap + 1]
    int *cell_fill;           // [cell_cap]
    int *cell_items;          // [cap] sorted-order index per cell slot
    int *block_sums;          // scan scratch
    int cell_cap;
    unsigned long long *bbox; // 8 ordered-int words per scene: lo[3], hi[3], rmax
    int *src, *dst;           // permutation at re-sort
    int *part_sums;           // [2][cap / kPartBlock + 2] per-block counts of the re-sort's partition
};

constexpr int kPartBlock = 256;   // block size of the re-sort's partition kernels

// Bond slots (bonded DEM), slot-major like the contact history.
constexpr unsigned BQ10_INDEX_BY_J = 0x01u;   // history(i, partner id), BondedDEM_Force.hpp:207, :231-322
constexpr unsigned BQ11_HARDCODED_K = 0x02u;  // k from E, G and bond area, BondedDEM_Force.hpp:186-198
constexpr unsigned BQ1_VELJ_USES_UI = 0x04u;  // BondedDEM_Force.hpp:142-146

struct Bonds {
    int mb, cap;
    int *idx;          // [mb][cap] partner (sorted index), -1 empty
    double *init_len;  // [mb][cap]
    int *count;        // [cap]
    double *hist;      // [9][mb][cap]: ft x|y|z, mn x|y|z, mt x|y|z (FP64 solvers)
    float *hist32;     // the same in FP32 (mixed-precision solvers; hist is then unused)
    uint8_t *broken;   // [mb][cap]
    double *E, *G;     // [cap] per-particle moduli (sorted order)
};

struct BondConsts {
    unsigned quirks;
    double beta, radius_factor, kn, kt, break_strain;
};

// ---- launchers (dem_bonded.cu) ----------------------------------------------------
void launch_bond_setup(const Particles &P, const NbrList &L, const Bonds &B, Ctl *ctl, double factor, cudaStream_t s);
void launch_bond_step(const Particles &P, const Bonds &B, Ctl *ctl, const ForceConsts &fc, const BondConsts &bc,
                      cudaStream_t s);
void launch_bond_broken_count(const Bonds &B, int n, unsigned long long *out, cudaStream_t s);
void launch_bond_force(const Particles &P, const Bonds &B, Ctl *ctl, const BondConsts &bc, double dt, cudaStream_t s);
void launch_add_ext_force(const Particles &P, cudaStream_t s);
void launch_post_hooks(const Particles &P, const ForceConsts &fc, cudaStream_t s);

// ---- launchers (dem_step.cu) ------------------------------------------------------
// MODE_FUSED launches the fused step (kernels_per_step(fc) kernels); MODE_FORCE_ONLY one
// force-only kernel.  MODE_FUSED_DIRECT is the per-particle body of the one-kernel dense step.
enum StepMode { MODE_FUSED = 0, MODE_FORCE_ONLY = 1, MODE_FUSED_DIRECT = 2 };
int kernels_per_step(const ForceConsts &fc);
void launch_mesh_candidates(const Particles &P, const MeshDev &M, Ctl *ctl, double delta, double skin, cudaStream_t s);
void launch_permute_mesh(const MeshDev &M, const MeshDev &A, int n, int cap, const int *items, cudaStream_t s);
void launch_prologue(const Particles &P, Ctl *ctl, const ForceConsts &fc, cudaStream_t s);
// Second stream and fork/join events for steps whose streaming pass runs as two concurrent
// graph branches (ForceConsts::split == 3); a null stream runs the branches in sequence.
struct AuxStream {
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};
// Wall-gap flags of every particle after a build (static walls, no mesh): NbrList::wfar.
void launch_wall_far(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc, const WallGeom *walls,
                     double half_skin, cudaStream_t s);
void launch_step(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc, const PairConst *pp,
                 const PairConst *pw, const WallGeom *walls, int mode, cudaStream_t s, const AuxStream &aux = AuxStream());
// the pair-parallel dense step in mixed precision (dem_mixed.cu)
void launch_pairs_mixed(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc, const PairConst *pp,
                        const PairConst *pw, const WallGeom *walls, bool mesh, cudaStream_t s);
void launch_stage(const Particles &P, Ctl *ctl, const ForceConsts &fc, int stage, cudaStream_t s);
// dem_mixed.cu
void launch_contact_mixed_all(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc,
                              const PairConst *pp, const PairConst *pw, const WallGeom *walls, int blocks, bool mesh,
                              cudaStream_t s);
const void *contact_mixed_all_kernel(bool mesh);
void launch_contact_mixed(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc, const PairConst *pp,
                          const PairConst *pw, const WallGeom *walls, bool mesh, int blocks, cudaStream_t s);
void launch_force_mixed(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc, const PairConst *pp,
                        const PairConst *pw, const WallGeom *walls, bool mesh, cudaStream_t s);
const void *contact_mixed_kernel(int dense, int coop, bool mesh);
void launch_energy(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc, const PairConst *pp,
                   const PairConst *pw, const WallGeom *walls, double *partials, int nparts, double *out,
                   cudaStream_t s);

// ---- launchers (dem_nbr.cu) -------------------------------------------------------
// Builds the neighbour list of the current order; with `resort` the particles are first
// re-ordered by Morton cell key (state permuted, contact partners remapped).
// classes = false: a re-sort keeps the plain cell order (scene-major for batched scenes), without
// the partition into particles with no listed neighbour, clear ones and the rest.
void launch_build(const Particles &P, Particles &alt, const NbrList &L, BuildBuffers &B, Ctl *ctl, double delta,
                  double skin, bool resort, bool check_run, cudaStream_t s, bool classes = true);
// Batched small scenes in one persistent launch per run (dem_scenes.cuh): the scene table of
// the current storage (false when some scene is not contiguous or exceeds the block), and the
// run's steps.
bool launch_scene_table(const Particles &P, int nscenes, int2 *table, int *counts, int *bad, cudaStream_t s);
void launch_scene_steps(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc, const PairConst *pp,
                        const PairConst *pw, const WallGeom *walls, const int2 *table, int nscenes, int nsteps,
                        double delta, double skin, cudaStream_t s);
void launch_scene_steps_mixed(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc,
                              const PairConst *pp, const PairConst *pw, const WallGeom *walls, const int2 *table,
                              int nscenes, int nsteps, double delta, double skin, cudaStream_t s);
constexpr int kSceneMaxParticles = 64;   // largest scene of the persistent form
// The one-kernel step's run in one cooperative launch (dem_persist.cuh): at most `max_steps`
// steps, ending at the target, a stale list or a stop bit.  An error when the launch is refused
// (e.g. the grid cannot be resident at once).
constexpr int kCoopMaxN = 65536;   // largest system the cooperative step loop takes
// scratch: kCoopScratch words of device memory for the symmetric barrier (static walls, no
// moving mesh).
constexpr int kCoopScratch = 1 + 4 * (kCoopMaxN / 128);
cudaError_t launch_steps_coop(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc, const PairConst *pp,
                              const PairConst *pw, const WallGeom *walls, int max_steps, unsigned long long *scratch,
                              cudaStream_t s);
cudaError_t launch_steps_coop_mixed(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc,
                                    const PairConst *pp, const PairConst *pw, const WallGeom *walls, int max_steps,
                                    unsigned long long *scratch, cudaStream_t s);

// dense layers of the surrogate (dem_nn.cu)
int nn_mlp_forward(const dem_nn_mlp &m, long rows, const dem_nn_rows *src, int nsrc, const void *resid, void *out,
                   float *out_f32, void *h1, int *err, cudaStream_t s);
int nn_mlp_backward(const dem_nn_mlp &m, long rows, const dem_nn_rows *src, int nsrc, const void *dy, const void *h1,
                    void *dz1, float *dx, float *g_w1t, int ld_w1, float *g_b1, float *g_w2t, float *g_b2,
                    float *part, int *err, cudaStream_t s);
long nn_wgrad_scratch(int kin, int nout);
int nn_debug_waits(int poll_limit, int drop_mma, cudaStream_t s);
// factorised edge layer of the surrogate (dem_nn.cu)
int nn_linear_pq(long rows, const void *h, const void *w1ij_t, void *pq, int *err, cudaStream_t s);
int nn_linear_pq_backward(long rows, const void *dpq, const void *w1ij, float *dh, int *err, cudaStream_t s);
int nn_linear_pq_wgrad(long rows, const void *dpq, const void *h, float *g_w1t, int ld, int col0, float *part,
                       int *err, cudaStream_t s);
int nn_edge_forward(long rows, const void *e, const void *pq, const int *recv, const int *send, const void *w1e_t,
                    const float *b1, const void *w2t, const float *b2, void *out, void *h1, int *err, cudaStream_t s,
                    int form = -1);
long nn_linear_wgrad_scratch();

// internal access to a solver's device state (dem_api.cu), used by the surrogate
struct SolverView {
    Particles P;
    Ctl *ctl;
    cudaStream_t stream;
    double dt;
    dem_ctx *ctx;
};
int solver_view(dem_solver *s, SolverView *v);
void solver_particles_changed(dem_solver *s);
cudaStream_t ctx_stream(dem_ctx *ctx);
int ctx_fail(dem_ctx *ctx, int code, const char *msg);
int ctx_cuda(dem_ctx *ctx, cudaError_t e, const char *what);
int ctx_nn_scratch(dem_ctx *ctx, long part_floats, int **err, float **part);

}  // namespace b200dem
