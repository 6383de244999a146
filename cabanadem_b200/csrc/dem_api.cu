// dem_api.cu -- the C ABI of libb200dem.so (declared in include/b200dem.h).
//
// Host side of the library: device allocation, caller-order <-> Morton-order staging,
// material/pair constant tables, and the solver loop.  The loop replaces
// SolverDEM::run (src/CabanaDEM_Solver.hpp:66-98): a prologue kernel does stage1+stage2
// of the first step, then chunks of fused step kernels run as one CUDA graph launch;
// the neighbour list is rebuilt on the device when the displacement bound since the
// last build reaches skin/2 (or before every step when rebuild_every_step is set).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <limits>
#include <thread>
#include <vector>

#include "b200dem.h"
#include "dem_internal.cuh"

using namespace b200dem;

struct dem_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    int *d_err = nullptr;           // error word of the tensor-core kernels
    float *nn_part = nullptr;       // per-CTA weight-gradient partials
    long nn_part_floats = 0;
};

struct dem_particles {
    dem_ctx *ctx = nullptr;
    Particles P{};
    Particles alt{};   // scratch for re-sorting
    Ctl *ctl = nullptr;
    std::vector<double> rho, E, nu, G;   // caller order, host copies
    double rmax = 0.0;
    bool dirty = true;       // state changed through set(): list must be rebuilt
    bool mat_dirty = true;   // E, nu, G changed: tables must be rebuilt
    bool has_bonds = false;  // bond slots hold sorted indices: no re-sort from now on
    bool any_fix = false;    // some particle carries a DEM_FIX_* flag
    int nscenes = 1;         // 1 + largest DEM_F_SCENE value
    int max_scene = 0;       // particles of the largest scene (DEM_F_SCENE set), else 0
    void *stage = nullptr;   // device staging buffer for set/get (largest field)
    size_t stage_bytes = 0;
    std::vector<uint8_t> mat;   // caller order
    std::vector<std::tuple<double, double, double>> mats;
};

struct dem_walls {
    dem_ctx *ctx = nullptr;
    int n = 0;
    std::vector<double> x, u, omega, normal, E, nu, G;
};

struct dem_solver {
    dem_ctx *ctx = nullptr;
    dem_particles *p = nullptr;
    dem_walls *w = nullptr;
    dem_force_params fp{};
    dem_solver_params sp{};
    ForceConsts fc{};
    PairConst *d_pp = nullptr, *d_pw = nullptr;
    WallGeom *d_walls = nullptr;
    std::vector<double> wall_pos;   // wall positions at the last preparation ([nw][3])
    bool walls_move = false;        // some wall has a velocity and Q6 is clear
    // triangle-mesh wall (dem_solver_set_mesh): host copy of its definition, device arrays
    int mesh_nt = 0;
    double mesh_mat[3] = {0., 0., 0.};   // E, nu, G
    double mesh_u[3] = {0., 0., 0.};
    MeshDev mesh{};                 // device arrays (tri, D, tid, th, cnt, cand, ncand); pm set by prepare
    MeshDev mesh_alt{};             // tid, th, cnt of the re-sort
    PairConst *d_mesh_pm = nullptr;
    SceneConst *d_scenes = nullptr;
    int nscenes = 0, wps = 0;
    bool walls_ok = true;
    NbrList L{};
    BuildBuffers B{};
    double *d_epart = nullptr, *d_eout = nullptr;
    int nparts = 0;
    bool built = false;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    long graph_version = -1;
    long version = 0;   // bumps when anything baked into the graph changes
    long launches = 0;  // kernels launched (graph nodes counted per replay)
    long graph_nodes = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;   // around each step-graph replay
    AuxStream aux;                              // second branch of the split streaming pass
    bool loop = false;                          // steps in a graph while-loop (steps_per_launch 0)
    double graph_ms = 0.0;                      // device time of the replays
    long graph_steps_run = 0;                   // steps those replays advanced
    int graph_done_mark = 0;                    // steps_done before the current replay
    // batched small scenes in one persistent launch per run (scene_kernel 0)
    int2 *d_scene_table = nullptr;              // [nscenes] first storage index, count
    int *d_scene_counts = nullptr, *d_scene_bad = nullptr;
    int scene_table_n = 0;                      // scenes the table holds
    bool scenes_ready = false;                  // the table matches the storage order
    bool scenes_unfit = false;                  // a scene was found not contiguous: per-step form
    bool no_overlap = false;                    // a step graph with dependent launches failed to build
    bool coop_refused = false;                  // a cooperative launch of the step loop was refused
    bool coop_ran = false;                      // the last run's steps ran in cooperative launches
    unsigned long long *d_coop = nullptr;       // kCoopScratch words: barrier counter and slots
};

struct dem_bonds {
    dem_solver *s = nullptr;
    Bonds B{};
    BondConsts bc{};
    unsigned long long *d_count = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    long graph_version = -1;
    bool set_up = false;
};

namespace {

int fail(dem_ctx *ctx, int code, const std::string &msg) {
    if (ctx) ctx->err = msg;
    return code;
}

int cuda_check(dem_ctx *ctx, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return DEM_OK;
    return fail(ctx, e == cudaErrorMemoryAllocation ? DEM_ERR_NOMEM : DEM_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                                  \
    do {                                                          \
        int _st = cuda_check(ctx, (call), #call);                 \
        if (_st) return _st;                                      \
    } while (0)

template <class T>
cudaError_t dalloc(T **p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    return cudaMalloc((void **)p, count * sizeof(T));
}

// Runs f(begin, end) over [0, n) split across the host's cores (at most 32 threads, at least
// 256k elements each); smaller ranges run on the calling thread.  For the host-side passes over
// per-particle arrays that sit between the copies of a set/run/get cycle.
template <typename F>
void host_parallel(long n, F f) {
    const long kMinChunk = 1L << 18;
    long nt = std::min<long>(std::max(1u, std::thread::hardware_concurrency()), 32);
    nt = std::min(nt, (n + kMinChunk - 1) / kMinChunk);
    if (nt <= 1) {
        f(0L, n, 0);
        return;
    }
    const long chunk = (n + nt - 1) / nt;
    std::vector<std::thread> th;
    for (long t = 1; t < nt; ++t) th.emplace_back(f, std::min(n, t * chunk), std::min(n, (t + 1) * chunk), (int)t);
    f(0L, std::min(n, chunk), 0);
    for (auto &x : th) x.join();
}
int host_threads(long n) {
    const long kMinChunk = 1L << 18;
    long nt = std::min<long>(std::max(1u, std::thread::hardware_concurrency()), 32);
    return (int)std::max(1L, std::min(nt, (n + kMinChunk - 1) / kMinChunk));
}

// ---- staging kernels (caller order <-> sorted order) --------------------------------
__global__ void k_scatter_d(const double *src, double *dst, int n, int ncomp, int cap, const int *rank) {
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < (long)n * ncomp; t += (long)gridDim.x * blockDim.x) {
        const int c = (int)(t / ncomp), k = (int)(t % ncomp);
        dst[(long)k * cap + rank[c]] = src[t];
    }
}
__global__ void k_gather_f2d(const float *src, double *dst, int n, int ncomp, int cap, const int *rank) {
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < (long)n * ncomp; t += (long)gridDim.x * blockDim.x) {
        const int c = (int)(t / ncomp), k = (int)(t % ncomp);
        dst[t] = (double)src[(long)k * cap + rank[c]];
    }
}

__global__ void k_gather_d(const double *src, double *dst, int n, int ncomp, int cap, const int *rank) {
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < (long)n * ncomp; t += (long)gridDim.x * blockDim.x) {
        const int c = (int)(t / ncomp), k = (int)(t % ncomp);
        dst[t] = src[(long)k * cap + rank[c]];
    }
}
// mode 0: partner ids (caller -> sorted via rank), 1: plain
__global__ void k_scatter_i(const int *src, int *dst, int n, int ncomp, int cap, const int *rank, int remap) {
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < (long)n * ncomp; t += (long)gridDim.x * blockDim.x) {
        const int c = (int)(t / ncomp), k = (int)(t % ncomp);
        int v = src[t];
        if (remap && v >= 0 && v < n) v = rank[v];
        dst[(long)k * cap + rank[c]] = v;
    }
}
__global__ void k_gather_i(const int *src, int *dst, int n, int ncomp, int cap, const int *rank, const int *perm,
                           int remap) {
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < (long)n * ncomp; t += (long)gridDim.x * blockDim.x) {
        const int c = (int)(t / ncomp), k = (int)(t % ncomp);
        int v = src[(long)k * cap + rank[c]];
        if (remap && v >= 0 && v < n) v = perm[v];
        dst[t] = v;
    }
}
// Ping-pong buffers picked on the device from the control word (`sel` = &ctl->cur or
// &ctl->vcur), so that a set or get queues behind the steps without a host round trip.
__global__ void k_scatter_pos_sel(const double *src, double4 *pos0, double4 *pos1, const int *sel, int n,
                                  const int *rank, int rad) {
    double4 *pos = *sel ? pos1 : pos0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        double4 &p = pos[rank[c]];
        if (rad) p.w = src[c];
        else {
            p.x = src[3 * c];
            p.y = src[3 * c + 1];
            p.z = src[3 * c + 2];
        }
    }
}
__global__ void k_gather_pos_sel(const double4 *pos0, const double4 *pos1, const int *sel, double *dst, int n,
                                 const int *rank, int rad) {
    const double4 *pos = *sel ? pos1 : pos0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const double4 p = pos[rank[c]];
        if (rad) dst[c] = p.w;
        else {
            dst[3 * c] = p.x;
            dst[3 * c + 1] = p.y;
            dst[3 * c + 2] = p.z;
        }
    }
}
__global__ void k_scatter_d_sel(const double *src, double *d0, double *d1, const int *sel, int n, int ncomp, int cap,
                                const int *rank) {
    double *dst = *sel ? d1 : d0;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < (long)n * ncomp; t += (long)gridDim.x * blockDim.x) {
        const int c = (int)(t / ncomp), k = (int)(t % ncomp);
        dst[(long)k * cap + rank[c]] = src[t];
    }
}
__global__ void k_gather_d_sel(const double *s0, const double *s1, const int *sel, double *dst, int n, int ncomp,
                               int cap, const int *rank) {
    const double *src = *sel ? s1 : s0;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < (long)n * ncomp; t += (long)gridDim.x * blockDim.x) {
        const int c = (int)(t / ncomp), k = (int)(t % ncomp);
        dst[t] = src[(long)k * cap + rank[c]];
    }
}
__global__ void k_scatter_mI(const double *src, double *mI, int n, int cap, const int *rank, int which) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
        mI[(long)which * cap + rank[c]] = src[c];
}
__global__ void k_gather_mI(const double *mI, double *dst, int n, int cap, const int *rank, int which) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
        dst[c] = mI[(long)which * cap + rank[c]];
}
__global__ void k_scatter_u8(const uint8_t *src, uint8_t *dst, int n, const int *rank) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) dst[rank[c]] = src[c];
}
__global__ void k_gather_u8(const uint8_t *src, uint8_t *dst, int n, const int *rank) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) dst[c] = src[rank[c]];
}
__global__ void k_gather_u8n(const uint8_t *src, uint8_t *dst, int n, int ncomp, int cap, const int *rank) {
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < (long)n * ncomp; t += (long)gridDim.x * blockDim.x) {
        const int c = (int)(t / ncomp), k = (int)(t % ncomp);
        dst[t] = src[(long)k * cap + rank[c]];
    }
}
__global__ void k_scatter_u8n(const uint8_t *src, uint8_t *dst, int n, int ncomp, int cap, const int *rank) {
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < (long)n * ncomp; t += (long)gridDim.x * blockDim.x) {
        const int c = (int)(t / ncomp), k = (int)(t % ncomp);
        dst[(long)k * cap + rank[c]] = src[t];
    }
}
__global__ void k_scatter_d2f(const double *src, float *dst, int n, int ncomp, int cap, const int *rank) {
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < (long)n * ncomp; t += (long)gridDim.x * blockDim.x) {
        const int c = (int)(t / ncomp), k = (int)(t % ncomp);
        dst[(long)k * cap + rank[c]] = (float)src[t];
    }
}
__global__ void k_fill_i(int *a, long count, int v) {
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < count; t += (long)gridDim.x * blockDim.x) a[t] = v;
}
__global__ void k_scatter_count(const int *src, int *cstate, int n, const int *rank) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const int p = rank[c];
        cstate[p] = (cstate[p] & ~0xff) | (src[c] & 0xff);
    }
}
__global__ void k_gather_count(const int *cstate, int *dst, int n, const int *rank) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) dst[c] = cstate[rank[c]] & 0xff;
}
// wall-history-active bits = any stored component nonzero
__global__ void k_sw_mask(Particles P) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += gridDim.x * blockDim.x) {
        unsigned m = 0;
        for (int w = 0; w < P.mw; ++w)
            for (int d = 0; d < 3; ++d)
                if (P.sw[((long)d * P.mw + w) * P.cap + i] != 0.0) m |= 1u << w;
        P.cstate[i] = (P.cstate[i] & 0xff) | (int)(m << 8);
    }
}
__global__ void k_init_particles(Particles P) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += gridDim.x * blockDim.x) {
        P.perm[i] = i;
        P.rank[i] = i;
        for (int k = 0; k < P.mc; ++k) P.tidx[(long)k * P.cap + i] = -1;
    }
}
// `fresh_list`: every step builds its list first (the rebuild-every-step mode), so a list
// invalidated by a change of the particles is not stale for the run's first step.
__global__ void k_run_begin(Ctl *ctl, int target, double half_skin, int fresh_list = 0) {
    if (threadIdx.x == 0) {
        if (fresh_list) ctl->disp = 0.0;
        ctl->ndefer = 0;   // a run starts at a step boundary (a step stopped by an error left its list)
        ctl->steps_done = 0;
        ctl->target = target;
        ctl->half_skin = half_skin;
        ctl->ticket = 0u;
        ctl->vmax2 = 0ull;
        ctl->npairs = 0;
    }
}
// Step loop of a graph replay: conditional while nodes of 8, 4, 2 and 1 steps per iteration,
// each running while at least that many steps remain, so that no step of a replay past the
// target is launched (a gated streaming kernel still costs its block launches) and a run's
// tail takes at most one iteration of each short loop (an iteration's conditional turn-around
// costs about 5 us).  A loop continues while steps remain, the list is still valid, no list
// overflowed, no bounded wait gave up and the density regime the kernels were chosen for still
// holds.  Each loop's condition is set before it by a node of the replay (k_loop_begin,
// k_loop_mid) and after every iteration by one thread of its body (k_loop_ctl); an iteration
// counter bounds every loop by target + 1 iterations, so a replay ends even if some step made
// no progress.
// `dense` < 0: the kernel forms do not depend on the density (no density exit).
__device__ __forceinline__ bool loop_go(const Ctl *ctl, int n, int dense, int min_left) {
    bool go = ctl->steps_done + min_left <= ctl->target && ctl->disp < ctl->half_skin &&
              !(ctl->status & kStopBits) && ctl->loop_iter <= ctl->target;
    if (go && n > 0 && dense >= 0) {   // the thresholds of adapt_density: leave the loop to switch kernel forms
        const double f = (double)ctl->last_ndefer / n;
        go = dense ? f >= 0.10 : !(f > 0.30);
    }
    return go;
}
__global__ void k_loop_begin(Ctl *ctl, cudaGraphConditionalHandle h, int n, int dense, int min_left) {
    if (threadIdx.x != 0) return;
    ctl->loop_iter = 0;
    // the first step of a run is always taken (the density of the step before the run does
    // not decide the form of the run's first steps)
    const bool go = ctl->steps_done + min_left <= ctl->target && ctl->disp < ctl->half_skin &&
                    !(ctl->status & kStopBits);
    cudaGraphSetConditional(h, go ? 1u : 0u);
}
__global__ void k_loop_mid(Ctl *ctl, cudaGraphConditionalHandle h, int n, int dense, int min_left) {
    if (threadIdx.x != 0) return;
    // no iteration of an earlier loop (fewer steps left than they take): the replay's first
    // step is taken here, whatever the density (as in k_loop_begin)
    cudaGraphSetConditional(h, loop_go(ctl, n, ctl->loop_iter == 0 ? -1 : dense, min_left) ? 1u : 0u);
}
__global__ void k_loop_ctl(Ctl *ctl, cudaGraphConditionalHandle h, int n, int dense, int min_left) {
    grid_dep_wait();   // launched as a dependent (launch_k): the kernel before has completed
    grid_dep_release();
    if (threadIdx.x != 0) return;
    ++ctl->loop_iter;
    cudaGraphSetConditional(h, loop_go(ctl, n, dense, min_left) ? 1u : 0u);
}
__global__ void k_invalidate(Ctl *ctl) {
    if (threadIdx.x == 0) ctl->disp = 1e300;
}

constexpr int kGS = 148 * 4;
constexpr int kTB = 256;

bool field_layout(const dem_particles *p, int field, long *count, int *esize) {
    const long n = p->P.n;
    switch (field) {
        case DEM_F_X: case DEM_F_U: case DEM_F_OMEGA: case DEM_F_FORCE: case DEM_F_TORQUE: case DEM_F_EXT_FORCE:
            *count = 3 * n; *esize = 8; return true;
        case DEM_F_M: case DEM_F_RHO: case DEM_F_RAD: case DEM_F_I: case DEM_F_E: case DEM_F_NU: case DEM_F_G:
            *count = n; *esize = 8; return true;
        case DEM_F_TNG_IDX: *count = n * p->P.mc; *esize = 4; return true;
        case DEM_F_TNG_SS_X: case DEM_F_TNG_SS_Y: case DEM_F_TNG_SS_Z: *count = n * p->P.mc; *esize = 8; return true;
        case DEM_F_TNG_COUNT: *count = n; *esize = 4; return true;
        case DEM_F_TNG_SW_X: case DEM_F_TNG_SW_Y: case DEM_F_TNG_SW_Z: *count = n * p->P.mw; *esize = 8; return true;
        case DEM_F_FIX: *count = n; *esize = 1; return true;
        case DEM_F_SCENE: *count = n; *esize = 4; return true;
        default: return false;
    }
}


}  // namespace

// =====================================================================================
extern "C" int dem_version(void) { return 1; }

extern "C" int dem_ctx_create(int device, dem_ctx **out) {
    if (!out) return DEM_ERR_INVALID;
    *out = nullptr;
    dem_ctx *ctx = new dem_ctx();
    ctx->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete ctx;
        return DEM_ERR_CUDA;
    }
    *out = ctx;
    return DEM_OK;
}

extern "C" int dem_ctx_destroy(dem_ctx *ctx) {
    if (!ctx) return DEM_ERR_INVALID;
    cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->d_err);
    cudaFree(ctx->nn_part);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return DEM_OK;
}

extern "C" int dem_ctx_sync(dem_ctx *ctx) {
    if (!ctx) return DEM_ERR_INVALID;
    CK(cudaStreamSynchronize(ctx->stream));
    return DEM_OK;
}

extern "C" const char *dem_last_error(dem_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

extern "C" void *dem_ctx_stream(dem_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

// ---- particles ----------------------------------------------------------------------
static cudaError_t alloc_particles(Particles &P, int n, int mc, int mw, bool pingpong) {
    cudaError_t e = cudaSuccess;
    auto A = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
    P.n = n;
    P.cap = (n + 63) / 64 * 64;   // component rows of the SoA arrays start 512-byte aligned
    P.mc = mc;
    P.mw = mw;
    const size_t cap = P.cap;
    for (int b = 0; b < (pingpong ? 2 : 1); ++b) {
        A(dalloc(&P.pos[b], cap));
        A(dalloc(&P.vel[b], 3 * cap));
        A(dalloc(&P.omg[b], 3 * cap));
    }
    A(dalloc(&P.force, 3 * cap));
    A(dalloc(&P.torque, 3 * cap));
    A(dalloc(&P.mI, 2 * (size_t)cap));
    A(dalloc(&P.mat, cap));
    A(dalloc(&P.cstate, cap));
    A(dalloc(&P.tidx, (size_t)std::max(mc, 1) * cap));
    A(dalloc(&P.th, 3 * (size_t)std::max(mc, 1) * cap));
    A(dalloc(&P.sw, 3 * (size_t)std::max(mw, 1) * cap));
    A(dalloc(&P.fix, cap));
    A(dalloc(&P.perm, cap));
    A(dalloc(&P.rank, cap));
    A(dalloc(&P.vslots, 32 * kVmaxSlots));
    P.scene = nullptr;
    if (e == cudaSuccess) e = cudaMemset(P.vslots, 0, sizeof(unsigned long long) * 32 * kVmaxSlots);
    P.ext = nullptr;
    return e;
}

static void free_particles(Particles &P) {
    for (int b = 0; b < 2; ++b) {
        cudaFree(P.pos[b]);
        cudaFree(P.vel[b]);
        cudaFree(P.omg[b]);
    }
    cudaFree(P.force); cudaFree(P.torque); cudaFree(P.mI); cudaFree(P.mat); cudaFree(P.cstate);
    cudaFree(P.tidx); cudaFree(P.th); cudaFree(P.sw); cudaFree(P.fix); cudaFree(P.perm); cudaFree(P.rank);
    cudaFree(P.vslots);
    cudaFree(P.scene);
    cudaFree(P.ext);
    P = Particles{};
}

extern "C" int dem_particles_create(dem_ctx *ctx, int n, int max_contacts, int max_walls, dem_particles **out) {
    if (!ctx || !out || n <= 0 || max_contacts < 0 || max_contacts > 255 || max_walls < 0 || max_walls > kMaxWalls)
        return fail(ctx, DEM_ERR_INVALID, "dem_particles_create: n > 0, 0 <= max_contacts <= 255, max_walls <= 24");
    *out = nullptr;
    dem_particles *p = new dem_particles();
    p->ctx = ctx;
    cudaError_t e = alloc_particles(p->P, n, max_contacts, max_walls, true);
    if (e == cudaSuccess) e = alloc_particles(p->alt, n, max_contacts, max_walls, false);
    if (e == cudaSuccess) e = dalloc(&p->ctl, 1);
    if (e == cudaSuccess) {
        p->stage_bytes = sizeof(double) * (size_t)p->P.cap * std::max(3, std::max(max_contacts, max_walls));
        e = cudaMalloc(&p->stage, p->stage_bytes);
    }
    if (e != cudaSuccess) {
        free_particles(p->P);
        free_particles(p->alt);
        cudaFree(p->ctl);
        cudaFree(p->stage);
        delete p;
        return cuda_check(ctx, e, "dem_particles_create");
    }
    cudaStream_t s = ctx->stream;
    const Particles &P = p->P;
    const size_t cn = (size_t)P.cap;
    for (int b = 0; b < 2; ++b) {
        cudaMemsetAsync(P.pos[b], 0, sizeof(double4) * cn, s);
        cudaMemsetAsync(P.vel[b], 0, sizeof(double) * 3 * cn, s);
        cudaMemsetAsync(P.omg[b], 0, sizeof(double) * 3 * cn, s);
    }
    cudaMemsetAsync(P.force, 0, sizeof(double) * 3 * cn, s);
    cudaMemsetAsync(P.torque, 0, sizeof(double) * 3 * cn, s);
    cudaMemsetAsync(P.mI, 0, sizeof(double) * 2 * cn, s);
    cudaMemsetAsync(P.mat, 0, cn, s);
    cudaMemsetAsync(P.cstate, 0, sizeof(int) * cn, s);
    cudaMemsetAsync(P.th, 0, sizeof(double) * 3 * std::max(max_contacts, 1) * cn, s);
    cudaMemsetAsync(P.sw, 0, sizeof(double) * 3 * std::max(max_walls, 1) * cn, s);
    cudaMemsetAsync(P.fix, 0, cn, s);
    cudaMemsetAsync(p->ctl, 0, sizeof(Ctl), s);
    k_init_particles<<<kGS, kTB, 0, s>>>(p->P);
    p->rho.assign(n, 0.0);
    p->E.assign(n, 0.0);
    p->nu.assign(n, 0.0);
    p->G.assign(n, 0.0);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    *out = p;
    return DEM_OK;
}

extern "C" int dem_particles_destroy(dem_particles *p) {
    if (!p) return DEM_ERR_INVALID;
    cudaStreamSynchronize(p->ctx->stream);
    free_particles(p->P);
    free_particles(p->alt);
    cudaFree(p->ctl);
    cudaFree(p->stage);
    delete p;
    return DEM_OK;
}

extern "C" int dem_particles_size(dem_particles *p) { return p ? p->P.n : -1; }

extern "C" int dem_particles_set(dem_particles *p, int field, const void *host, long count) {
    if (!p || !host) return DEM_ERR_INVALID;
    dem_ctx *ctx = p->ctx;
    long need;
    int es;
    if (!field_layout(p, field, &need, &es) || count != need)
        return fail(ctx, DEM_ERR_INVALID, "dem_particles_set: unknown field or wrong element count");
    const int n = p->P.n;
    cudaStream_t s = ctx->stream;
    Particles &P = p->P;
    if (field == DEM_F_RHO || field == DEM_F_E || field == DEM_F_NU || field == DEM_F_G) {
        // host copies; the material table is re-derived only when E, nu or G changed
        std::vector<double> &dst = field == DEM_F_RHO ? p->rho : field == DEM_F_E ? p->E : field == DEM_F_NU ? p->nu : p->G;
        const double *src = (const double *)host;
        std::vector<char> changed(host_threads(n), 0);
        host_parallel(n, [&](long b, long e, int t) {
            if (e > b && std::memcmp(dst.data() + b, src + b, sizeof(double) * (e - b)) != 0) {
                std::memcpy(dst.data() + b, src + b, sizeof(double) * (e - b));
                changed[t] = 1;
            }
        });
        if (field != DEM_F_RHO && std::find(changed.begin(), changed.end(), 1) != changed.end()) p->mat_dirty = true;
        return DEM_OK;
    }
    void *tmp = p->stage;
    CK(cudaMemcpyAsync(tmp, host, (size_t)need * es, cudaMemcpyHostToDevice, s));
    const int *cur = &p->ctl->cur, *vcur = &p->ctl->vcur;
    switch (field) {
        case DEM_F_X: k_scatter_pos_sel<<<kGS, kTB, 0, s>>>((double *)tmp, P.pos[0], P.pos[1], cur, n, P.rank, 0); break;
        case DEM_F_RAD: {
            k_scatter_pos_sel<<<kGS, kTB, 0, s>>>((double *)tmp, P.pos[0], P.pos[1], cur, n, P.rank, 1);
            const double *r = (const double *)host;
            std::vector<double> part(host_threads(n), 0.0);
            host_parallel(n, [&](long b, long e, int t) {
                double m = 0.0;
                for (long i = b; i < e; ++i) m = std::max(m, r[i]);
                part[t] = m;
            });
            p->rmax = *std::max_element(part.begin(), part.end());
            break;
        }
        case DEM_F_U:
            k_scatter_d_sel<<<kGS, kTB, 0, s>>>((double *)tmp, P.vel[0], P.vel[1], vcur, n, 3, P.cap, P.rank);
            break;
        case DEM_F_OMEGA:
            k_scatter_d_sel<<<kGS, kTB, 0, s>>>((double *)tmp, P.omg[0], P.omg[1], vcur, n, 3, P.cap, P.rank);
            break;
        case DEM_F_FORCE: k_scatter_d<<<kGS, kTB, 0, s>>>((double *)tmp, P.force, n, 3, P.cap, P.rank); break;
        case DEM_F_TORQUE: k_scatter_d<<<kGS, kTB, 0, s>>>((double *)tmp, P.torque, n, 3, P.cap, P.rank); break;
        case DEM_F_EXT_FORCE:
            if (!P.ext) {
                CK(dalloc(&P.ext, 3 * (size_t)P.cap));
                CK(dalloc(&p->alt.ext, 3 * (size_t)P.cap));
            }
            k_scatter_d<<<kGS, kTB, 0, s>>>((double *)tmp, P.ext, n, 3, P.cap, P.rank);
            break;
        case DEM_F_M: k_scatter_mI<<<kGS, kTB, 0, s>>>((double *)tmp, P.mI, n, P.cap, P.rank, 0); break;
        case DEM_F_I: k_scatter_mI<<<kGS, kTB, 0, s>>>((double *)tmp, P.mI, n, P.cap, P.rank, 1); break;
        case DEM_F_TNG_IDX: k_scatter_i<<<kGS, kTB, 0, s>>>((int *)tmp, P.tidx, n, P.mc, P.cap, P.rank, 1); break;
        case DEM_F_TNG_SS_X: case DEM_F_TNG_SS_Y: case DEM_F_TNG_SS_Z:
            k_scatter_d<<<kGS, kTB, 0, s>>>((double *)tmp, P.th + (long)(field - DEM_F_TNG_SS_X) * P.mc * P.cap, n, P.mc,
                                            P.cap, P.rank);
            break;
        case DEM_F_TNG_COUNT: k_scatter_count<<<kGS, kTB, 0, s>>>((int *)tmp, P.cstate, n, P.rank); break;
        case DEM_F_TNG_SW_X: case DEM_F_TNG_SW_Y: case DEM_F_TNG_SW_Z:
            k_scatter_d<<<kGS, kTB, 0, s>>>((double *)tmp, P.sw + (long)(field - DEM_F_TNG_SW_X) * P.mw * P.cap, n, P.mw,
                                            P.cap, P.rank);
            k_sw_mask<<<kGS, kTB, 0, s>>>(P);
            break;
        case DEM_F_SCENE: {
            const int *sc = (const int *)host;
            int mx = 0;
            for (int i = 0; i < n; ++i) {
                if (sc[i] < 0 || sc[i] > (1 << 24)) return fail(ctx, DEM_ERR_INVALID, "scene index out of range");
                mx = std::max(mx, sc[i]);
            }
            if (!P.scene) {
                CK(dalloc(&P.scene, (size_t)P.cap));
                CK(dalloc(&p->alt.scene, (size_t)P.cap));
            }
            k_scatter_i<<<kGS, kTB, 0, s>>>((int *)tmp, P.scene, n, 1, P.cap, P.rank, 0);
            p->nscenes = mx + 1;
            {
                std::vector<int> cnt(p->nscenes, 0);
                for (int i = 0; i < n; ++i) ++cnt[sc[i]];
                p->max_scene = *std::max_element(cnt.begin(), cnt.end());
            }
            p->mat_dirty = true;
            break;
        }
        case DEM_F_FIX: {
            k_scatter_u8<<<kGS, kTB, 0, s>>>((uint8_t *)tmp, P.fix, n, P.rank);
            const uint8_t *f = (const uint8_t *)host;
            bool any = false;
            for (int i = 0; i < n && !any; ++i) any = f[i] != 0;
            p->any_fix = any;
            p->mat_dirty = true;   // re-derive the force constants (has_fix)
            break;
        }
    }
    cudaError_t e = cudaGetLastError();
    CK(e);
    p->dirty = true;
    k_invalidate<<<1, 32, 0, s>>>(p->ctl);
    return DEM_OK;
}

__global__ void k_clear_slots(Particles P) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += gridDim.x * blockDim.x)
        for (int k = 0; k < P.mc; ++k) P.tidx[(long)k * P.cap + i] = -1;
}

extern "C" int dem_particles_clear_contacts(dem_particles *p) {
    if (!p) return DEM_ERR_INVALID;
    dem_ctx *ctx = p->ctx;
    cudaStream_t s = ctx->stream;
    Particles &P = p->P;
    const size_t cn = (size_t)P.cap;
    CK(cudaMemsetAsync(P.cstate, 0, sizeof(int) * cn, s));
    CK(cudaMemsetAsync(P.th, 0, sizeof(double) * 3 * std::max(P.mc, 1) * cn, s));
    CK(cudaMemsetAsync(P.sw, 0, sizeof(double) * 3 * std::max(P.mw, 1) * cn, s));
    k_clear_slots<<<kGS, kTB, 0, s>>>(P);
    CK(cudaGetLastError());
    p->dirty = true;
    k_invalidate<<<1, 32, 0, s>>>(p->ctl);
    return DEM_OK;
}

extern "C" int dem_particles_clear_forces(dem_particles *p) {
    if (!p) return DEM_ERR_INVALID;
    dem_ctx *ctx = p->ctx;
    const size_t cn = (size_t)p->P.cap;
    CK(cudaMemsetAsync(p->P.force, 0, sizeof(double) * 3 * cn, ctx->stream));
    CK(cudaMemsetAsync(p->P.torque, 0, sizeof(double) * 3 * cn, ctx->stream));
    return DEM_OK;
}

static int particles_get_impl(dem_particles *p, int field, void *host, long count, bool device) {
    if (!p || !host) return DEM_ERR_INVALID;
    dem_ctx *ctx = p->ctx;
    long need;
    int es;
    if (!field_layout(p, field, &need, &es) || count != need)
        return fail(ctx, DEM_ERR_INVALID, "dem_particles_get: unknown field or wrong element count");
    const int n = p->P.n;
    cudaStream_t s = ctx->stream;
    Particles &P = p->P;
    if (field == DEM_F_RHO || field == DEM_F_E || field == DEM_F_NU || field == DEM_F_G) {
        const std::vector<double> &src = field == DEM_F_RHO ? p->rho : field == DEM_F_E ? p->E : field == DEM_F_NU ? p->nu : p->G;
        if (device) {
            CK(cudaMemcpyAsync(host, src.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));
            CK(cudaStreamSynchronize(s));
        } else {
            std::memcpy(host, src.data(), sizeof(double) * n);
        }
        return DEM_OK;
    }
    if (field == DEM_F_EXT_FORCE && !P.ext) {
        if (device) CK(cudaMemsetAsync(host, 0, sizeof(double) * 3 * n, s));
        else std::memset(host, 0, sizeof(double) * 3 * n);
        return DEM_OK;
    }
    void *tmp = p->stage;
    const int *cur = &p->ctl->cur, *vcur = &p->ctl->vcur;
    switch (field) {
        case DEM_F_X: k_gather_pos_sel<<<kGS, kTB, 0, s>>>(P.pos[0], P.pos[1], cur, (double *)tmp, n, P.rank, 0); break;
        case DEM_F_RAD: k_gather_pos_sel<<<kGS, kTB, 0, s>>>(P.pos[0], P.pos[1], cur, (double *)tmp, n, P.rank, 1); break;
        case DEM_F_U:
            k_gather_d_sel<<<kGS, kTB, 0, s>>>(P.vel[0], P.vel[1], vcur, (double *)tmp, n, 3, P.cap, P.rank);
            break;
        case DEM_F_OMEGA:
            k_gather_d_sel<<<kGS, kTB, 0, s>>>(P.omg[0], P.omg[1], vcur, (double *)tmp, n, 3, P.cap, P.rank);
            break;
        case DEM_F_FORCE: k_gather_d<<<kGS, kTB, 0, s>>>(P.force, (double *)tmp, n, 3, P.cap, P.rank); break;
        case DEM_F_TORQUE: k_gather_d<<<kGS, kTB, 0, s>>>(P.torque, (double *)tmp, n, 3, P.cap, P.rank); break;
        case DEM_F_EXT_FORCE: k_gather_d<<<kGS, kTB, 0, s>>>(P.ext, (double *)tmp, n, 3, P.cap, P.rank); break;
        case DEM_F_M: k_gather_mI<<<kGS, kTB, 0, s>>>(P.mI, (double *)tmp, n, P.cap, P.rank, 0); break;
        case DEM_F_I: k_gather_mI<<<kGS, kTB, 0, s>>>(P.mI, (double *)tmp, n, P.cap, P.rank, 1); break;
        case DEM_F_TNG_IDX: k_gather_i<<<kGS, kTB, 0, s>>>(P.tidx, (int *)tmp, n, P.mc, P.cap, P.rank, P.perm, 1); break;
        case DEM_F_TNG_SS_X: case DEM_F_TNG_SS_Y: case DEM_F_TNG_SS_Z:
            k_gather_d<<<kGS, kTB, 0, s>>>(P.th + (long)(field - DEM_F_TNG_SS_X) * P.mc * P.cap, (double *)tmp, n, P.mc,
                                           P.cap, P.rank);
            break;
        case DEM_F_TNG_COUNT: k_gather_count<<<kGS, kTB, 0, s>>>(P.cstate, (int *)tmp, n, P.rank); break;
        case DEM_F_TNG_SW_X: case DEM_F_TNG_SW_Y: case DEM_F_TNG_SW_Z:
            k_gather_d<<<kGS, kTB, 0, s>>>(P.sw + (long)(field - DEM_F_TNG_SW_X) * P.mw * P.cap, (double *)tmp, n, P.mw,
                                           P.cap, P.rank);
            break;
        case DEM_F_FIX: k_gather_u8<<<kGS, kTB, 0, s>>>(P.fix, (uint8_t *)tmp, n, P.rank); break;
        case DEM_F_SCENE:
            if (P.scene) k_gather_i<<<kGS, kTB, 0, s>>>(P.scene, (int *)tmp, n, 1, P.cap, P.rank, P.perm, 0);
            else cudaMemsetAsync(tmp, 0, sizeof(int) * n, s);
            break;
    }
    cudaError_t e = cudaGetLastError();
    if (device) {
        // stream-ordered: the copy is complete for any later work on this context's stream
        if (e == cudaSuccess) e = cudaMemcpyAsync(host, tmp, (size_t)need * es, cudaMemcpyDeviceToDevice, s);
    } else {
        if (e == cudaSuccess) e = cudaMemcpyAsync(host, tmp, (size_t)need * es, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    CK(e);
    return DEM_OK;
}

extern "C" int dem_particles_get(dem_particles *p, int field, void *host, long count) {
    return particles_get_impl(p, field, host, count, false);
}

extern "C" int dem_particles_get_device(dem_particles *p, int field, void *dev, long count) {
    return particles_get_impl(p, field, dev, count, true);
}

// ---- walls --------------------------------------------------------------------------
extern "C" int dem_walls_create(dem_ctx *ctx, int n, dem_walls **out) {
    if (!ctx || !out || n < 0 || n > (1 << 20)) return fail(ctx, DEM_ERR_INVALID, "dem_walls_create: 0 <= n <= 2^20");
    dem_walls *w = new dem_walls();
    w->ctx = ctx;
    w->n = n;
    w->x.assign(3 * n, 0.0);
    w->u.assign(3 * n, 0.0);
    w->omega.assign(3 * n, 0.0);
    w->normal.assign(3 * n, 0.0);
    w->E.assign(n, 0.0);
    w->nu.assign(n, 0.0);
    w->G.assign(n, 0.0);
    *out = w;
    return DEM_OK;
}

extern "C" int dem_walls_destroy(dem_walls *w) {
    if (!w) return DEM_ERR_INVALID;
    delete w;
    return DEM_OK;
}

extern "C" int dem_walls_set(dem_walls *w, int field, const double *host, long count) {
    if (!w || !host) return DEM_ERR_INVALID;
    std::vector<double> *dst = nullptr;
    long need = w->n;
    switch (field) {
        case DEM_W_X: dst = &w->x; need = 3L * w->n; break;
        case DEM_W_U: dst = &w->u; need = 3L * w->n; break;
        case DEM_W_OMEGA: dst = &w->omega; need = 3L * w->n; break;
        case DEM_W_NORMAL: dst = &w->normal; need = 3L * w->n; break;
        case DEM_W_E: dst = &w->E; break;
        case DEM_W_NU: dst = &w->nu; break;
        case DEM_W_G: dst = &w->G; break;
        default: return fail(w->ctx, DEM_ERR_INVALID, "dem_walls_set: unknown field");
    }
    if (count != need) return fail(w->ctx, DEM_ERR_INVALID, "dem_walls_set: wrong element count");
    std::copy(host, host + count, dst->begin());
    return DEM_OK;
}

// ---- solver -------------------------------------------------------------------------
namespace {

// Host-side constants, each in the reference's expression order.
PairConst pair_const(double E_i, double nu_i, double G_i, double E_j, double nu_j, double G_j) {
    PairConst c{};
    double tmp_1 = (1. - (nu_i * nu_i)) / E_i;   // Force.hpp:196-198
    double tmp_2 = (1. - (nu_j * nu_j)) / E_j;
    const double E_eff = 1. / (tmp_1 + tmp_2);
    tmp_1 = (2. - nu_i) / G_i;                    // Force.hpp:218-220
    tmp_2 = (2. - nu_j) / G_j;
    const double G_eff = 1. / (tmp_1 + tmp_2);
    c.c_kn = 4. / 3. * E_eff;
    c.c_Sn = 2. * E_eff;
    c.c_kt = 8. * G_eff;
    return c;
}

double beta_of(double cor) {   // Force.hpp:206-210
    const double tmp_1 = std::log(cor);
    const double tmp_2 = tmp_1 * tmp_1 + M_PI * M_PI;
    return tmp_1 / std::sqrt(tmp_2);
}

void pick_contact_kernel(dem_solver *s);

int prepare(dem_solver *s) {
    dem_ctx *ctx = s->ctx;
    dem_particles *p = s->p;
    cudaStream_t st = ctx->stream;
    const int n = p->P.n;
    if (p->mat_dirty) {
        // materials = distinct (E, nu, G) in order of first appearance in caller order: each
        // host thread lists those of its range in order, the lists are merged in range order,
        // then each thread writes its particles' material ids
        using Mat = std::tuple<double, double, double>;
        const int nt = host_threads(n);
        std::vector<std::vector<Mat>> found(nt);
        auto index_of = [](const std::vector<Mat> &v, const Mat &k) {
            for (size_t a = 0; a < v.size(); ++a)
                if (v[a] == k) return (int)a;
            return -1;
        };
        host_parallel(n, [&](long b, long e, int t) {
            std::vector<Mat> &mine = found[t];
            int last = -1;   // neighbours in caller order usually share a material: test it first
            for (long i = b; i < e && (int)mine.size() <= kMaxMat; ++i) {
                const Mat k(p->E[i], p->nu[i], p->G[i]);
                if (last >= 0 && mine[last] == k) continue;
                last = index_of(mine, k);
                if (last < 0) {
                    last = (int)mine.size();
                    mine.push_back(k);
                }
            }
        });
        p->mats.clear();
        for (const auto &mine : found)
            for (const Mat &k : mine)
                if (index_of(p->mats, k) < 0) p->mats.push_back(k);
        if ((int)p->mats.size() > kMaxMat) {
            p->mats.clear();
            return fail(ctx, DEM_ERR_UNSUPPORTED, "more than 32 distinct (E, nu, G) materials");
        }
        p->mat.resize(n);
        std::vector<char> nan(nt, 0);   // a NaN constant equals no material (not even its own)
        host_parallel(n, [&](long b, long e, int t) {
            int last = 0;
            for (long i = b; i < e; ++i) {
                const Mat k(p->E[i], p->nu[i], p->G[i]);
                if (!(p->mats[last] == k)) last = index_of(p->mats, k);
                if (last < 0) {
                    nan[t] = 1;
                    last = 0;
                }
                p->mat[i] = (uint8_t)last;
            }
        });
        if (std::find(nan.begin(), nan.end(), 1) != nan.end()) {
            p->mats.clear();
            return fail(ctx, DEM_ERR_INVALID, "a particle's E, nu or G is not a number");
        }
        // through the staging buffer (cap * 24 bytes or more) of the particle set
        uint8_t *tmp = (uint8_t *)p->stage;
        CK(cudaMemcpyAsync(tmp, p->mat.data(), n, cudaMemcpyHostToDevice, st));
        k_scatter_u8<<<kGS, kTB, 0, st>>>(tmp, p->P.mat, n, p->P.rank);
        CK(cudaStreamSynchronize(st));
        p->mat_dirty = false;
        s->built = false;
    }
    const int nm = (int)p->mats.size();
    const int nw = s->w ? s->w->n : 0;
    // wall history slots: checked when the solver runs (scenes may be assigned after creation)
    s->walls_ok = s->wps == 0 ? nw <= p->P.mw : (s->wps <= p->P.mw && nw >= s->nscenes * s->wps);
    if (s->nscenes > 0 && p->nscenes > s->nscenes)
        return fail(ctx, DEM_ERR_INVALID, "a particle's scene index has no scene parameters");
    if (std::max(p->nscenes, s->nscenes) > s->B.cell_cap)   // every scene takes at least one cell key
        return fail(ctx, DEM_ERR_INVALID, "more scenes than cell keys (8 per particle slot)");
    std::vector<PairConst> pp((size_t)nm * nm), pw((size_t)nm * std::max(nw, 1));
    for (int a = 0; a < nm; ++a) {
        const auto &A = p->mats[a];
        for (int b = 0; b < nm; ++b) {
            const auto &B = p->mats[b];
            pp[(size_t)a * nm + b] = pair_const(std::get<0>(A), std::get<1>(A), std::get<2>(A), std::get<0>(B),
                                                std::get<1>(B), std::get<2>(B));
        }
        for (int w = 0; w < nw; ++w)
            pw[(size_t)a * nw + w] = pair_const(std::get<0>(A), std::get<1>(A), std::get<2>(A), s->w->E[w], s->w->nu[w],
                                                s->w->G[w]);
    }
    // moving walls keep their current (device) positions across a re-preparation
    if (s->d_walls && s->walls_move && (int)s->wall_pos.size() == 3 * nw) {
        std::vector<WallGeom> now(nw);
        CK(cudaMemcpyAsync(now.data(), s->d_walls, nw * sizeof(WallGeom), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (int w = 0; w < nw; ++w)
            for (int d = 0; d < 3; ++d) s->wall_pos[3 * w + d] = now[w].x[d];
    } else {
        if (s->w)
            s->wall_pos = s->w->x;
        else
            s->wall_pos.clear();
    }
    const bool wall_static = (s->fp.quirks & DEM_Q6_WALL_STATIC) != 0;
    bool moving = false;
    std::vector<WallGeom> wg(std::max(nw, 1));
    for (int w = 0; w < nw; ++w)
        for (int d = 0; d < 3; ++d) {
            wg[w].x[d] = s->wall_pos[3 * w + d];
            wg[w].n[d] = s->w->normal[3 * w + d];
            wg[w].u[d] = wall_static ? 0.0 : s->w->u[3 * w + d];
            moving = moving || wg[w].u[d] != 0.0;
        }
    cudaFree(s->d_pp);
    cudaFree(s->d_pw);
    cudaFree(s->d_walls);
    CK(dalloc(&s->d_pp, pp.size()));
    CK(dalloc(&s->d_pw, pw.size()));
    CK(dalloc(&s->d_walls, wg.size()));
    CK(cudaMemcpyAsync(s->d_pp, pp.data(), pp.size() * sizeof(PairConst), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(s->d_pw, pw.data(), pw.size() * sizeof(PairConst), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(s->d_walls, wg.data(), wg.size() * sizeof(WallGeom), cudaMemcpyHostToDevice, st));
    // the wall-gap flags of the last build were taken against the previous walls
    CK(cudaMemsetAsync(&p->ctl->wfar_build, 0xff, sizeof(long long), st));
    // mesh: particle materials against the mesh's, in the plane walls' expression order
    cudaFree(s->d_mesh_pm);
    s->d_mesh_pm = nullptr;
    if (s->mesh_nt > 0) {
        std::vector<PairConst> pm(std::max(nm, 1));
        for (int a = 0; a < nm; ++a) {
            const auto &A = p->mats[a];
            pm[a] = pair_const(std::get<0>(A), std::get<1>(A), std::get<2>(A), s->mesh_mat[0], s->mesh_mat[1],
                               s->mesh_mat[2]);
        }
        CK(dalloc(&s->d_mesh_pm, pm.size()));
        CK(cudaMemcpyAsync(s->d_mesh_pm, pm.data(), pm.size() * sizeof(PairConst), cudaMemcpyHostToDevice, st));
    }
    ForceConsts &fc = s->fc;
    fc = ForceConsts{};
    s->walls_move = moving;
    fc.mwalls = moving ? s->d_walls : nullptr;
    if (s->mesh_nt > 0) {
        fc.mesh = s->mesh;
        fc.mesh.pm = s->d_mesh_pm;
        bool mv = false;
        for (int d = 0; d < 3; ++d) {
            fc.mesh.u[d] = wall_static ? 0.0 : s->mesh_u[d];
            mv = mv || fc.mesh.u[d] != 0.0;
        }
        fc.mesh_moving = mv ? 1 : 0;
    }
    const unsigned q = s->fp.quirks;
    const double bpp = beta_of(s->fp.cor_pp), bpw = beta_of(s->fp.cor_pw);
    fc.K_n_pp = -2. * std::sqrt(5. / 6.) * bpp;             // Force.hpp:215
    fc.K_n_pw = -2. * std::sqrt(5. / 6.) * bpw;             // Force.hpp:580
    fc.K_t_pp = (q & DEM_Q2_ETA_T_ZERO) ? -2 * std::sqrt((double)(5 / 6)) * bpp : fc.K_n_pp;   // :224
    fc.K_t_pw = (q & DEM_Q2_ETA_T_ZERO) ? -2 * std::sqrt((double)(5 / 6)) * bpw : fc.K_n_pw;   // :618
    fc.mu_pp = s->fp.mu_pp;
    fc.mu_pw = s->fp.mu_pw;
    fc.dt = s->sp.dt;
    fc.half_dt = 0.5 * s->sp.dt;                             // Integrator.hpp:25
    for (int d = 0; d < 3; ++d) fc.g[d] = s->sp.gravity[d];
    fc.has_gravity = (fc.g[0] != 0.0 || fc.g[1] != 0.0 || fc.g[2] != 0.0) ? 1 : 0;
    fc.quirks = q;
    fc.nmat = nm;
    fc.nwall = nw;
    fc.has_ext = p->P.ext ? 1 : 0;
    fc.has_fix = p->any_fix ? 1 : 0;
    fc.mixed = s->sp.precision == DEM_MIXED ? 1 : 0;
    fc.stream_block = (s->sp.stream_block == 64 || s->sp.stream_block == 256) ? s->sp.stream_block : 128;
    // the staged streaming kernel unless asked: on the 2M lattice (B200, kernel time per step over
    // 1,000 steps) 64.1 us against 68.1 us with one thread per particle; the split forms ran the
    // step in 76.5 us (two kernels) and 78.4 us (two branches)
    fc.split = (s->sp.stream_split >= 1 && s->sp.stream_split <= 4) ? s->sp.stream_split : 4;
    // each step kernel launched as the dependent of the one before (launch_k), unless asked not
    // to or a graph with such launches failed to build on this device (s->no_overlap)
    fc.pdl = (s->sp.launch_overlap != 2 && !s->no_overlap) ? 1 : 0;
    pick_contact_kernel(s);
    fc.scenes = s->nscenes > 0 ? s->d_scenes : nullptr;
    fc.wps = s->nscenes > 0 ? s->wps : 0;
    if (s->B.nscenes < p->nscenes) {   // per-scene grid descriptors and bounding boxes
        cudaFree(s->B.grid);
        cudaFree(s->B.bbox);
        CK(dalloc(&s->B.grid, (size_t)p->nscenes));
        CK(dalloc(&s->B.bbox, 8 * (size_t)p->nscenes));
        s->B.nscenes = p->nscenes;
        s->version++;
    }
    CK(cudaStreamSynchronize(st));
    s->version++;
    return DEM_OK;
}

void free_pairs(dem_solver *s) {
    cudaFree(s->L.pitem);
    cudaFree(s->L.pterm);
    cudaFree(s->L.prec);
    s->L.pitem = nullptr;
    s->L.pterm = nullptr;
    s->L.prec = nullptr;
}

// Work-item buffers of the pair-parallel dense step: one item per list entry and one per wall
// at most, so (maxnb + mw) * cap items (16 B each, and 48 B of force/torque terms); the item
// count cannot pass the buffer.
int ensure_pairs(dem_solver *s) {
    if (s->L.pitem) return DEM_OK;
    dem_ctx *ctx = s->ctx;
    const size_t items = ((size_t)s->L.maxnb + std::max(s->p->P.mw, 0)) * s->p->P.cap;
    CK(dalloc(&s->L.pitem, items));
    CK(dalloc(&s->L.pterm, 3 * items));
    CK(dalloc(&s->L.prec, (size_t)s->p->P.cap));
    return DEM_OK;
}

int alloc_lists(dem_solver *s, int maxnb) {
    dem_ctx *ctx = s->ctx;
    cudaFree(s->L.nn);
    cudaFree(s->L.idx);
    cudaFree(s->L.defer);
    cudaFree(s->L.defer_v);
    cudaFree(s->L.defer_w);
    cudaFree(s->L.wfar);
    cudaFree(s->L.nn_old);
    cudaFree(s->L.idx_old);
    const bool pairs = s->L.pitem != nullptr;
    free_pairs(s);
    s->L.maxnb = maxnb;
    CK(dalloc(&s->L.nn, s->p->P.cap));
    CK(dalloc(&s->L.idx, (size_t)maxnb * s->p->P.cap));
    CK(dalloc(&s->L.defer, s->p->P.cap));
    CK(dalloc(&s->L.defer_v, 3 * (size_t)s->p->P.cap));
    CK(dalloc(&s->L.defer_w, 3 * (size_t)s->p->P.cap));
    CK(dalloc(&s->L.wfar, (size_t)s->p->P.cap));
    CK(dalloc(&s->L.nn_old, (size_t)s->p->P.cap));
    CK(dalloc(&s->L.idx_old, (size_t)maxnb * s->p->P.cap));
    CK(cudaMemsetAsync(s->L.nn, 0, sizeof(int) * s->p->P.cap, ctx->stream));
    CK(cudaMemsetAsync(s->L.wfar, 0, s->p->P.cap, ctx->stream));
    if (pairs) {
        const int st = ensure_pairs(s);
        if (st) return st;
    }
    s->version++;
    s->built = false;
    return DEM_OK;
}

Ctl read_ctl(dem_solver *s) {
    Ctl c{};
    cudaMemcpyAsync(&c, s->p->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s->ctx->stream);
    cudaStreamSynchronize(s->ctx->stream);
    return c;
}

__global__ void k_clear_status(Ctl *ctl, int bits) {
    if (threadIdx.x == 0) ctl->status &= ~bits;
}

bool ref_mode(const dem_solver *s) { return s->sp.rebuild_every_step != 0; }

// Kernels of the next graph.  Up to kOneKernelMaxN particles: always the one-kernel step (the
// three-kernel step is launch-bound there; B200, 4,096 spheres in a walled box: 16.8 -> 10.6 us
// per step).  Larger, few particles in contact (a sparse step): streaming kernel,
// cooperative contact kernel, apply kernel; the cooperative kernel's short dependent chains
// hide memory latency (B200, 2M-sphere lattice: 105 -> 87 us per step late in the run at 8
// lanes).  Most particles in contact (a dense step): one per-thread kernel over every
// particle, which issues fewer instructions per contact than the cooperative one (200k-disk
// dam break at t = 0.3 s: 131 us per step against 197 us at 8 lanes) and needs neither the
// streaming pass nor the apply pass.  contact_lanes 1, 4 or 8 keeps the three-kernel step
// with that contact kernel.
void pick_contact_kernel(dem_solver *s) {
    const int req = s->sp.contact_lanes;
    const bool fits = s->p->P.mc <= kCoopSlots;
    s->fc.all = 0;
    if (req == 1) {
        s->fc.coop = 0;
    } else if (req == 4 || req == 8) {
        s->fc.coop = fits ? req : 0;
    } else {
        // small systems are launch-bound: one kernel per step whatever the density
        const bool one = s->fc.dense || s->p->P.n <= kOneKernelMaxN;
        s->fc.all = one ? 1 : 0;
        s->fc.coop = (!one && fits) ? 8 : 0;
        // a dense step of a larger system: the pair-parallel form, unless the caller asked for
        // the one-kernel form (dense_form 1); dense_form 2 uses it at every size and density
        const int df = s->sp.dense_form;
        if ((one && df == 0 && s->p->P.n > kOneKernelMaxN) || df == 2) s->fc.all = 2;
    }
}

// Whether the kernel forms depend on the density: not for small systems (one kernel per step
// at any density) nor for a pair-parallel step the caller forced (dense_form 2).
bool density_matters(const dem_solver *s) {
    return s->fc.all == 0 || (s->p->P.n > kOneKernelMaxN && s->sp.dense_form != 2);
}

// Pick the contact-kernel build for the next graph from the last step's deferred count: the
// dense build (more resident blocks, wider apply grid) above 30 % of the particles, back to
// the sparse one below 10 %.  Same arithmetic either way; a switch re-captures the graph.
void adapt_density(dem_solver *s, const Ctl &c) {
    if (!density_matters(s)) return;
    const int n = s->p->P.n;
    const double f = n > 0 ? (double)c.last_ndefer / n : 0.0;
    const int want = s->fc.dense ? (f >= 0.10 ? 1 : 0) : (f > 0.30 ? 1 : 0);
    if (want != s->fc.dense) {
        s->fc.dense = want;
        pick_contact_kernel(s);
        s->version++;
    }
}

int check_walls(dem_solver *s) {
    if (s->walls_ok) return DEM_OK;
    return fail(s->ctx, DEM_ERR_INVALID,
                "more walls than MaxNoWalls history slots per particle (assign per-scene walls with "
                "dem_solver_set_scenes) or too few walls for the scenes");
}

// kernels issued by one launch_build (see dem_nbr.cu)
long build_kernel_count(bool resort) { return 13 + (resort ? 7 : 0); }

// Build with overflow handling (host-driven; re-sorts into Morton order).
int build_with(dem_solver *s, bool resort, double delta, double skin);
int build_now(dem_solver *s, bool resort) { return build_with(s, resort, s->sp.delta, s->sp.skin); }

int build_with(dem_solver *s, bool resort, double delta, double skin) {
    dem_ctx *ctx = s->ctx;
    s->scenes_ready = false;   // this build's order partitions the storage by class, not by scene
    if (s->p->has_bonds) resort = false;
    for (int attempt = 0; attempt < 8; ++attempt) {
        launch_build(s->p->P, s->p->alt, s->L, s->B, s->p->ctl, delta, skin, resort, false, ctx->stream);
        s->launches += build_kernel_count(resort);
        if (resort && s->mesh_nt > 0) {   // tracked triangle contacts follow the re-sort (B.key: new <- old)
            const size_t cap = (size_t)s->p->P.cap;
            const MeshDev &M = s->mesh, &A = s->mesh_alt;
            launch_permute_mesh(M, A, s->p->P.n, s->p->P.cap, s->B.key, ctx->stream);
            s->launches += 1;
            CK(cudaMemcpyAsync(M.tid, A.tid, (size_t)M.mt * cap * sizeof(int), cudaMemcpyDeviceToDevice, ctx->stream));
            CK(cudaMemcpyAsync(M.th, A.th, 3 * (size_t)M.mt * cap * sizeof(double), cudaMemcpyDeviceToDevice,
                               ctx->stream));
            CK(cudaMemcpyAsync(M.cnt, A.cnt, cap, cudaMemcpyDeviceToDevice, ctx->stream));
        }
        CK(cudaGetLastError());
        Ctl c = read_ctl(s);
        CK(cudaGetLastError());
        if (!(c.status & DEM_ERR_NEIGHBOR_OVERFLOW)) {
            if (s->mesh_nt > 0) {
                launch_mesh_candidates(s->p->P, s->fc.mesh, s->p->ctl, delta, skin, ctx->stream);
                s->launches += 1;
                CK(cudaGetLastError());
            }
            // wall-gap flags against the stale threshold of the solver's runs
            const double half = s->sp.delta > 0.0 ? std::max(0.0, s->sp.delta - 2.0 * s->p->rmax) / 2.0
                                                  : s->sp.skin / 2.0;
            if (s->d_walls && s->fc.nwall > 0) {
                launch_wall_far(s->p->P, s->L, s->p->ctl, s->fc, s->d_walls, half, ctx->stream);
                s->launches += 1;
                CK(cudaGetLastError());
            }
            s->built = true;
            s->p->dirty = false;
            return DEM_OK;
        }
        const int want = std::min(std::max(2 * s->L.maxnb, c.max_nbr + 8), 128);
        if (c.max_nbr > 128) return fail(ctx, DEM_ERR_NEIGHBOR_OVERFLOW, "more than 128 neighbours per particle");
        int st = alloc_lists(s, want);
        if (st) return st;
        k_clear_status<<<1, 32, 0, ctx->stream>>>(s->p->ctl, DEM_ERR_NEIGHBOR_OVERFLOW);
        resort = false;
    }
    return fail(ctx, DEM_ERR_NEIGHBOR_OVERFLOW, "neighbour list did not converge");
}

int capture_graph(dem_solver *s, int steps) {
    dem_ctx *ctx = s->ctx;
    if (s->fc.all == 2) {
        const int st = ensure_pairs(s);
        if (st) return st;
    }
    if (s->graph) {
        cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < steps; ++k) {
        if (ref_mode(s)) {
            launch_build(s->p->P, s->p->alt, s->L, s->B, s->p->ctl, s->sp.delta, s->sp.skin, false, true, ctx->stream);
            if (s->mesh_nt > 0) launch_mesh_candidates(s->p->P, s->fc.mesh, s->p->ctl, s->sp.delta, s->sp.skin, ctx->stream);
        }
        launch_step(s->p->P, s->L, s->p->ctl, s->fc, s->d_pp, s->d_pw, s->d_walls, MODE_FUSED, ctx->stream, s->aux);
    }
    CK(cudaStreamEndCapture(ctx->stream, &g));
    s->graph_nodes = (long)steps * (kernels_per_step(s->fc) +
                                    (ref_mode(s) ? build_kernel_count(false) + (s->mesh_nt > 0 ? 1 : 0) : 0));
    cudaError_t e = cudaGraphInstantiate(&s->graph, g, 0);
    cudaGraphDestroy(g);
    CK(e);
    s->graph_steps = steps;
    s->graph_version = s->version;
    return DEM_OK;
}

// Steps per iteration of the graph while-loops, longest first: each iteration pays for the
// conditional and the control kernel (about 5 us on a B200).
constexpr int kLoopUnroll = 8;
constexpr int kLoopUnits[] = {kLoopUnroll, 4, 2, 1};
constexpr int kLoopLevels = sizeof(kLoopUnits) / sizeof(kLoopUnits[0]);

// `steps` fused steps (each with the neighbour build first in the rebuild-every-step mode).
static void capture_steps(dem_solver *s, int steps, cudaStream_t st) {
    for (int k = 0; k < steps; ++k) {
        if (ref_mode(s)) {
            launch_build(s->p->P, s->p->alt, s->L, s->B, s->p->ctl, s->sp.delta, s->sp.skin, false, true, st);
            if (s->mesh_nt > 0) launch_mesh_candidates(s->p->P, s->fc.mesh, s->p->ctl, s->sp.delta, s->sp.skin, st);
        }
        launch_step(s->p->P, s->L, s->p->ctl, s->fc, s->d_pp, s->d_pw, s->d_walls, MODE_FUSED, st, s->aux);
    }
}

// Adds a while node after `dep` whose body is `steps` fused steps and k_loop_ctl.
static cudaError_t add_loop(dem_solver *s, cudaGraph_t g, cudaGraphNode_t dep, cudaGraphConditionalHandle h, int steps,
                            int dense, cudaGraphNode_t *node) {
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaError_t e = cudaGraphAddNode(node, g, &dep, 1, &cp);
    if (e != cudaSuccess) return e;
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    cudaStream_t st = s->ctx->stream;
    e = cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    capture_steps(s, steps, st);
    launch_k(k_loop_ctl, 1, 32, 0, st, s->fc.pdl != 0, s->p->ctl, h, s->p->P.n, dense, steps);
    return cudaStreamEndCapture(st, &body);
}

// One kernel node after `dep` (nullptr: a root node), captured from a launch on the stream.
template <typename F>
static cudaError_t add_kernel(cudaGraph_t g, cudaGraphNode_t dep, cudaStream_t st, F launch, cudaGraphNode_t *node) {
    cudaError_t e = cudaStreamBeginCaptureToGraph(st, g, dep ? &dep : nullptr, nullptr, dep ? 1 : 0,
                                                  cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    launch();
    cudaGraph_t out = g;
    e = cudaStreamEndCapture(st, &out);
    if (e != cudaSuccess) return e;
    // the node just added is the one without a dependent
    size_t nn = 0;
    e = cudaGraphGetNodes(g, nullptr, &nn);
    if (e != cudaSuccess) return e;
    std::vector<cudaGraphNode_t> nodes(nn);
    e = cudaGraphGetNodes(g, nodes.data(), &nn);
    if (e != cudaSuccess) return e;
    for (cudaGraphNode_t c : nodes) {
        size_t nd = 0;
        if (cudaGraphNodeGetDependentNodes(c, nullptr, &nd) == cudaSuccess && nd == 0 && c != dep) {
            cudaGraphNodeType t;
            if (cudaGraphNodeGetType(c, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) *node = c;
        }
    }
    return cudaSuccess;
}

// The step loop as one graph: k_loop_begin (loop counter reset, condition of the first loop),
// a while node of kLoopUnroll steps per iteration, then for 4, 2 and 1 steps a k_loop_mid
// (condition of the next loop) and a while node of that many steps per iteration.
int capture_loop_graph(dem_solver *s) {
    dem_ctx *ctx = s->ctx;
    cudaStream_t st = ctx->stream;
    if (s->fc.all == 2) {
        const int e = ensure_pairs(s);
        if (e) return e;
    }
    if (s->graph) {
        cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    CK(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h[kLoopLevels];
    cudaError_t e = cudaSuccess;
    for (int l = 0; l < kLoopLevels && e == cudaSuccess; ++l)
        e = cudaGraphConditionalHandleCreate(&h[l], g, 0, cudaGraphCondAssignDefault);
    const int n = s->p->P.n, dense = density_matters(s) ? s->fc.dense : -1;
    Ctl *ctl = s->p->ctl;
    cudaGraphNode_t cond = nullptr, loop = nullptr;
    if (e == cudaSuccess)
        e = add_kernel(g, nullptr, st, [&] { k_loop_begin<<<1, 32, 0, st>>>(ctl, h[0], n, dense, kLoopUnits[0]); },
                       &cond);
    if (e == cudaSuccess) e = add_loop(s, g, cond, h[0], kLoopUnits[0], dense, &loop);
    for (int l = 1; l < kLoopLevels && e == cudaSuccess; ++l) {
        const cudaGraphConditionalHandle hl = h[l];
        const int unit = kLoopUnits[l];
        e = add_kernel(g, loop, st, [&] { k_loop_mid<<<1, 32, 0, st>>>(ctl, hl, n, dense, unit); }, &cond);
        if (e == cudaSuccess) e = add_loop(s, g, cond, hl, unit, dense, &loop);
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&s->graph, g, 0);
    cudaGraphDestroy(g);
    CK(e);
    s->graph_nodes = kernels_per_step(s->fc) + (ref_mode(s) ? build_kernel_count(false) + (s->mesh_nt > 0 ? 1 : 0) : 0);
    s->graph_steps = -1;
    s->graph_version = s->version;
    return DEM_OK;
}

}  // namespace

extern "C" int dem_solver_create(dem_ctx *ctx, dem_particles *p, dem_walls *w, const dem_force_params *fp,
                                 const dem_solver_params *sp, dem_solver **out) {
    if (!ctx || !p || !fp || !sp || !out || !(sp->dt > 0.0))
        return fail(ctx, DEM_ERR_INVALID, "dem_solver_create: null argument or dt <= 0");
    if (sp->precision != DEM_FP64 && sp->precision != DEM_MIXED)
        return fail(ctx, DEM_ERR_INVALID, "dem_solver_create: unknown precision");
    if (sp->delta <= 0.0 && sp->skin < 0.0) return fail(ctx, DEM_ERR_INVALID, "dem_solver_create: skin < 0");
    dem_solver *s = new dem_solver();
    s->ctx = ctx;
    s->p = p;
    s->w = w;
    s->fp = *fp;
    s->sp = *sp;
    s->loop = s->sp.steps_per_launch <= 0;
    if (s->sp.steps_per_launch <= 0) s->sp.steps_per_launch = 32;
    const int n = p->P.cap;
    BuildBuffers &B = s->B;
    B.cell_cap = std::min<long>(std::max<long>(8L * n, 32768L), 1L << 28);
    cudaError_t e = cudaSuccess;
    auto A = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
    A(dalloc(&B.grid, 1));
    A(dalloc(&B.total, 1));
    B.nscenes = 1;
    A(dalloc(&B.key, n));
    A(dalloc(&B.cell_start, (size_t)B.cell_cap + 1));
    A(dalloc(&B.cell_fill, (size_t)B.cell_cap + 1));
    A(dalloc(&B.cell_items, n));
    A(dalloc(&B.block_sums, (size_t)B.cell_cap / 2048 + 2));
    A(dalloc(&B.bbox, 8));
    A(dalloc(&B.src, n));
    A(dalloc(&B.dst, n));
    A(dalloc(&B.part_sums, 2 * ((size_t)n / kPartBlock + 2)));
    s->nparts = (p->P.n + 127) / 128;
    A(dalloc(&s->d_epart, 4 * (size_t)s->nparts));
    A(dalloc(&s->d_eout, 4));
    A(cudaStreamCreateWithFlags(&s->aux.stream, cudaStreamNonBlocking));
    A(cudaEventCreateWithFlags(&s->aux.fork, cudaEventDisableTiming));
    A(cudaEventCreateWithFlags(&s->aux.join, cudaEventDisableTiming));
    if (e != cudaSuccess) {
        dem_solver_destroy(s);
        return cuda_check(ctx, e, "dem_solver_create");
    }
    int st = alloc_lists(s, sp->max_neighbors > 0 ? std::min(sp->max_neighbors, 128) : 32);
    if (!st) st = prepare(s);
    if (st) {
        dem_solver_destroy(s);
        return st;
    }
    *out = s;
    return DEM_OK;
}

static void free_mesh(dem_solver *s) {
    cudaFree(const_cast<double *>(s->mesh.tri));
    cudaFree(s->mesh.D);
    cudaFree(s->mesh.tid);
    cudaFree(s->mesh.th);
    cudaFree(s->mesh.cnt);
    cudaFree(s->mesh.cand);
    cudaFree(s->mesh.ncand);
    cudaFree(s->mesh_alt.tid);
    cudaFree(s->mesh_alt.th);
    cudaFree(s->mesh_alt.cnt);
    cudaFree(s->d_mesh_pm);
    s->mesh = MeshDev{};
    s->mesh_alt = MeshDev{};
    s->d_mesh_pm = nullptr;
    s->mesh_nt = 0;
}

extern "C" int dem_solver_destroy(dem_solver *s) {
    if (!s) return DEM_ERR_INVALID;
    cudaStreamSynchronize(s->ctx->stream);
    if (s->graph) cudaGraphExecDestroy(s->graph);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    if (s->aux.stream) {
        cudaStreamSynchronize(s->aux.stream);
        cudaStreamDestroy(s->aux.stream);
    }
    if (s->aux.fork) cudaEventDestroy(s->aux.fork);
    if (s->aux.join) cudaEventDestroy(s->aux.join);
    cudaFree(s->d_pp); cudaFree(s->d_pw); cudaFree(s->d_walls); cudaFree(s->d_scenes);
    cudaFree(s->d_scene_table); cudaFree(s->d_scene_counts); cudaFree(s->d_scene_bad);
    cudaFree(s->L.nn); cudaFree(s->L.idx); cudaFree(s->L.defer); cudaFree(s->L.defer_v); cudaFree(s->L.defer_w);
    cudaFree(s->L.wfar); cudaFree(s->L.nn_old); cudaFree(s->L.idx_old);
    free_pairs(s);
    BuildBuffers &B = s->B;
    cudaFree(B.grid); cudaFree(B.total); cudaFree(B.key); cudaFree(B.cell_start); cudaFree(B.cell_fill); cudaFree(B.cell_items);
    cudaFree(B.block_sums); cudaFree(B.bbox); cudaFree(B.src); cudaFree(B.dst);
    cudaFree(B.part_sums);
    cudaFree(s->d_epart); cudaFree(s->d_eout);
    cudaFree(s->d_coop);
    free_mesh(s);
    delete s;
    return DEM_OK;
}

extern "C" int dem_solver_set_mesh(dem_solver *s, const double *tri, int nt, double E, double nu, double G,
                                   const double *velocity, int max_contacts) {
    if (!s) return DEM_ERR_INVALID;
    dem_ctx *ctx = s->ctx;
    if (nt < 0 || nt > kMeshMaxTri || (nt > 0 && !tri))
        return fail(ctx, DEM_ERR_INVALID, "dem_solver_set_mesh: 0 <= triangles <= 4096");
    if (nt > 0 && (max_contacts < 1 || max_contacts > kMeshMaxContacts))
        return fail(ctx, DEM_ERR_INVALID, "dem_solver_set_mesh: 1 <= max_contacts <= 16");
    if (nt > 0 && !(E > 0. && G > 0.)) return fail(ctx, DEM_ERR_INVALID, "dem_solver_set_mesh: E, G > 0");
    if (nt > 0 && (s->nscenes > 0 || s->p->has_bonds))
        return fail(ctx, DEM_ERR_UNSUPPORTED, "dem_solver_set_mesh: not with batched scenes or bonds");
    CK(cudaStreamSynchronize(ctx->stream));
    free_mesh(s);
    if (nt > 0) {
        const size_t cap = (size_t)s->p->P.cap;
        MeshDev &M = s->mesh;
        double *dtri = nullptr;
        cudaError_t e = cudaSuccess;
        auto A = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
        A(dalloc(&dtri, 9 * (size_t)nt));
        A(dalloc(&M.D, 3));
        A(dalloc(&M.tid, (size_t)max_contacts * cap));
        A(dalloc(&M.th, 3 * (size_t)max_contacts * cap));
        A(dalloc(&M.cnt, cap));
        A(dalloc(&M.cand, (size_t)kMeshCand * cap));
        A(dalloc(&M.ncand, cap));
        A(dalloc(&s->mesh_alt.tid, (size_t)max_contacts * cap));
        A(dalloc(&s->mesh_alt.th, 3 * (size_t)max_contacts * cap));
        A(dalloc(&s->mesh_alt.cnt, cap));
        M.tri = dtri;
        if (e != cudaSuccess) {
            free_mesh(s);
            return cuda_check(ctx, e, "dem_solver_set_mesh");
        }
        cudaStream_t st = ctx->stream;
        CK(cudaMemcpyAsync(dtri, tri, 9 * (size_t)nt * sizeof(double), cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(M.D, 0, 3 * sizeof(double), st));
        CK(cudaMemsetAsync(M.tid, 0xff, (size_t)max_contacts * cap * sizeof(int), st));   // -1
        CK(cudaMemsetAsync(M.th, 0, 3 * (size_t)max_contacts * cap * sizeof(double), st));
        CK(cudaMemsetAsync(M.cnt, 0, cap, st));
        CK(cudaMemsetAsync(M.ncand, 0, cap, st));
        M.nt = nt;
        M.mt = max_contacts;
        s->mesh_alt.nt = nt;
        s->mesh_alt.mt = max_contacts;
        s->mesh_nt = nt;
        s->mesh_mat[0] = E;
        s->mesh_mat[1] = nu;
        s->mesh_mat[2] = G;
        for (int d = 0; d < 3; ++d) s->mesh_u[d] = velocity ? velocity[d] : 0.0;
        CK(cudaStreamSynchronize(st));
    }
    s->built = false;
    return prepare(s);
}

extern "C" int dem_solver_mesh_translation(dem_solver *s, double *host3) {
    if (!s || !host3) return DEM_ERR_INVALID;
    host3[0] = host3[1] = host3[2] = 0.0;
    if (s->mesh_nt == 0) return DEM_OK;
    dem_ctx *ctx = s->ctx;
    CK(cudaMemcpyAsync(host3, s->mesh.D, 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return DEM_OK;
}

namespace {
// Whether a run takes the persistent per-scene form: batched scenes of at most
// kSceneMaxParticles particles, the Verlet-skin mode, static walls, no mesh, no bonds, the
// per-step forms not chosen by the caller.
bool scenes_persistent(const dem_solver *s) {
    return s->sp.scene_kernel == 0 && s->nscenes > 0 && s->p->P.scene && s->p->max_scene > 0 &&
           s->p->max_scene <= kSceneMaxParticles && !ref_mode(s) && s->mesh_nt == 0 && !s->fc.mwalls &&
           !s->p->has_bonds && s->sp.contact_lanes == 0 && s->sp.dense_form == 0 && !s->scenes_unfit;
}

// A run in one persistent launch (dem_scenes.cuh).  Returns DEM_ERR_UNSUPPORTED, with nothing
// changed, when the storage turns out not to hold every scene contiguously (the caller then
// takes the per-step form).
int run_scenes(dem_solver *s, int nsteps) {
    dem_ctx *ctx = s->ctx;
    cudaStream_t st = ctx->stream;
    if (s->L.maxnb < kSceneMaxParticles) {
        const int e = alloc_lists(s, kSceneMaxParticles);
        if (e) return e;
    }
    if (!s->scenes_ready || s->p->dirty) {
        // re-sort in plain cell order (scene-major keys): every scene contiguous
        for (int attempt = 0;; ++attempt) {
            launch_build(s->p->P, s->p->alt, s->L, s->B, s->p->ctl, s->sp.delta, s->sp.skin, true, false, st, false);
            s->launches += build_kernel_count(true);
            const Ctl c = read_ctl(s);
            if (!(c.status & DEM_ERR_NEIGHBOR_OVERFLOW)) break;
            if (attempt >= 2 || c.max_nbr > 128) return fail(ctx, DEM_ERR_NEIGHBOR_OVERFLOW, "neighbour list overflow");
            const int e = alloc_lists(s, std::min(std::max(2 * s->L.maxnb, c.max_nbr + 8), 128));
            if (e) return e;
            k_clear_status<<<1, 32, 0, st>>>(s->p->ctl, DEM_ERR_NEIGHBOR_OVERFLOW);
        }
        s->p->dirty = false;
        const int ns = s->p->nscenes;
        if (s->scene_table_n < ns) {
            cudaFree(s->d_scene_table);
            cudaFree(s->d_scene_counts);
            cudaFree(s->d_scene_bad);
            s->d_scene_table = nullptr;
            s->d_scene_counts = s->d_scene_bad = nullptr;
            CK(dalloc(&s->d_scene_table, (size_t)ns));
            CK(dalloc(&s->d_scene_counts, (size_t)ns));
            CK(dalloc(&s->d_scene_bad, 1));
            s->scene_table_n = ns;
        }
        if (!launch_scene_table(s->p->P, ns, s->d_scene_table, s->d_scene_counts, s->d_scene_bad, st)) {
            CK(cudaGetLastError());
            s->scenes_unfit = true;
            s->built = false;
            return DEM_ERR_UNSUPPORTED;
        }
        s->scenes_ready = true;
    }
    const double half_skin = 1e300;   // lists are rebuilt inside the launch, every step
    k_run_begin<<<1, 32, 0, st>>>(s->p->ctl, nsteps, half_skin);
    launch_prologue(s->p->P, s->p->ctl, s->fc, st);
    launch_scene_steps(s->p->P, s->L, s->p->ctl, s->fc, s->d_pp, s->d_pw, s->d_walls, s->d_scene_table,
                       s->p->nscenes, nsteps, s->sp.delta, s->sp.skin, st);
    s->launches += 4;
    CK(cudaGetLastError());
    const Ctl c = read_ctl(s);
    CK(cudaGetLastError());
    s->built = false;   // the lists are per-scene lists of the last step, not a Verlet list
    if (c.status & DEM_ERR_NEIGHBOR_OVERFLOW) return fail(ctx, DEM_ERR_NEIGHBOR_OVERFLOW, "scene list overflow");
    return c.status & (DEM_ERR_CONTACT_OVERFLOW | DEM_ERR_NAN);
}
}  // namespace

// The run's steps in cooperative launches (dem_persist.cuh) rather than graph replays: the
// one-kernel step of a small system in the Verlet-skin mode, with the step loop in while-loop
// graphs (steps_per_launch 0, so no profiler asked for fixed graphs).
bool coop_loop(const dem_solver *s) {
    return s->sp.cooperative_loop != 2 && !s->coop_refused && s->fc.all == 1 && s->p->P.n <= kCoopMaxN &&
           s->loop && !ref_mode(s);
}

extern "C" int dem_solver_run(dem_solver *s, int nsteps) {
    if (!s) return DEM_ERR_INVALID;
    if (nsteps <= 0) return DEM_OK;
    dem_ctx *ctx = s->ctx;
    if (s->p->mat_dirty || (s->p->P.ext != nullptr) != (s->fc.has_ext != 0)) {
        int st = prepare(s);
        if (st) return st;
    }
    {
        const int wst = check_walls(s);
        if (wst) return wst;
    }
    if (scenes_persistent(s)) {
        const int e = run_scenes(s, nsteps);
        if (e != DEM_ERR_UNSUPPORTED) return e;
    }
    cudaStream_t st = ctx->stream;
    double half_skin;
    if (ref_mode(s)) half_skin = 1e300;
    else if (s->sp.delta > 0.0) half_skin = std::max(0.0, s->sp.delta - 2.0 * s->p->rmax) / 2.0;
    else half_skin = s->sp.skin / 2.0;
    k_run_begin<<<1, 32, 0, st>>>(s->p->ctl, nsteps, half_skin, ref_mode(s) ? 1 : 0);
    launch_prologue(s->p->P, s->p->ctl, s->fc, st);
    s->launches += 2;
    s->graph_done_mark = 0;
    CK(cudaGetLastError());
    const int chunk = s->sp.steps_per_launch;
    // the graph of the next replay: the step loop (while node), or `chunk` gated steps
    auto ensure_graph = [&]() -> int {
        const bool loop_stale = !s->graph || s->graph_version != s->version || s->graph_steps != -1;
        const bool chunk_stale = !s->graph || s->graph_version != s->version || s->graph_steps != chunk;
        if (s->loop ? !loop_stale : !chunk_stale) return DEM_OK;
        int e = s->loop ? capture_loop_graph(s) : capture_graph(s, chunk);
        if (e != DEM_OK && s->fc.pdl) {   // dependent launches refused in a graph: capture without them
            (void)cudaGetLastError();
            s->no_overlap = true;
            s->fc.pdl = 0;
            e = s->loop ? capture_loop_graph(s) : capture_graph(s, chunk);
        }
        return e;
    };
    // kernels one replay launched: per iteration of the loop graph, per captured step otherwise
    // (loop graph: every step's kernels, a control kernel per iteration, the two condition nodes)
    int steps_before = 0;
    auto count_launches = [&](const Ctl &c) {
        s->launches += s->loop ? kLoopLevels + (long)(c.steps_done - steps_before) * s->graph_nodes + c.loop_iter
                               : s->graph_nodes;
        steps_before = c.steps_done;
    };
    if (ref_mode(s)) {
        // rebuild before every force pass, inside the graph (no re-sort)
        for (;;) {
            {
                int e = ensure_graph();
                if (e) return e;
            }
            Ctl c{};
            int done_before = -1;
            for (;;) {
                CK(cudaGraphLaunch(s->graph, st));
                c = read_ctl(s);
                count_launches(c);
                if (c.status & DEM_ERR_TIMEOUT) return fail(ctx, DEM_ERR_TIMEOUT, "a bounded device wait gave up");
                adapt_density(s, c);
                if (c.steps_done >= c.target || (c.status & DEM_ERR_NEIGHBOR_OVERFLOW) || c.steps_done == done_before)
                    break;
                done_before = c.steps_done;
                if (s->loop && s->graph_version != s->version) break;   // kernel form switched: recapture
            }
            if (c.status & DEM_ERR_NEIGHBOR_OVERFLOW) {
                const int want = std::min(std::max(2 * s->L.maxnb, c.max_nbr + 8), 128);
                if (c.max_nbr > 128) return fail(ctx, DEM_ERR_NEIGHBOR_OVERFLOW, "more than 128 neighbours");
                int e = alloc_lists(s, want);
                if (e) return e;
                k_clear_status<<<1, 32, 0, st>>>(s->p->ctl, DEM_ERR_NEIGHBOR_OVERFLOW);
                continue;
            }
            if (c.steps_done >= c.target) break;
            // the loop graph left to switch kernel forms (a switch needs a step, so this progresses)
            if (s->loop && s->graph_version != s->version) continue;
            return fail(ctx, DEM_ERR_CUDA, "solver made no progress");
        }
    } else {
        if (!s->built || s->p->dirty) {
            int e = build_now(s, true);
            if (e) return e;
        }
        if (!s->ev0) {
            CK(cudaEventCreate(&s->ev0));
            CK(cudaEventCreate(&s->ev1));
        }
        s->coop_ran = false;
        for (int guard = 0;; ++guard) {
            if (coop_loop(s)) {   // every step until the target or a stale list in one launch
                if (!s->d_coop) CK(dalloc(&s->d_coop, (size_t)kCoopScratch));
                CK(cudaEventRecord(s->ev0, st));
                const cudaError_t le = launch_steps_coop(s->p->P, s->L, s->p->ctl, s->fc, s->d_pp, s->d_pw, s->d_walls,
                                                         nsteps, s->d_coop, st);
                if (le != cudaSuccess) {   // not resident at once (or refused): graph replays from here on
                    (void)cudaGetLastError();
                    s->coop_refused = true;
                    continue;
                }
                CK(cudaEventRecord(s->ev1, st));
                s->coop_ran = true;
                s->launches += 1;
                const int done_before = s->graph_done_mark;
                Ctl c = read_ctl(s);
                CK(cudaGetLastError());
                if (c.status & DEM_ERR_TIMEOUT) return fail(ctx, DEM_ERR_TIMEOUT, "a bounded device wait gave up");
                float ms = 0.f;
                CK(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
                s->graph_ms += ms;
                s->graph_steps_run += c.steps_done - done_before;
                s->graph_done_mark = c.steps_done;
                if (c.steps_done >= c.target) break;
                if (!(c.disp < c.half_skin)) {
                    int e = build_now(s, true);
                    if (e) return e;
                } else if (c.steps_done == done_before) {
                    return fail(ctx, DEM_ERR_CUDA, "solver made no progress");
                }
                if (guard > 4 * (nsteps + 4)) return fail(ctx, DEM_ERR_CUDA, "solver made no progress");
                continue;
            }
            {
                int e = ensure_graph();
                if (e) return e;
            }
            CK(cudaEventRecord(s->ev0, st));
            CK(cudaGraphLaunch(s->graph, st));
            CK(cudaEventRecord(s->ev1, st));
            const int done_before = s->graph_done_mark;
            Ctl c = read_ctl(s);
            CK(cudaGetLastError());
            count_launches(c);
            if (c.status & DEM_ERR_TIMEOUT) return fail(ctx, DEM_ERR_TIMEOUT, "a bounded device wait gave up");
            adapt_density(s, c);
            {
                float ms = 0.f;
                CK(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
                s->graph_ms += ms;
                s->graph_steps_run += c.steps_done - done_before;
                s->graph_done_mark = c.steps_done;
            }
            if (c.steps_done >= c.target) break;
            if (!(c.disp < c.half_skin)) {
                int e = build_now(s, true);
                if (e) return e;
            }
            if (guard > 4 * (nsteps + 4)) return fail(ctx, DEM_ERR_CUDA, "solver made no progress");
        }
    }
    Ctl c = read_ctl(s);
    CK(cudaGetLastError());
    return c.status & (DEM_ERR_CONTACT_OVERFLOW | DEM_ERR_NAN);
}

extern "C" int dem_solver_wall_positions(dem_solver *s, double *host, long count) {
    if (!s || !host) return DEM_ERR_INVALID;
    const int nw = s->w ? s->w->n : 0;
    if (count != 3L * nw) return fail(s->ctx, DEM_ERR_INVALID, "dem_solver_wall_positions: count != 3 * walls");
    if (nw == 0) return DEM_OK;
    if (!s->d_walls) {
        std::copy(s->w->x.begin(), s->w->x.end(), host);
        return DEM_OK;
    }
    std::vector<WallGeom> now(nw);
    dem_ctx *ctx = s->ctx;
    CK(cudaMemcpyAsync(now.data(), s->d_walls, nw * sizeof(WallGeom), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (int w = 0; w < nw; ++w)
        for (int d = 0; d < 3; ++d) host[3 * w + d] = now[w].x[d];
    return DEM_OK;
}

extern "C" int dem_solver_stats(dem_solver *s, dem_run_stats *out) {
    if (!s || !out) return DEM_ERR_INVALID;
    Ctl c = read_ctl(s);
    out->steps = c.total_steps;
    out->rebuilds = c.rebuilds;
    out->max_neighbors = c.max_nbr;
    out->neighbor_capacity = s->L.maxnb;
    out->status = c.status;
    out->disp_bound = c.disp;
    out->launches = s->launches;
    out->graph_ms = s->graph_ms;
    out->graph_steps = s->graph_steps_run;
    out->launch_overlap = s->fc.pdl;
    out->cooperative_loop = s->coop_ran ? 1 : 0;
    return DEM_OK;
}

extern "C" int dem_solver_set_scenes(dem_solver *s, const dem_scene_params *params, int nscenes, int walls_per_scene) {
    if (!s || !params || nscenes <= 0 || walls_per_scene < 0) return DEM_ERR_INVALID;
    dem_ctx *ctx = s->ctx;
    std::vector<SceneConst> sc(nscenes);
    for (int k = 0; k < nscenes; ++k) {
        const double bpp = beta_of(params[k].cor_pp), bpw = beta_of(params[k].cor_pw);
        const unsigned q = s->fp.quirks;
        sc[k].K_n_pp = -2. * std::sqrt(5. / 6.) * bpp;
        sc[k].K_n_pw = -2. * std::sqrt(5. / 6.) * bpw;
        sc[k].K_t_pp = (q & DEM_Q2_ETA_T_ZERO) ? -2 * std::sqrt((double)(5 / 6)) * bpp : sc[k].K_n_pp;
        sc[k].K_t_pw = (q & DEM_Q2_ETA_T_ZERO) ? -2 * std::sqrt((double)(5 / 6)) * bpw : sc[k].K_n_pw;
        sc[k].mu_pp = params[k].mu_pp;
        sc[k].mu_pw = params[k].mu_pw;
    }
    cudaFree(s->d_scenes);
    s->d_scenes = nullptr;
    CK(dalloc(&s->d_scenes, (size_t)nscenes));
    CK(cudaMemcpy(s->d_scenes, sc.data(), sizeof(SceneConst) * nscenes, cudaMemcpyHostToDevice));
    s->nscenes = nscenes;
    s->wps = walls_per_scene;
    s->built = false;
    return prepare(s);
}

extern "C" int dem_solver_profile(dem_solver *s, int nsteps, double *kernel_ms) {
    if (!s || !kernel_ms) return DEM_ERR_INVALID;
    *kernel_ms = 0.0;
    if (nsteps <= 0) return DEM_OK;
    dem_ctx *ctx = s->ctx;
    if (ref_mode(s)) return fail(ctx, DEM_ERR_UNSUPPORTED, "dem_solver_profile: skin mode only");
    if (s->p->mat_dirty || (s->p->P.ext != nullptr) != (s->fc.has_ext != 0)) {
        int st = prepare(s);
        if (st) return st;
    }
    {
        const int wst = check_walls(s);
        if (wst) return wst;
    }
    cudaStream_t st = ctx->stream;
    const double half_skin = s->sp.delta > 0.0 ? std::max(0.0, s->sp.delta - 2.0 * s->p->rmax) / 2.0 : s->sp.skin / 2.0;
    k_run_begin<<<1, 32, 0, st>>>(s->p->ctl, nsteps, half_skin);
    launch_prologue(s->p->P, s->p->ctl, s->fc, st);
    s->launches += 2;
    if (!s->built || s->p->dirty) {
        int e = build_now(s, true);
        if (e) return e;
    }
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    double sum = 0.0;
    long timed = 0;
    int done = 0;
    for (int guard = 0; guard < 4 * (nsteps + 4); ++guard) {
        CK(cudaEventRecord(e0, st));
        launch_step(s->p->P, s->L, s->p->ctl, s->fc, s->d_pp, s->d_pw, s->d_walls, MODE_FUSED, st, s->aux);
        CK(cudaEventRecord(e1, st));
        s->launches += kernels_per_step(s->fc);
        CK(cudaEventSynchronize(e1));
        const Ctl c = read_ctl(s);
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        if (c.steps_done > done) {   // the launch did a step (a stale list makes it a no-op)
            sum += ms;
            ++timed;
            done = c.steps_done;
        }
        if (c.steps_done >= c.target) break;
        if (!(c.disp < c.half_skin)) {
            int e = build_now(s, true);
            if (e) return e;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *kernel_ms = timed ? sum / timed : 0.0;
    Ctl c = read_ctl(s);
    return c.status & (DEM_ERR_CONTACT_OVERFLOW | DEM_ERR_NAN);
}

extern "C" int dem_stage1(dem_solver *s) {
    if (!s) return DEM_ERR_INVALID;
    dem_ctx *ctx = s->ctx;
    launch_stage(s->p->P, s->p->ctl, s->fc, 1, ctx->stream);
    CK(cudaGetLastError());
    return DEM_OK;
}
extern "C" int dem_stage2(dem_solver *s) {
    if (!s) return DEM_ERR_INVALID;
    dem_ctx *ctx = s->ctx;
    launch_stage(s->p->P, s->p->ctl, s->fc, 2, ctx->stream);
    k_invalidate<<<1, 32, 0, ctx->stream>>>(s->p->ctl);
    CK(cudaGetLastError());
    return DEM_OK;
}
extern "C" int dem_stage3(dem_solver *s) {
    if (!s) return DEM_ERR_INVALID;
    dem_ctx *ctx = s->ctx;
    launch_stage(s->p->P, s->p->ctl, s->fc, 3, ctx->stream);
    CK(cudaGetLastError());
    return DEM_OK;
}
extern "C" int dem_build_neighbors(dem_solver *s) {
    if (!s) return DEM_ERR_INVALID;
    if (s->p->mat_dirty || (s->p->P.ext != nullptr) != (s->fc.has_ext != 0)) {
        int st = prepare(s);
        if (st) return st;
    }
    int st = build_now(s, false);
    if (st) return st;
    return DEM_OK;
}
extern "C" int dem_solver_set_timestep(dem_solver *s, double dt) {
    if (!s || !(dt > 0.0)) return DEM_ERR_INVALID;
    if (dt == s->sp.dt) return DEM_OK;
    s->sp.dt = dt;
    s->fc.dt = dt;
    s->fc.half_dt = 0.5 * dt;   // Integrator.hpp:25
    s->version++;               // captured graphs hold the old step constants
    return DEM_OK;
}
extern "C" int dem_solver_rebuild(dem_solver *s) {
    if (!s) return DEM_ERR_INVALID;
    if (s->p->mat_dirty || (s->p->P.ext != nullptr) != (s->fc.has_ext != 0)) {
        int st = prepare(s);
        if (st) return st;
    }
    return build_now(s, true);
}
extern "C" int dem_compute_force(dem_solver *s) {
    if (!s) return DEM_ERR_INVALID;
    dem_ctx *ctx = s->ctx;
    if (s->p->mat_dirty || (s->p->P.ext != nullptr) != (s->fc.has_ext != 0)) {
        int st = prepare(s);
        if (st) return st;
    }
    {
        const int wst = check_walls(s);
        if (wst) return wst;
    }
    if (!s->built) return fail(ctx, DEM_ERR_INVALID, "dem_compute_force: build the neighbour list first");
    launch_step(s->p->P, s->L, s->p->ctl, s->fc, s->d_pp, s->d_pw, s->d_walls, MODE_FORCE_ONLY, ctx->stream);
    CK(cudaGetLastError());
    Ctl c = read_ctl(s);
    return c.status & (DEM_ERR_CONTACT_OVERFLOW | DEM_ERR_NAN);
}

extern "C" int dem_neighbors_get(dem_solver *s, int *offsets, int *idx, long *total) {
    if (!s || !offsets) return DEM_ERR_INVALID;
    dem_ctx *ctx = s->ctx;
    const int n = s->p->P.n, cap = s->p->P.cap, mb = s->L.maxnb;
    std::vector<int> nn(n), li((size_t)mb * cap), perm(n), rank(n);
    cudaStream_t st = ctx->stream;
    CK(cudaMemcpyAsync(nn.data(), s->L.nn, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(li.data(), s->L.idx, sizeof(int) * li.size(), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(perm.data(), s->p->P.perm, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(rank.data(), s->p->P.rank, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    offsets[0] = 0;
    for (int c = 0; c < n; ++c) offsets[c + 1] = offsets[c] + nn[rank[c]];
    if (total) *total = offsets[n];
    if (idx)
        for (int c = 0; c < n; ++c) {
            const int p = rank[c];
            for (int k = 0; k < nn[p]; ++k) idx[offsets[c] + k] = perm[li[(size_t)k * cap + p]];
        }
    return DEM_OK;
}

extern "C" int dem_energy(dem_solver *s, double out[4]) {
    if (!s || !out) return DEM_ERR_INVALID;
    dem_ctx *ctx = s->ctx;
    launch_energy(s->p->P, s->L, s->p->ctl, s->fc, s->d_pp, s->d_pw, s->d_walls, s->d_epart, s->nparts, s->d_eout,
                  ctx->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, s->d_eout, 4 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return DEM_OK;
}

// ---- bonded DEM ---------------------------------------------------------------------
extern "C" int dem_bonds_create(dem_solver *s, int max_bonds, const dem_bond_params *bp, dem_bonds **out) {
    if (!s || !bp || !out || max_bonds <= 0 || max_bonds > 64) return DEM_ERR_INVALID;
    dem_ctx *ctx = s->ctx;
    dem_bonds *b = new dem_bonds();
    b->s = s;
    const int cap = s->p->P.cap;
    Bonds &B = b->B;
    B.mb = max_bonds;
    B.cap = cap;
    cudaError_t e = cudaSuccess;
    auto A = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
    A(dalloc(&B.idx, (size_t)max_bonds * cap));
    A(dalloc(&B.init_len, (size_t)max_bonds * cap));
    A(dalloc(&B.count, cap));
    const bool mixed = s->sp.precision == DEM_MIXED;   // FP32 bond force/moment history
    B.hist = nullptr;
    B.hist32 = nullptr;
    if (mixed) A(dalloc(&B.hist32, 9 * (size_t)max_bonds * cap));
    else A(dalloc(&B.hist, 9 * (size_t)max_bonds * cap));
    A(dalloc(&B.broken, (size_t)max_bonds * cap));
    A(dalloc(&B.E, cap));
    A(dalloc(&B.G, cap));
    A(dalloc(&b->d_count, 1));
    if (e != cudaSuccess) {
        dem_bonds_destroy(b);
        return cuda_check(ctx, e, "dem_bonds_create");
    }
    cudaStream_t st = ctx->stream;
    k_fill_i<<<kGS, kTB, 0, st>>>(B.idx, (long)max_bonds * cap, -1);
    cudaMemsetAsync(B.init_len, 0, sizeof(double) * max_bonds * (size_t)cap, st);
    cudaMemsetAsync(B.count, 0, sizeof(int) * cap, st);
    if (B.hist) cudaMemsetAsync(B.hist, 0, sizeof(double) * 9 * max_bonds * (size_t)cap, st);
    if (B.hist32) cudaMemsetAsync(B.hist32, 0, sizeof(float) * 9 * max_bonds * (size_t)cap, st);
    cudaMemsetAsync(B.broken, 0, (size_t)max_bonds * cap, st);
    b->bc.quirks = bp->quirks;
    b->bc.beta = bp->beta;
    b->bc.radius_factor = bp->radius_factor;
    b->bc.kn = bp->kn;
    b->bc.kt = bp->kt;
    b->bc.break_strain = bp->break_strain;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    *out = b;
    return DEM_OK;
}

extern "C" int dem_bonds_destroy(dem_bonds *b) {
    if (!b) return DEM_ERR_INVALID;
    cudaStreamSynchronize(b->s->ctx->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    Bonds &B = b->B;
    cudaFree(B.idx); cudaFree(B.init_len); cudaFree(B.count); cudaFree(B.hist); cudaFree(B.hist32); cudaFree(B.broken);
    cudaFree(B.E); cudaFree(B.G); cudaFree(b->d_count);
    delete b;
    return DEM_OK;
}

extern "C" int dem_bonds_setup(dem_bonds *b, double factor, double search_cutoff) {
    if (!b || !(factor > 0.0)) return DEM_ERR_INVALID;
    dem_solver *s = b->s;
    dem_ctx *ctx = s->ctx;
    dem_particles *p = s->p;
    if (p->mat_dirty || (p->P.ext != nullptr) != (s->fc.has_ext != 0)) {
        int st = prepare(s);
        if (st) return st;
    }
    if (!(search_cutoff > 0.0)) search_cutoff = factor * p->rmax;
    int st = build_with(s, true, search_cutoff, 0.0);
    if (st) return st;
    cudaStream_t cs = ctx->stream;
    launch_bond_setup(p->P, s->L, b->B, p->ctl, factor, cs);
    // per-particle moduli in the (now fixed) particle order
    double *tmp = nullptr;
    const int n = p->P.n;
    CK(cudaMalloc(&tmp, sizeof(double) * n));
    CK(cudaMemcpyAsync(tmp, p->E.data(), sizeof(double) * n, cudaMemcpyHostToDevice, cs));
    k_scatter_d<<<kGS, kTB, 0, cs>>>(tmp, b->B.E, n, 1, p->P.cap, p->P.rank);
    CK(cudaStreamSynchronize(cs));
    CK(cudaMemcpyAsync(tmp, p->G.data(), sizeof(double) * n, cudaMemcpyHostToDevice, cs));
    k_scatter_d<<<kGS, kTB, 0, cs>>>(tmp, b->B.G, n, 1, p->P.cap, p->P.rank);
    CK(cudaStreamSynchronize(cs));
    cudaFree(tmp);
    CK(cudaGetLastError());
    p->has_bonds = true;
    s->built = false;   // the list was built with the bond search cutoff
    b->set_up = true;
    Ctl c = read_ctl(s);
    return c.status & DEM_ERR_BOND_OVERFLOW;
}

extern "C" int dem_bonds_get(dem_bonds *b, int field, void *host, long count) {
    if (!b || !host) return DEM_ERR_INVALID;
    dem_solver *s = b->s;
    dem_ctx *ctx = s->ctx;
    const Particles &P = s->p->P;
    const Bonds &B = b->B;
    const int n = P.n, mb = B.mb;
    const long per = (field == DEM_B_COUNT) ? n : (long)n * mb;
    const int es = (field == DEM_B_IDX || field == DEM_B_COUNT) ? 4 : (field == DEM_B_BROKEN ? 1 : 8);
    if (field < DEM_B_IDX || field > DEM_B_BROKEN || count != per)
        return fail(ctx, DEM_ERR_INVALID, "dem_bonds_get: unknown field or wrong element count");
    cudaStream_t st = ctx->stream;
    void *tmp = nullptr;
    CK(cudaMalloc(&tmp, (size_t)per * es));
    switch (field) {
        case DEM_B_IDX: k_gather_i<<<kGS, kTB, 0, st>>>(B.idx, (int *)tmp, n, mb, P.cap, P.rank, P.perm, 1); break;
        case DEM_B_INIT_LEN: k_gather_d<<<kGS, kTB, 0, st>>>(B.init_len, (double *)tmp, n, mb, P.cap, P.rank); break;
        case DEM_B_COUNT: k_gather_i<<<kGS, kTB, 0, st>>>(B.count, (int *)tmp, n, 1, P.cap, P.rank, P.perm, 0); break;
        case DEM_B_BROKEN: k_gather_u8n<<<kGS, kTB, 0, st>>>(B.broken, (uint8_t *)tmp, n, mb, P.cap, P.rank); break;
        default:
            if (B.hist32)
                k_gather_f2d<<<kGS, kTB, 0, st>>>(B.hist32 + (long)(field - DEM_B_FT_X) * mb * P.cap, (double *)tmp, n,
                                                  mb, P.cap, P.rank);
            else
                k_gather_d<<<kGS, kTB, 0, st>>>(B.hist + (long)(field - DEM_B_FT_X) * mb * P.cap, (double *)tmp, n, mb,
                                               P.cap, P.rank);
    }
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, tmp, (size_t)per * es, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(tmp);
    CK(e);
    return DEM_OK;
}

extern "C" int dem_bonds_set(dem_bonds *b, int field, const void *host, long count) {
    if (!b || !host) return DEM_ERR_INVALID;
    dem_solver *s = b->s;
    dem_ctx *ctx = s->ctx;
    const Particles &P = s->p->P;
    const Bonds &B = b->B;
    const int n = P.n, mb = B.mb;
    const long per = (field == DEM_B_COUNT) ? n : (long)n * mb;
    const int es = (field == DEM_B_IDX || field == DEM_B_COUNT) ? 4 : (field == DEM_B_BROKEN ? 1 : 8);
    if (field < DEM_B_IDX || field > DEM_B_BROKEN || count != per)
        return fail(ctx, DEM_ERR_INVALID, "dem_bonds_set: unknown field or wrong element count");
    if (field == DEM_B_IDX || field == DEM_B_COUNT) {
        const int *v = static_cast<const int *>(host);
        for (long t = 0; t < per; ++t) {
            const bool ok = field == DEM_B_IDX ? (v[t] >= -1 && v[t] < n) : (v[t] >= 0 && v[t] <= mb);
            if (!ok) return fail(ctx, DEM_ERR_INVALID, "dem_bonds_set: bond partner or count out of range");
        }
    }
    cudaStream_t st = ctx->stream;
    void *tmp = nullptr;
    CK(cudaMalloc(&tmp, (size_t)per * es));
    {
        const cudaError_t e = cudaMemcpyAsync(tmp, host, (size_t)per * es, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) {
            cudaFree(tmp);
            return cuda_check(ctx, e, "dem_bonds_set");
        }
    }
    switch (field) {
        case DEM_B_IDX: k_scatter_i<<<kGS, kTB, 0, st>>>((const int *)tmp, B.idx, n, mb, P.cap, P.rank, 1); break;
        case DEM_B_INIT_LEN: k_scatter_d<<<kGS, kTB, 0, st>>>((const double *)tmp, B.init_len, n, mb, P.cap, P.rank); break;
        case DEM_B_COUNT: k_scatter_i<<<kGS, kTB, 0, st>>>((const int *)tmp, B.count, n, 1, P.cap, P.rank, 0); break;
        case DEM_B_BROKEN: k_scatter_u8n<<<kGS, kTB, 0, st>>>((const uint8_t *)tmp, B.broken, n, mb, P.cap, P.rank); break;
        default:
            if (B.hist32)
                k_scatter_d2f<<<kGS, kTB, 0, st>>>((const double *)tmp, B.hist32 + (long)(field - DEM_B_FT_X) * mb * P.cap,
                                                   n, mb, P.cap, P.rank);
            else
                k_scatter_d<<<kGS, kTB, 0, st>>>((const double *)tmp, B.hist + (long)(field - DEM_B_FT_X) * mb * P.cap, n,
                                                 mb, P.cap, P.rank);
    }
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(tmp);
    CK(e);
    if (field == DEM_B_IDX || field == DEM_B_COUNT) {
        // bonds given by the caller define the particle order from now on, as setupBonds does
        s->p->has_bonds = true;
        b->set_up = true;
    }
    return DEM_OK;
}

extern "C" int dem_bonded_reset(dem_bonds *b) {
    if (!b) return DEM_ERR_INVALID;
    dem_ctx *ctx = b->s->ctx;
    const Particles &P = b->s->p->P;
    cudaStream_t st = b->s->ctx->stream;
    CK(cudaMemsetAsync(P.force, 0, sizeof(double) * 3 * (size_t)P.cap, st));
    CK(cudaMemsetAsync(P.torque, 0, sizeof(double) * 3 * (size_t)P.cap, st));
    return DEM_OK;
}

extern "C" int dem_apply_external_force(dem_solver *s) {
    if (!s) return DEM_ERR_INVALID;
    dem_ctx *ctx = s->ctx;
    launch_add_ext_force(s->p->P, s->ctx->stream);
    CK(cudaGetLastError());
    return DEM_OK;
}

extern "C" int dem_bonded_force(dem_bonds *b, double dt) {
    if (!b || !(dt > 0.0)) return DEM_ERR_INVALID;
    dem_solver *s = b->s;
    dem_ctx *ctx = s->ctx;
    if (!b->set_up) return fail(ctx, DEM_ERR_INVALID, "dem_bonded_force: call dem_bonds_setup first");
    if (s->p->mat_dirty) {
        int st = prepare(s);
        if (st) return st;
    }
    launch_bond_force(s->p->P, b->B, s->p->ctl, b->bc, dt, ctx->stream);
    CK(cudaGetLastError());
    int status = 0;
    CK(cudaMemcpyAsync(&status, &s->p->ctl->status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return status & (DEM_ERR_BOND_OVERFLOW | DEM_ERR_NAN);
}

extern "C" int dem_apply_boundary_conditions(dem_solver *s) {
    if (!s) return DEM_ERR_INVALID;
    if (s->p->mat_dirty || (s->p->P.ext != nullptr) != (s->fc.has_ext != 0)) {
        int st = prepare(s);
        if (st) return st;
    }
    dem_ctx *ctx = s->ctx;
    launch_post_hooks(s->p->P, s->fc, ctx->stream);
    CK(cudaGetLastError());
    return DEM_OK;
}

extern "C" int dem_bonds_broken(dem_bonds *b, long *count) {
    if (!b || !count) return DEM_ERR_INVALID;
    dem_ctx *ctx = b->s->ctx;
    launch_bond_broken_count(b->B, b->s->p->P.n, b->d_count, ctx->stream);
    unsigned long long c = 0;
    CK(cudaMemcpyAsync(&c, b->d_count, sizeof(c), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    *count = (long)c;
    return DEM_OK;
}

extern "C" int dem_bonded_run(dem_bonds *b, int nsteps) {
    if (!b) return DEM_ERR_INVALID;
    if (nsteps <= 0) return DEM_OK;
    dem_solver *s = b->s;
    dem_ctx *ctx = s->ctx;
    if (!b->set_up) return fail(ctx, DEM_ERR_INVALID, "dem_bonded_run: call dem_bonds_setup first");
    if (s->p->mat_dirty || (s->p->P.ext != nullptr) != (s->fc.has_ext != 0)) {
        int st = prepare(s);
        if (st) return st;
    }
    cudaStream_t st = ctx->stream;
    // the bonded step reads no neighbour list: no displacement bound may stop it (an upload
    // marks the list stale with a bound of 1e300)
    k_run_begin<<<1, 32, 0, st>>>(s->p->ctl, nsteps, std::numeric_limits<double>::infinity());
    launch_prologue(s->p->P, s->p->ctl, s->fc, st);
    s->launches += 2;
    CK(cudaGetLastError());
    const int chunk = s->sp.steps_per_launch;
    if (!b->graph || b->graph_version != s->version || b->graph_steps != chunk) {
        if (b->graph) {
            cudaGraphExecDestroy(b->graph);
            b->graph = nullptr;
        }
        auto capture = [&]() -> cudaError_t {
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) return e;
            for (int k = 0; k < chunk; ++k) launch_bond_step(s->p->P, b->B, s->p->ctl, s->fc, b->bc, st);
            e = cudaStreamEndCapture(st, &g);
            if (e != cudaSuccess) return e;
            e = cudaGraphInstantiate(&b->graph, g, 0);
            cudaGraphDestroy(g);
            return e;
        };
        cudaError_t e = capture();
        if (e != cudaSuccess && s->fc.pdl) {   // dependent launches refused in a graph: without them
            (void)cudaGetLastError();
            s->no_overlap = true;
            s->fc.pdl = 0;
            e = capture();
        }
        CK(e);
        b->graph_steps = chunk;
        b->graph_version = s->version;
    }
    for (int guard = 0; guard < 4 * (nsteps / chunk + 4); ++guard) {
        CK(cudaGraphLaunch(b->graph, st));
        s->launches += chunk;
        Ctl c = read_ctl(s);
        if (c.steps_done >= c.target) return c.status & (DEM_ERR_BOND_OVERFLOW | DEM_ERR_NAN);
    }
    return fail(ctx, DEM_ERR_CUDA, "dem_bonded_run made no progress");
}

// ---- surrogate dense layers ---------------------------------------------------------
namespace {
int nn_prepare(dem_ctx *ctx, long part_floats) {
    if (!ctx->d_err) {
        CK(cudaMalloc(&ctx->d_err, sizeof(int)));
        CK(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
    }
    if (part_floats > ctx->nn_part_floats) {
        CK(cudaStreamSynchronize(ctx->stream));
        cudaFree(ctx->nn_part);
        ctx->nn_part = nullptr;
        ctx->nn_part_floats = 0;
        CK(cudaMalloc(&ctx->nn_part, sizeof(float) * (size_t)part_floats));
        ctx->nn_part_floats = part_floats;
    }
    return DEM_OK;
}

bool nn_args_ok(const dem_nn_mlp *m, long rows, const dem_nn_rows *src, int nsrc) {
    if (!m || !src || nsrc < 1 || nsrc > 3 || rows < 0) return false;
    int kin = 0;
    for (int k = 0; k < nsrc; ++k) {
        if (!src[k].data || src[k].width <= 0 || src[k].width % 8) return false;
        kin += src[k].width;
    }
    return kin == m->kin && m->w1t && m->w2t && m->b1 && m->b2;
}
}  // namespace

extern "C" int dem_nn_mlp_forward(dem_ctx *ctx, const dem_nn_mlp *m, long rows, const dem_nn_rows *src, int nsrc,
                                  const void *resid, void *out, float *out_f32, void *h1) {
    if (!ctx) return DEM_ERR_INVALID;
    if (!nn_args_ok(m, rows, src, nsrc))
        return fail(ctx, DEM_ERR_INVALID, "dem_nn_mlp_forward: bad layer description or sources");
    int st = nn_prepare(ctx, 0);
    if (st) return st;
    st = nn_mlp_forward(*m, rows, src, nsrc, resid, out, out_f32, h1, ctx->d_err, ctx->stream);
    if (st == DEM_ERR_UNSUPPORTED) return fail(ctx, st, "dem_nn_mlp_forward: unsupported (kin, nout)");
    if (st) return cuda_check(ctx, cudaGetLastError(), "dem_nn_mlp_forward");
    return DEM_OK;
}

extern "C" int dem_nn_mlp_backward(dem_ctx *ctx, const dem_nn_mlp *m, long rows, const dem_nn_rows *src, int nsrc,
                                   const void *dy, const void *h1, void *dz1, float *dx, float *g_w1t, float *g_b1,
                                   float *g_w2t, float *g_b2) {
    if (!ctx) return DEM_ERR_INVALID;
    if (!nn_args_ok(m, rows, src, nsrc) || !dy || !h1 || !dz1 || !g_w1t || !g_b1 || !g_w2t || !g_b2 ||
        (dx && !m->w1) || !m->w2)
        return fail(ctx, DEM_ERR_INVALID, "dem_nn_mlp_backward: bad arguments");
    int st = nn_prepare(ctx, nn_wgrad_scratch(m->kin, m->nout));
    if (st) return st;
    st = nn_mlp_backward(*m, rows, src, nsrc, dy, h1, dz1, dx, g_w1t, m->kin, g_b1, g_w2t, g_b2, ctx->nn_part,
                         ctx->d_err, ctx->stream);
    if (st == DEM_ERR_UNSUPPORTED) return fail(ctx, st, "dem_nn_mlp_backward: unsupported (kin, nout)");
    if (st) return cuda_check(ctx, cudaGetLastError(), "dem_nn_mlp_backward");
    return DEM_OK;
}

extern "C" int dem_nn_edge_forward(dem_ctx *ctx, long rows, const void *e, const void *pq, const int *recv,
                                   const int *send, const void *w1e_t, const float *b1, const void *w2t,
                                   const float *b2, void *out, void *h1, int form) {
    if (!ctx) return DEM_ERR_INVALID;
    if (rows < 0 || (rows > 0 && (!e || !pq || !recv || !send || !w1e_t || !b1 || !w2t || !b2 || !out)) ||
        (form != 0 && form != 1))
        return fail(ctx, DEM_ERR_INVALID, "dem_nn_edge_forward: bad arguments");
    int st = nn_prepare(ctx, 0);
    if (st) return st;
    st = nn_edge_forward(rows, e, pq, recv, send, w1e_t, b1, w2t, b2, out, h1, ctx->d_err, ctx->stream, form);
    if (st) return cuda_check(ctx, cudaGetLastError(), "dem_nn_edge_forward");
    return DEM_OK;
}

extern "C" int dem_solver_debug_stream_waits(dem_solver *s, int poll_limit, int drop_copies) {
    if (!s || poll_limit < 0) return DEM_ERR_INVALID;
    dem_ctx *ctx = s->ctx;
    s->fc.wait_polls = poll_limit;
    s->fc.drop_copies = drop_copies ? 1 : 0;
    s->version++;   // graphs are captured again with the new settings
    if (!drop_copies) k_clear_status<<<1, 32, 0, ctx->stream>>>(s->p->ctl, DEM_ERR_TIMEOUT);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    return DEM_OK;
}

extern "C" int dem_nn_debug_waits(dem_ctx *ctx, int poll_limit, int drop_mma) {
    if (!ctx || poll_limit < 0) return DEM_ERR_INVALID;
    const int st = nn_debug_waits(poll_limit, drop_mma, ctx->stream);
    if (st) return fail(ctx, st, "dem_nn_debug_waits: cannot set the wait bounds");
    return DEM_OK;
}

extern "C" int dem_nn_status(dem_ctx *ctx, int *status) {
    if (!ctx || !status) return DEM_ERR_INVALID;
    *status = 0;
    if (!ctx->d_err) return DEM_OK;
    CK(cudaMemcpyAsync(status, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return DEM_OK;
}

// ---- internal access for the surrogate (dem_surrogate.cu) ---------------------------
namespace b200dem {
int solver_view(dem_solver *s, SolverView *v) {
    if (!s || !v) return DEM_ERR_INVALID;
    v->P = s->p->P;
    v->ctl = s->p->ctl;
    v->stream = s->ctx->stream;
    v->dt = s->sp.dt;
    v->ctx = s->ctx;
    return DEM_OK;
}
void solver_particles_changed(dem_solver *s) {
    s->p->dirty = true;
    s->built = false;
}
cudaStream_t ctx_stream(dem_ctx *ctx) { return ctx->stream; }
int ctx_fail(dem_ctx *ctx, int code, const char *msg) { return fail(ctx, code, msg); }
int ctx_cuda(dem_ctx *ctx, cudaError_t e, const char *what) { return cuda_check(ctx, e, what); }
int ctx_nn_scratch(dem_ctx *ctx, long part_floats, int **err, float **part) {
    const int st = nn_prepare(ctx, part_floats);
    *err = ctx->d_err;
    *part = ctx->nn_part;
    return st;
}
}  // namespace b200dem

// ---- checkpoint: every particle field in caller order ---------------------------------
// File: "B200DEMC", u32 version 1, i32 n, MaxCnts, MaxNoWalls, i32 field count, then per
// field i32 id, i64 bytes, data.  Fields that were never set (external force, scene) are
// left out.
extern "C" int dem_checkpoint_save(dem_particles *p, const char *path) {
    if (!p || !path) return DEM_ERR_INVALID;
    dem_ctx *ctx = p->ctx;
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(ctx, DEM_ERR_INVALID, std::string("dem_checkpoint_save: cannot open ") + path);
    std::vector<int> fields;
    for (int fld = 0; fld < DEM_F_COUNT_; ++fld) {
        if (fld == DEM_F_EXT_FORCE && !p->P.ext) continue;
        if (fld == DEM_F_SCENE && !p->P.scene) continue;
        fields.push_back(fld);
    }
    const uint32_t version = 1;
    const int hdr[4] = {p->P.n, p->P.mc, p->P.mw, (int)fields.size()};
    bool ok = std::fwrite("B200DEMC", 1, 8, f) == 8 && std::fwrite(&version, 4, 1, f) == 1 &&
              std::fwrite(hdr, 4, 4, f) == 4;
    std::vector<unsigned char> buf;
    for (int fld : fields) {
        if (!ok) break;
        long count;
        int es;
        field_layout(p, fld, &count, &es);
        buf.resize((size_t)count * es);
        const int st = dem_particles_get(p, fld, buf.data(), count);
        if (st) {
            std::fclose(f);
            return st;
        }
        const long long bytes = (long long)buf.size();
        ok = std::fwrite(&fld, 4, 1, f) == 1 && std::fwrite(&bytes, 8, 1, f) == 1 &&
             std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? DEM_OK : fail(ctx, DEM_ERR_INVALID, "dem_checkpoint_save: write failed");
}

extern "C" int dem_checkpoint_load(dem_particles *p, const char *path) {
    if (!p || !path) return DEM_ERR_INVALID;
    dem_ctx *ctx = p->ctx;
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(ctx, DEM_ERR_INVALID, std::string("dem_checkpoint_load: cannot open ") + path);
    char magic[8];
    uint32_t version = 0;
    int hdr[4];
    auto bad = [&](const char *why) {
        std::fclose(f);
        return fail(ctx, DEM_ERR_INVALID, std::string("dem_checkpoint_load: ") + why);
    };
    if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, "B200DEMC", 8) != 0) return bad("not a checkpoint");
    if (std::fread(&version, 4, 1, f) != 1 || version != 1) return bad("unknown version");
    if (std::fread(hdr, 4, 4, f) != 4) return bad("truncated header");
    if (hdr[0] != p->P.n || hdr[1] != p->P.mc || hdr[2] != p->P.mw)
        return bad("particle count, MaxCnts or MaxNoWalls differ from the particles object");
    if (hdr[3] < 0 || hdr[3] > DEM_F_COUNT_) return bad("bad field count");
    // read and check every field first, then apply them all: a truncated or mismatched file
    // leaves the particles object as it was
    struct Field {
        int fld;
        long count;
        std::vector<unsigned char> data;
    };
    std::vector<Field> fields((size_t)hdr[3]);
    for (Field &F : fields) {
        long long bytes;
        if (std::fread(&F.fld, 4, 1, f) != 1 || std::fread(&bytes, 8, 1, f) != 1) return bad("truncated field header");
        int es;
        if (!field_layout(p, F.fld, &F.count, &es) || bytes != (long long)F.count * es) return bad("field size mismatch");
        F.data.resize((size_t)bytes);
        if (std::fread(F.data.data(), 1, F.data.size(), f) != F.data.size()) return bad("truncated field");
    }
    std::fclose(f);
    for (const Field &F : fields) {
        const int st = dem_particles_set(p, F.fld, F.data.data(), F.count);
        if (st) return st;
    }
    return DEM_OK;
}
