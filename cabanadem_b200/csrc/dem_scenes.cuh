// dem_scenes.cuh -- batched small scenes in one persistent launch per run.
//
// Scenes never interact, and after a re-sorting build every scene occupies a contiguous range
// of the storage (the cell keys are scene-major).  k_scene_steps gives each scene a block of
// its own and runs all the steps of a run inside that one launch: per step, every particle
// lists the scene's particles within the list cutoff (r_i + r_j + skin, or delta) in
// ascending caller index, then takes the full step of the one-kernel form (particle_full:
// compaction, pair and wall laws, hooks, velocity Verlet; positions and velocities to the other
// buffers), and a block barrier separates the steps.  No step waits on another block, so the
// launch needs no grid barrier and no device-side wait.  The lists are rebuilt each step from
// positions of that step, a superset of the overlapping pairs summed in caller order as the
// Verlet list is, so the results are those of the other forms bit for bit.
//
// Included by dem_step.cu (FP64, no contraction) and dem_mixed.cu (mixed precision).
#pragma once
#include "dem_particle.cuh"

namespace b200dem {
namespace {

constexpr int kSceneBlock = kSceneMaxParticles;   // one thread per particle of a scene

// Scene table after a build that re-sorted without the class partition (cell order, scene-major
// keys): table[s] = (first storage index, count).  k_scene_bounds marks each scene's first and
// end index from its neighbours in storage; k_scene_check turns the end into a count and sets
// *bad unless it equals the scene's particle count (the scene is contiguous) and fits a block.
__global__ void k_scene_hist(const int *scene, int n, int *counts) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) atomicAdd(&counts[scene[i]], 1);
}
__global__ void k_scene_bounds(const int *scene, int n, int2 *table) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int s = scene[i];
        if (i == 0 || scene[i - 1] != s) table[s].x = i;
        if (i == n - 1 || scene[i + 1] != s) table[s].y = i + 1;
    }
}
__global__ void k_scene_check(int nscenes, int2 *table, const int *counts, int *bad) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nscenes; s += gridDim.x * blockDim.x) {
        const int2 t = table[s];
        const int c = counts[s] > 0 ? t.y - t.x : 0;
        if (c != counts[s] || c > kSceneBlock) atomicOr(bad, 1);
        table[s] = make_int2(counts[s] > 0 ? t.x : 0, c);
    }
}

template <bool MIXED>
__global__ void __launch_bounds__(kSceneBlock) k_scene_steps(Particles P, NbrList L, Ctl *ctl, ForceConsts fc,
                                                             const PairConst *__restrict__ pp,
                                                             const PairConst *__restrict__ pw,
                                                             const WallGeom *__restrict__ walls, const int2 *table,
                                                             int nsteps, double delta, double skin) {
    __shared__ int order[kSceneBlock];
    __shared__ D4 spos[kSceneBlock];   // the scene's positions of the step, for the list search
    const int2 sc = table[blockIdx.x];
    const int first = sc.x, count = sc.y, t = threadIdx.x, cap = P.cap;
    if (count <= 0) return;   // block-uniform
    // the scene's particles in ascending caller index (the order of every per-particle sum)
    if (t < count) {
        const int i = first + t, ki = P.perm[i];
        int r = 0;
        for (int u = 0; u < count; ++u) r += P.perm[first + u] < ki ? 1 : 0;
        order[r] = i;
    }
    int cur = ctl->cur, vcur = ctl->vcur;   // no other kernel runs during this launch
    int status = 0;
    for (int k = 0; k < nsteps; ++k) {
        __syncthreads();   // the previous step's positions and velocities (and `order`) are complete
        if (t < count) spos[t] = ld4(P.pos[cur], first + t);   // one load per particle, then shared
        __syncthreads();
        if (t < count) {
            const int i = first + t;
            const D4 pi = spos[t];
            int nn = 0;
            for (int r = 0; r < count; ++r) {
                const int j = order[r];
                if (j == i) continue;
                const D4 pj = spos[j - first];
                const double px = pi.x - pj.x, py = pi.y - pj.y, pz = pi.z - pj.z;
                const double r2 = px * px + py * py + pz * pz;
                const double cut = delta > 0.0 ? delta : pi.w + pj.w + skin;
                if (r2 <= cut * cut) {
                    if (nn < L.maxnb) L.idx[(long)nn * cap + i] = j;
                    else status |= DEM_ERR_NEIGHBOR_OVERFLOW;
                    ++nn;
                }
            }
            L.nn[i] = nn < L.maxnb ? nn : L.maxnb;
            double v2 = 0.0;
            int a = 0;
            particle_full<MODE_FUSED_DIRECT, MIXED, false>(P, L, fc, pp, pw, walls, cur, cur ^ 1, vcur,
                                                           k == nsteps - 1, i, i, v2, status, &a);
        }
        cur ^= 1;
        vcur ^= 1;
    }
    if (status) atomicOr(&ctl->status, status);
}

// The same launch with the whole scene in shared memory for the run: positions, velocities,
// spins (both buffers), mass and inertia, contact words, tracked slots and their history,
// wall history, force and torque, external force, fix flags, materials and the lists, copied
// in at the start and out at the end (partners renamed to and from scene-local indices).
// `particle_full` then runs on a particle set whose arrays are shared memory (generic loads),
// so a step's loads are shared-memory loads instead of a chain of global round trips.  The
// scene's lists are Verlet lists of its own: built at the first step with the solver's cutoff
// (r_i + r_j + skin, or delta) and again only once the block's displacement bound -- the sum
// over steps of dt max |u| in the scene, as the solver keeps it -- reaches half the margin
// (skin / 2, or (delta - 2 r_max) / 2 with the scene's largest radius); every pair in contact
// is then in the lists, in caller order.  Same arithmetic, same bits.
constexpr int kSceneSmemMax = 110 * 1024;   // a larger copy (many tracked slots) keeps the global form

struct SceneSmem {   // byte offsets of a scene's copy; kSceneBlock rows per field
    int pos, vel, omg, force, torque, mI, th, sw, ext, tidx, cstate, lidx, lnn, scene, mat, fix, bytes;
};
__host__ __device__ inline SceneSmem scene_smem(int mc, int mw, bool ext, bool fix, bool mat) {
    constexpr int S = kSceneBlock;
    SceneSmem o;
    int b = 0;
    o.pos = b;    b += 2 * S * 32;
    o.vel = b;    b += 2 * 3 * S * 8;
    o.omg = b;    b += 2 * 3 * S * 8;
    o.force = b;  b += 3 * S * 8;
    o.torque = b; b += 3 * S * 8;
    o.mI = b;     b += 2 * S * 8;
    o.th = b;     b += 3 * mc * S * 8;
    o.sw = b;     b += 3 * mw * S * 8;
    o.ext = b;    b += ext ? 3 * S * 8 : 0;
    o.tidx = b;   b += mc * S * 4;
    o.cstate = b; b += S * 4;
    o.lidx = b;   b += S * S * 4;
    o.lnn = b;    b += S * 4;
    o.scene = b;  b += S * 4;
    o.mat = b;    b += mat ? S : 0;
    o.fix = b;    b += fix ? S : 0;
    o.bytes = (b + 15) & ~15;
    return o;
}

template <bool MIXED>
__global__ void __launch_bounds__(kSceneBlock) k_scene_steps_smem(Particles P, NbrList L, Ctl *ctl, ForceConsts fc,
                                                                  const PairConst *__restrict__ pp,
                                                                  const PairConst *__restrict__ pw,
                                                                  const WallGeom *__restrict__ walls,
                                                                  const int2 *table, int nsteps, double delta,
                                                                  double skin) {
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ int order[kSceneBlock];
    constexpr int S = kSceneBlock;
    const int2 sc = table[blockIdx.x];
    const int first = sc.x, count = sc.y, t = threadIdx.x, cap = P.cap, mc = P.mc, mw = P.mw;
    if (count <= 0) return;   // block-uniform
    const bool has_mat = fc.nmat > 1;
    const SceneSmem o = scene_smem(mc, mw, P.ext != nullptr, P.fix != nullptr, has_mat);
    // the scene-local particle set: the same fields, kSceneBlock rows, arrays in shared memory
    Particles Q = P;
    Q.n = count;
    Q.cap = S;
    Q.pos[0] = reinterpret_cast<double4 *>(sm + o.pos);
    Q.pos[1] = Q.pos[0] + S;
    Q.vel[0] = reinterpret_cast<double *>(sm + o.vel);
    Q.vel[1] = Q.vel[0] + 3 * S;
    Q.omg[0] = reinterpret_cast<double *>(sm + o.omg);
    Q.omg[1] = Q.omg[0] + 3 * S;
    Q.force = reinterpret_cast<double *>(sm + o.force);
    Q.torque = reinterpret_cast<double *>(sm + o.torque);
    Q.mI = reinterpret_cast<double *>(sm + o.mI);
    Q.th = reinterpret_cast<double *>(sm + o.th);
    Q.sw = reinterpret_cast<double *>(sm + o.sw);
    Q.ext = P.ext ? reinterpret_cast<double *>(sm + o.ext) : nullptr;
    Q.tidx = reinterpret_cast<int *>(sm + o.tidx);
    Q.cstate = reinterpret_cast<int *>(sm + o.cstate);
    Q.scene = reinterpret_cast<int *>(sm + o.scene);
    Q.mat = has_mat ? sm + o.mat : P.mat;
    Q.fix = P.fix ? sm + o.fix : nullptr;
    Q.perm = nullptr;
    Q.rank = nullptr;
    NbrList M = L;
    M.idx = reinterpret_cast<int *>(sm + o.lidx);
    M.nn = reinterpret_cast<int *>(sm + o.lnn);
    M.maxnb = S;
    int cur = ctl->cur, vcur = ctl->vcur;   // no other kernel runs during this launch
    if (t < count) {   // copy in
        const int g = first + t;
        const D4 p = ld4(P.pos[cur], g);
        st4(Q.pos[cur], t, p);
        for (int d = 0; d < 3; ++d) {
            Q.vel[vcur][d * S + t] = P.vel[vcur][(long)d * cap + g];
            Q.omg[vcur][d * S + t] = P.omg[vcur][(long)d * cap + g];
            if (P.ext) Q.ext[d * S + t] = P.ext[(long)d * cap + g];
        }
        Q.mI[t] = P.mI[g];
        Q.mI[S + t] = P.mI[(long)cap + g];
        Q.cstate[t] = P.cstate[g];
        Q.scene[t] = P.scene[g];
        if (has_mat) Q.mat[t] = P.mat[g];
        if (P.fix) Q.fix[t] = P.fix[g];
        for (int s = 0; s < mc; ++s) {
            const int v = P.tidx[(long)s * cap + g];
            Q.tidx[s * S + t] = (v >= first && v < first + count) ? v - first : -1;
            for (int c = 0; c < 3; ++c) Q.th[(c * mc + s) * S + t] = P.th[((long)c * mc + s) * cap + g];
        }
        for (int w = 0; w < mw; ++w)
            for (int c = 0; c < 3; ++c) Q.sw[(c * mw + w) * S + t] = P.sw[((long)c * mw + w) * cap + g];
        // the scene's particles in ascending caller index (the order of every per-particle sum)
        const int ki = P.perm[g];
        int r = 0;
        for (int u = 0; u < count; ++u) r += P.perm[first + u] < ki ? 1 : 0;
        order[r] = t;
    }
    int status = 0;
    __shared__ double s_red[kSceneBlock / 32];
    __shared__ double s_half;
    __syncthreads();   // the copy-in and `order` are complete
    {   // the margin of the lists: skin / 2, or (delta - 2 r_max) / 2 with the scene's r_max
        double rm = t < count ? ld4(Q.pos[cur], t).w : 0.0;
        for (int o2 = 16; o2 > 0; o2 >>= 1) rm = fmax(rm, __shfl_xor_sync(0xffffffffu, rm, o2));
        if ((t & 31) == 0) s_red[t >> 5] = rm;
        __syncthreads();
        if (t == 0) {
            double m = 0.0;
            for (int w = 0; w < kSceneBlock / 32; ++w) m = fmax(m, s_red[w]);
            s_half = delta > 0.0 ? fmax(0.0, delta - 2.0 * m) / 2.0 : skin / 2.0;
        }
    }
    double disp = 1e300;   // displacement bound since the lists were built (none yet)
    for (int k = 0; k < nsteps; ++k) {
        __syncthreads();   // the previous step's state is complete
        const bool build = !(disp < s_half);   // the same in every thread
        if (build) disp = 0.0;
        if (t < count) {
            if (build) {
                const double4 *pc = Q.pos[cur];
                const D4 pi = ld4(pc, t);
                int nn = 0;
                for (int r = 0; r < count; ++r) {
                    const int j = order[r];
                    if (j == t) continue;
                    const D4 pj = ld4(pc, j);
                    const double px = pi.x - pj.x, py = pi.y - pj.y, pz = pi.z - pj.z;
                    const double r2 = px * px + py * py + pz * pz;
                    const double cut = delta > 0.0 ? delta : pi.w + pj.w + skin;
                    if (r2 <= cut * cut) M.idx[nn++ * S + t] = j;   // nn < count <= S
                }
                M.nn[t] = nn;
            }
        }
        double v2 = 0.0;
        if (t < count) {
            int a = 0;
            particle_full<MODE_FUSED_DIRECT, MIXED, false, false>(Q, M, fc, pp, pw, walls, cur, cur ^ 1, vcur,
                                                                  k == nsteps - 1, t, t, v2, status, &a);
        }
        // the block's largest |u|^2 of the drift: dt |u|max added to the bound, as the solver does
        for (int o2 = 16; o2 > 0; o2 >>= 1) v2 = fmax(v2, __shfl_xor_sync(0xffffffffu, v2, o2));
        if ((t & 31) == 0) s_red[t >> 5] = v2;
        __syncthreads();
        double m = s_red[0];
        for (int w = 1; w < kSceneBlock / 32; ++w) m = fmax(m, s_red[w]);
        disp = disp + fc.dt * sqrt(m) * (1.0 + 1e-9);
        cur ^= 1;
        vcur ^= 1;
    }
    __syncthreads();
    if (t < count) {   // copy out: the state the per-step kernels would have left
        const int g = first + t;
        st4(P.pos[cur], g, ld4(Q.pos[cur], t));
        for (int d = 0; d < 3; ++d) {
            P.vel[vcur][(long)d * cap + g] = Q.vel[vcur][d * S + t];
            P.omg[vcur][(long)d * cap + g] = Q.omg[vcur][d * S + t];
            if (nsteps > 0) {
                P.force[(long)d * cap + g] = Q.force[d * S + t];
                P.torque[(long)d * cap + g] = Q.torque[d * S + t];
            }
        }
        P.cstate[g] = Q.cstate[t];
        for (int s = 0; s < mc; ++s) {
            const int v = Q.tidx[s * S + t];
            P.tidx[(long)s * cap + g] = v >= 0 ? v + first : -1;
            for (int c = 0; c < 3; ++c) P.th[((long)c * mc + s) * cap + g] = Q.th[(c * mc + s) * S + t];
        }
        for (int w = 0; w < mw; ++w)
            for (int c = 0; c < 3; ++c) P.sw[((long)c * mw + w) * cap + g] = Q.sw[(c * mw + w) * S + t];
    }
    if (status) atomicOr(&ctl->status, status);
}

// After the launch: the buffer flips and step counts of its steps.
__global__ void k_scene_run_end(Ctl *ctl, int nsteps) {
    if (threadIdx.x == 0) {
        if (nsteps & 1) {
            ctl->cur ^= 1;
            ctl->vcur ^= 1;
        }
        ctl->steps_done += nsteps;
        ctl->total_steps += nsteps;
    }
}

}  // namespace
}  // namespace b200dem
