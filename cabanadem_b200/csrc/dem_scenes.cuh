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
