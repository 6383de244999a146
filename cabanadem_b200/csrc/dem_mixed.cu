// dem_mixed.cu -- mixed-precision contact kernels (built with FMA contraction).
//
// Same per-particle step as the FP64 path (dem_particle.cuh), instantiated with FP32
// normal/tangential force arithmetic: pair offset, distance and overlap are formed in FP64
// from the FP64 positions (the subtraction that cancels), then the Hertz/Mindlin forces,
// damping and Coulomb limit are evaluated in FP32; tangential history is accumulated and
// stored in FP64, per-particle force sums and the velocity-Verlet update stay FP64.  The
// streaming kernel (particles with no possible contact) is shared with the FP64 path.
#include "dem_particle.cuh"
#include "dem_contact_coop.cuh"
#include "dem_pairs.cuh"
#include "dem_persist.cuh"
#include "dem_scenes.cuh"

namespace b200dem {

namespace {

template <int MINB, bool MESH = false>
__global__ void __launch_bounds__(kBlock, MINB) k_contact_mixed(Particles P, NbrList L, Ctl *ctl, ForceConsts fc,
                                                          const PairConst *__restrict__ pp,
                                                          const PairConst *__restrict__ pw,
                                                          const WallGeom *__restrict__ walls) {
    grid_dep_wait();   // launched as a dependent (launch_k): the kernel before has completed
    grid_dep_release();
    if (ctl->steps_done >= ctl->target || (ctl->status & kStopBits) || !(ctl->disp < ctl->half_skin))
        return;
    const int nd = ctl->ndefer;
    if ((long)blockIdx.x * blockDim.x >= nd) return;
    const int cur = ctl->cur, vcur = ctl->vcur;
    const int last = ctl->steps_done + 1 >= ctl->target;
    double vmax2 = 0.0;
    int status = 0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nd; t += gridDim.x * blockDim.x) {
        double v2 = 0.0;
        particle_full<MODE_FUSED, true, MESH>(P, L, fc, pp, pw, walls, cur, cur ^ 1, vcur, last, L.defer[t], t, v2,
                                              status);
        vmax2 = fmax(vmax2, v2);
    }
    block_vmax(ctl, P.vslots, vmax2, status);
}

// One-kernel dense step in mixed precision (see k_contact_all in dem_step.cu).
template <int MINB, bool MESH = false>
__global__ void __launch_bounds__(kBlock, MINB) k_contact_mixed_all(Particles P, NbrList L, Ctl *ctl, ForceConsts fc,
                                                              const PairConst *__restrict__ pp,
                                                              const PairConst *__restrict__ pw,
                                                              const WallGeom *__restrict__ walls) {
    grid_dep_wait();   // launched as a dependent (launch_k): the kernel before has completed
    grid_dep_release();
    const CtlSnap c = read_ctl(ctl, true);
    if (!c.go) return;
    const int vcur = ctl->vcur;
    double vmax2 = 0.0;
    int status = 0, active = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += gridDim.x * blockDim.x) {
        double v2 = 0.0;
        int a = 0;
        particle_full<MODE_FUSED_DIRECT, true, MESH>(P, L, fc, pp, pw, walls, c.cur, c.cur ^ 1, vcur, c.last, i, i, v2,
                                               status, &a);
        vmax2 = fmax(vmax2, v2);
        active += a;
    }
    finish_step_counted(ctl, P.vslots, vmax2, fc.dt, status, active, fc, !c.last);
}

template <bool MESH>
__global__ void __launch_bounds__(kBlock) k_force_mixed(Particles P, NbrList L, Ctl *ctl, ForceConsts fc,
                                                        const PairConst *__restrict__ pp,
                                                        const PairConst *__restrict__ pw,
                                                        const WallGeom *__restrict__ walls) {
    if (ctl->status & DEM_ERR_NEIGHBOR_OVERFLOW) return;
    const int cur = ctl->cur, vcur = ctl->vcur;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double vmax2 = 0.0;
    int status = 0;
    if (i < P.n)
        particle_full<MODE_FORCE_ONLY, true, MESH>(P, L, fc, pp, pw, walls, cur, cur ^ 1, vcur, 1, i, 0, vmax2, status);
    if (status) atomicOr(&ctl->status, status);
}

}  // namespace

template <bool MESH>
static void contact_mixed_t(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc, const PairConst *pp,
                            const PairConst *pw, const WallGeom *walls, int blocks, cudaStream_t s) {
    const bool dep = fc.pdl && fc.split != 3;   // not after the concurrent streaming branches' join
    if (fc.coop == 8)
        launch_k(k_contact_coop<8, kCoopMinBlocks, true, MESH>, blocks, kBlock, 0, s, dep, P, L, ctl, fc, pp, pw, walls);
    else if (fc.coop == 4)
        launch_k(k_contact_coop<4, kCoopMinBlocks, true, MESH>, blocks, kBlock, 0, s, dep, P, L, ctl, fc, pp, pw, walls);
    else if (fc.dense)
        launch_k(k_contact_mixed<kContactMixedMinBlocksDense, MESH>, blocks, kBlock, 0, s, dep, P, L, ctl, fc, pp, pw,
                 walls);
    else
        launch_k(k_contact_mixed<1, MESH>, blocks, kBlock, 0, s, dep, P, L, ctl, fc, pp, pw, walls);
}

void launch_contact_mixed(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc, const PairConst *pp,
                          const PairConst *pw, const WallGeom *walls, bool mesh, int blocks, cudaStream_t s) {
    if (mesh)
        contact_mixed_t<true>(P, L, ctl, fc, pp, pw, walls, blocks, s);
    else
        contact_mixed_t<false>(P, L, ctl, fc, pp, pw, walls, blocks, s);
}

void launch_contact_mixed_all(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc,
                              const PairConst *pp, const PairConst *pw, const WallGeom *walls, int blocks, bool mesh,
                              cudaStream_t s) {
    if (mesh)
        launch_k(k_contact_mixed_all<kContactMixedMinBlocksDense, true>, blocks, kBlock, 0, s, fc.pdl, P, L, ctl, fc, pp,
                 pw, walls);
    else
        launch_k(k_contact_mixed_all<kContactMixedMinBlocksDense, false>, blocks, kBlock, 0, s, fc.pdl, P, L, ctl, fc, pp,
                 pw, walls);
}

const void *contact_mixed_all_kernel(bool mesh) {
    return mesh ? (const void *)k_contact_mixed_all<kContactMixedMinBlocksDense, true>
                : (const void *)k_contact_mixed_all<kContactMixedMinBlocksDense, false>;
}

void launch_force_mixed(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc, const PairConst *pp,
                        const PairConst *pw, const WallGeom *walls, bool mesh, cudaStream_t s) {
    if (mesh)
        k_force_mixed<true><<<(P.n + kBlock - 1) / kBlock, kBlock, 0, s>>>(P, L, ctl, fc, pp, pw, walls);
    else
        k_force_mixed<false><<<(P.n + kBlock - 1) / kBlock, kBlock, 0, s>>>(P, L, ctl, fc, pp, pw, walls);
}

template <bool MESH>
static const void *contact_mixed_kernel_t(int dense, int coop) {
    if (coop == 8) return (const void *)k_contact_coop<8, kCoopMinBlocks, true, MESH>;
    if (coop == 4) return (const void *)k_contact_coop<4, kCoopMinBlocks, true, MESH>;
    return dense ? (const void *)k_contact_mixed<kContactMixedMinBlocksDense, MESH>
                 : (const void *)k_contact_mixed<1, MESH>;
}

// Every block the SMs hold of a kernel (a persistent grid), at most enough for `work` threads.
static int fill_blocks(const void *kernel, int block, long work) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, block, 0);
    if (per <= 0) per = 1;
    const long need = (work + block - 1) / block;
    return (int)(need < (long)sms * per ? (need > 0 ? need : 1) : (long)sms * per);
}

template <bool MESH>
static void pairs_mixed_t(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc, const PairConst *pp,
                          const PairConst *pw, const WallGeom *walls, cudaStream_t s) {
    static thread_local int g2 = 0, g3 = 0, sms = 0, last_n = -1;
    if (last_n != P.n) {
        g2 = fill_blocks((const void *)k_pairs_eval<true>, kPairsBlock, 8L * P.n);
        g3 = fill_blocks((const void *)k_pairs_sum<true, MESH>, kPairsBlock, P.n);
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
        last_n = P.n;
    }
    launch_pairs_find<true>(P, L, ctl, fc, walls, sms, s);
    launch_k(k_pairs_eval<true>, g2, kPairsBlock, 0, s, fc.pdl, P, L, ctl, fc, pp, pw, walls);
    launch_k(k_pairs_sum<true, MESH>, g3, kPairsBlock, 0, s, fc.pdl, P, L, ctl, fc);
}

void launch_pairs_mixed(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc, const PairConst *pp,
                        const PairConst *pw, const WallGeom *walls, bool mesh, cudaStream_t s) {
    if (mesh)
        pairs_mixed_t<true>(P, L, ctl, fc, pp, pw, walls, s);
    else
        pairs_mixed_t<false>(P, L, ctl, fc, pp, pw, walls, s);
}

const void *contact_mixed_kernel(int dense, int coop, bool mesh) {
    return mesh ? contact_mixed_kernel_t<true>(dense, coop) : contact_mixed_kernel_t<false>(dense, coop);
}

// Cooperative launch of the step loop (dem_persist.cuh): a grid-stride grid of at most the
// blocks the SMs hold at once.
// With static walls and no moving mesh the symmetric-barrier form (its arrival counter zeroed
// first on the stream).
template <bool MIXED, bool MESH>
static cudaError_t steps_coop_t(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc,
                                const PairConst *pp, const PairConst *pw, const WallGeom *walls, int max_steps,
                                unsigned long long *scratch, cudaStream_t s) {
    const bool lean = !fc.mwalls && !fc.mesh_moving && scratch;
    const void *kernel = lean ? (const void *)k_steps_coop_lean<MIXED, MESH> : (const void *)k_steps_coop<MIXED, MESH>;
    static thread_local int fit[2] = {0, 0};   // resident blocks of each form, per host thread
    if (!fit[lean]) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kBlock, 0);
        fit[lean] = (sms > 0 ? sms : 148) * (per > 0 ? per : 1);
    }
    const int need = (P.n + kBlock - 1) / kBlock;
    int grid = need < fit[lean] ? (need > 0 ? need : 1) : fit[lean];
    if (lean && grid > kCoopMaxBlocks) grid = kCoopMaxBlocks;   // the scratch holds that many slots
    Particles p = P;
    NbrList l = L;
    ForceConsts f = fc;
    if (!lean) {
        void *args[] = {&p, &l, &ctl, &f, (void *)&pp, (void *)&pw, (void *)&walls, &max_steps};
        return cudaLaunchCooperativeKernel(kernel, dim3(grid), dim3(kBlock), args, 0, s);
    }
    const cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    void *args[] = {&p, &l, &ctl, &f, (void *)&pp, (void *)&pw, (void *)&walls, &max_steps, &scratch};
    return cudaLaunchCooperativeKernel(kernel, dim3(grid), dim3(kBlock), args, 0, s);
}

cudaError_t launch_steps_coop_mixed(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc,
                                    const PairConst *pp, const PairConst *pw, const WallGeom *walls, int max_steps,
                                    unsigned long long *scratch, cudaStream_t s) {
    return fc.mesh.nt ? steps_coop_t<true, true>(P, L, ctl, fc, pp, pw, walls, max_steps, scratch, s)
                      : steps_coop_t<true, false>(P, L, ctl, fc, pp, pw, walls, max_steps, scratch, s);
}

void launch_scene_steps_mixed(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc,
                              const PairConst *pp, const PairConst *pw, const WallGeom *walls, const int2 *table,
                              int nscenes, int nsteps, double delta, double skin, cudaStream_t s) {
    const SceneSmem o = scene_smem(P.mc, P.mw, P.ext != nullptr, P.fix != nullptr, fc.nmat > 1);
    if (o.bytes <= kSceneSmemMax &&
        cudaFuncSetAttribute(k_scene_steps_smem<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, o.bytes) ==
            cudaSuccess)
        k_scene_steps_smem<true><<<nscenes, kSceneBlock, o.bytes, s>>>(P, L, ctl, fc, pp, pw, walls, table, nsteps,
                                                                       delta, skin);
    else
        k_scene_steps<true><<<nscenes, kSceneBlock, 0, s>>>(P, L, ctl, fc, pp, pw, walls, table, nsteps, delta, skin);
    k_scene_run_end<<<1, 32, 0, s>>>(ctl, nsteps);
}

}  // namespace b200dem
