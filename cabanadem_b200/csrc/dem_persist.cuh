// dem_persist.cuh -- the step loop of a small system in one cooperative launch.
//
// Below a few tens of thousands of particles the one-kernel step (k_contact_all) takes a few
// microseconds, about what a kernel launch and the step's last-block finalisation cost on top.
// k_steps_coop runs a run's steps inside one launch with every block resident (cooperative
// launch): per step, the same per-particle body as k_contact_all (particle_full,
// MODE_FUSED_DIRECT: positions and velocities to the other buffers), the same finalisation by
// the last block to take the step's ticket (finish_step_counted's arithmetic: displacement
// bound, buffer flips, step counters, contact count), and then a grid barrier: the finalising
// block publishes a generation count with a release store and the other blocks wait for it with
// acquire loads, a bounded number of polls.  The next step's gate is read after the barrier,
// so every block takes the same decision: the launch ends at the run's target, when the list
// goes stale (the host rebuilds and launches again), or on a stop bit.  A wait that gives up
// sets DEM_ERR_TIMEOUT and ends that block's loop; every other block then stops at its next
// gate or gives up the same way, so the launch always ends.  Same results as the per-step
// kernels, bit for bit.
//
// Included by dem_step.cu (FP64, no contraction) and dem_mixed.cu (mixed precision).
#pragma once
#include "dem_particle.cuh"

namespace b200dem {
namespace {

constexpr int kCoopWaitPolls = 1 << 22;   // polls of the generation word per step barrier

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// finish_step_counted followed by the grid barrier of the cooperative loop.  `gen` is the
// generation this block last saw; on return (true) every block has finished the step and the
// control word holds the finalised values, and gen is the new generation.
__device__ __forceinline__ bool finish_step_grid(Ctl *ctl, unsigned long long *slots, double vmax2, double dt,
                                                 int status, int active, const ForceConsts &fc, bool advance,
                                                 unsigned &gen) {
    __shared__ int cnt_s[32];
    __shared__ double red[32];
    __shared__ int am_last, ok_s;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int c = active;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    for (int o = 16; o > 0; o >>= 1) vmax2 = fmax(vmax2, __shfl_xor_sync(0xffffffffu, vmax2, o));
    if (status) atomicOr(&ctl->status, status);
    if (lane == 0) {
        cnt_s[warp] = c;
        red[warp] = vmax2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        double m = red[0];
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            t += cnt_s[w];
            m = fmax(m, red[w]);
        }
        if (t) atomicAdd(&ctl->ndefer, t);
        vmax_fold(slots, m);
        const unsigned tk = take_ticket(&ctl->ticket);
        am_last = (tk == gridDim.x - 1);
        ok_s = 1;
    }
    __syncthreads();
    if (am_last && threadIdx.x < 32) {
        const double v2 = fmax(vmax_collect_warp(slots), mesh_speed2(fc));
        if (advance) advance_kinematics(fc);   // not on the last step of a run (no next drift)
        __threadfence();   // each lane's wall and mesh positions, then the generation (thread 0)
        __syncwarp();
        if (threadIdx.x == 0) {
            ctl->disp = ctl->disp + dt * sqrt(v2) * (1.0 + 1e-9);
            ctl->last_ndefer = atomicAdd(&ctl->ndefer, 0);
            ctl->ndefer = 0;
            ctl->npairs = 0;
            ctl->cur ^= 1;
            ctl->vcur ^= 1;
            ctl->steps_done += 1;
            ctl->total_steps += 1;
            ctl->ticket = 0u;
            st_release_u32(&ctl->gen, gen + 1u);   // every write above before the generation
        }
    } else if (!am_last && threadIdx.x == 0) {
        int k = 0;
        while (ld_acquire_u32(&ctl->gen) == gen && k < kCoopWaitPolls) {
            __nanosleep(32);
            ++k;
        }
        if (k == kCoopWaitPolls) {
            atomicOr(&ctl->status, DEM_ERR_TIMEOUT);
            ok_s = 0;
        }
    }
    gen += 1u;
    __syncthreads();   // the block's other threads read the control word after thread 0's acquire
    return ok_s != 0;
}

template <bool MIXED, bool MESH>
__global__ void __launch_bounds__(kBlock) k_steps_coop(Particles P, NbrList L, Ctl *ctl, ForceConsts fc,
                                                       const PairConst *__restrict__ pp,
                                                       const PairConst *__restrict__ pw,
                                                       const WallGeom *__restrict__ walls, int max_steps) {
    unsigned gen = ctl->gen;   // no block finalises a step before every block has read it
    for (int k = 0; k < max_steps; ++k) {
        const CtlSnap c = read_ctl(ctl, true);
        if (!c.go) break;
        const int vcur = ctl->vcur;
        double vmax2 = 0.0;
        int status = 0, active = 0;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += gridDim.x * blockDim.x) {
            double v2 = 0.0;
            int a = 0;
            particle_full<MODE_FUSED_DIRECT, MIXED, MESH>(P, L, fc, pp, pw, walls, c.cur, c.cur ^ 1, vcur, c.last, i, i,
                                                          v2, status, &a);
            vmax2 = fmax(vmax2, v2);
            active += a;
        }
        if (!finish_step_grid(ctl, P.vslots, vmax2, fc.dt, status, active, fc, !c.last, gen)) break;
    }
}

// The same loop with static walls and no moving mesh, where nothing but the particles changes
// between steps: every block keeps the step counters, the buffer parity and the displacement
// bound itself, and the barrier is symmetric.  Per step each block stores its largest |u|^2
// and its in-contact count in its own slot (two sets of slots, by step parity), then arrives on
// one counter with a release atomic and polls it with acquire loads until every block has
// arrived (bounded); then one warp of each block reads the step's slots and every block computes
// the same bound, disp + dt sqrt(max |u|^2) (1 + 1e-9), as the finaliser does.  Two dependent
// round trips fewer per step than a ticket, a finaliser and its generation (the control word is
// read once at the start and written once at the end, by block 0).  scratch: the arrival
// counter (zeroed before the launch), then 2 x gridDim.x slots of |u|^2 bits and 2 x gridDim.x
// counts.
constexpr int kCoopMaxBlocks = kCoopMaxN / kBlock;

template <bool MIXED, bool MESH>
__global__ void __launch_bounds__(kBlock) k_steps_coop_lean(Particles P, NbrList L, Ctl *ctl, ForceConsts fc,
                                                            const PairConst *__restrict__ pp,
                                                            const PairConst *__restrict__ pw,
                                                            const WallGeom *__restrict__ walls, int max_steps,
                                                            unsigned long long *scratch) {
    __shared__ int s_cur, s_vcur, s_done, s_target, s_stop, s_ok, s_cnt;
    __shared__ double s_disp, s_half, s_v2;
    __shared__ int cnt_s[32];
    __shared__ double red[32];
    if (threadIdx.x == 0) {
        s_cur = ctl->cur;
        s_vcur = ctl->vcur;
        s_done = ctl->steps_done;
        s_target = ctl->target;
        s_stop = ctl->status & kStopBits;
        s_disp = ctl->disp;
        s_half = ctl->half_skin;
        s_ok = 1;
        s_cnt = 0;
    }
    __syncthreads();
    unsigned *arrive = reinterpret_cast<unsigned *>(scratch);
    unsigned long long *vslot = scratch + 1, *cslot = scratch + 1 + 2 * gridDim.x;
    const int G = gridDim.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int cur = s_cur, vcur = s_vcur, done = s_done;
    const int target = s_target;
    double disp = s_disp;
    const double half = s_half;
    int steps = 0;
    // the arrival count of step k is G (k + 1): at most 2^31 - 1 in one launch (the host
    // launches again for the steps left)
    const int kmax = max_steps < (int)(0x7FFFFFFFu / (unsigned)G) ? max_steps : (int)(0x7FFFFFFFu / (unsigned)G);
    for (int k = 0; k < kmax; ++k) {
        if (!(done < target && !s_stop && disp < half && s_ok)) break;   // the same in every block
        const int last = done + 1 >= target;
        double vmax2 = 0.0;
        int status = 0, active = 0;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += gridDim.x * blockDim.x) {
            double v2 = 0.0;
            int a = 0;
            particle_full<MODE_FUSED_DIRECT, MIXED, MESH>(P, L, fc, pp, pw, walls, cur, cur ^ 1, vcur, last, i, i, v2,
                                                          status, &a);
            vmax2 = fmax(vmax2, v2);
            active += a;
        }
        int c = active;
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        for (int o = 16; o > 0; o >>= 1) vmax2 = fmax(vmax2, __shfl_xor_sync(0xffffffffu, vmax2, o));
        if (status) atomicOr(&ctl->status, status);
        if (lane == 0) {
            cnt_s[warp] = c;
            red[warp] = vmax2;
        }
        __syncthreads();
        const int par = (k & 1) * G;
        if (threadIdx.x == 0) {
            int t = 0;
            double m = red[0];
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
                t += cnt_s[w];
                m = fmax(m, red[w]);
            }
            vslot[par + blockIdx.x] = (unsigned long long)__double_as_longlong(m);
            cslot[par + blockIdx.x] = (unsigned long long)t;
            unsigned old;   // the slots before the arrival
            asm volatile("atom.release.gpu.global.add.u32 %0, [%1], 1;" : "=r"(old) : "l"(arrive) : "memory");
            const unsigned want = (unsigned)G * (unsigned)(k + 1);
            int n = 0;
            while (ld_acquire_u32(arrive) < want && n < kCoopWaitPolls) {
                __nanosleep(32);
                ++n;
            }
            if (n == kCoopWaitPolls) {
                atomicOr(&ctl->status, DEM_ERR_TIMEOUT);
                s_ok = 0;
            }
        }
        __syncthreads();   // every block has arrived (or this one gave up): the slots are complete
        if (!s_ok) break;
        if (warp == 0) {   // every block's slots of this step, read by one warp after thread 0's acquire
            unsigned long long v = 0ull, n = 0ull;
            for (int b = lane; b < G; b += 32) {
                const unsigned long long x = *reinterpret_cast<volatile unsigned long long *>(vslot + par + b);
                v = x > v ? x : v;
                n += *reinterpret_cast<volatile unsigned long long *>(cslot + par + b);
            }
            for (int o = 16; o > 0; o >>= 1) {
                const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
                v = w > v ? w : v;
                n += __shfl_xor_sync(0xffffffffu, n, o);
            }
            if (lane == 0) {
                s_v2 = __longlong_as_double((long long)v);
                s_cnt = (int)n;
            }
        }
        __syncthreads();
        disp = disp + fc.dt * sqrt(s_v2) * (1.0 + 1e-9);
        cur ^= 1;
        vcur ^= 1;
        done += 1;
        steps += 1;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {   // the control word as the per-step finaliser leaves it
        ctl->cur = cur;
        ctl->vcur = vcur;
        ctl->steps_done = done;
        ctl->total_steps += steps;
        ctl->disp = disp;
        if (steps > 0) ctl->last_ndefer = s_cnt;
        ctl->ndefer = 0;
        ctl->npairs = 0;
    }
}

}  // namespace
}  // namespace b200dem
