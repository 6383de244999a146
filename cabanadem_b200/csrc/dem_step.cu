// dem_step.cu -- FP64 contact step for sm_100a.  Built with --fmad=false: every
// expression keeps the reference's evaluation order, so results match the FP64
// oracle bit for bit (x^1.5 is evaluated as x*sqrt(x), |v| as sqrt).
//
// One thread per particle i (Morton-sorted order).  A fused launch does, for step n:
//   compact tracked contacts          src/CabanaDEM_Force.hpp:344-445
//   pp Hertz + Mindlin over the list  src/CabanaDEM_Force.hpp:50-341
//   particle-wall contact             src/CabanaDEM_Force.hpp:448-678
//   hooks (gravity, fix flags)        tst_01_BDEM:19-117 positions
//   stage3 of step n                  src/CabanaDEM_Integrator.hpp:77-102
//   stage1 + stage2 of step n+1       src/CabanaDEM_Integrator.hpp:31-74
// reading the current ping-pong buffer and writing the next, so that neighbours always
// see the positions and velocities of step n.  The sum over neighbours runs in
// ascending caller index (the list is sorted that way), the oracle's order.
#include "dem_internal.cuh"
#include "b200dem.h"

#include "dem_particle.cuh"
#include "dem_bulk.cuh"
#include "dem_contact_coop.cuh"
#include "dem_pairs.cuh"
#include "dem_persist.cuh"
#include "dem_scenes.cuh"

namespace b200dem {

// Unfused force pass (MODE_FORCE_ONLY): F and tau written in place.
template <bool MESH>
__global__ void __launch_bounds__(kBlock) k_force(Particles P, NbrList L, Ctl *ctl, ForceConsts fc,
                                                  const PairConst *__restrict__ pp, const PairConst *__restrict__ pw,
                                                  const WallGeom *__restrict__ walls) {
    if (ctl->status & DEM_ERR_NEIGHBOR_OVERFLOW) return;
    const int cur = ctl->cur, vcur = ctl->vcur;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double vmax2 = 0.0;
    int status = 0;
    if (i < P.n)
        particle_full<MODE_FORCE_ONLY, false, MESH>(P, L, fc, pp, pw, walls, cur, cur ^ 1, vcur, 1, i, 0, vmax2,
                                                    status);
    if (status) atomicOr(&ctl->status, status);
}

__device__ __forceinline__ bool step_gate(const Ctl *ctl) {
    return ctl->steps_done < ctl->target && !(ctl->status & kStopBits) && ctl->disp < ctl->half_skin;
}

// ---------------------------------------------------------------------------------------
// Fused step, kernel 1 of 3: streaming.  A particle with no tracked contact, no active wall
// history, no neighbour within r_i + r_j (1 + 5e-11) and no wall overlap has zero pair
// force and zero torque.  Its step is then: hooks, velocity half-kicks and drift -- done
// here with few registers so that the kernel runs at high occupancy.  Its angular
// velocity is unchanged (tau = 0), so omega is neither read nor written, and u is updated
// in place (no other thread reads the velocity of a particle without contacts: the pair
// terms that read a partner's velocity only run for overlapping pairs, and both partners
// of such a pair are deferred).  Positions still go to the next buffer because every
// neighbour reads them.  Every other particle is appended to L.defer for kernel 2.
// Each thread reads the control word itself (no block barrier before the work).
// ---------------------------------------------------------------------------------------

// Per-step values of the control word every streaming thread needs.
struct StreamCtl {
    int cur, vcur, nlone, nclear_end, n;
    bool last;
    bool wfar;   // the wall-gap flags of the last build hold (see k_wall_far)
};
__device__ __forceinline__ StreamCtl stream_ctl(const Ctl *ctl, int n) {
    StreamCtl c;
    c.cur = ctl->cur;
    c.vcur = ctl->vcur;
    c.nlone = ctl->nlone;
    // particles [nlone, nclear_end) had every listed neighbour at a gap above skin/2: while
    // twice the displacement bound stays below skin/2 none of them can touch
    c.nclear_end = (2.0 * ctl->disp < ctl->half_skin) ? c.nlone + ctl->nclear : c.nlone;
    c.wfar = ctl->wfar_build == ctl->rebuilds && 2.0 * ctl->disp < ctl->half_skin;
    c.last = ctl->steps_done + 1 >= ctl->target;
    c.n = n;
    return c;
}

// Appends the deferred lanes of a converged warp to L.defer (one atomic per warp).
__device__ __forceinline__ void defer_append(Ctl *ctl, const NbrList &L, bool defer, int i) {
    const unsigned dmask = __ballot_sync(0xffffffffu, defer);
    if (defer) {
        const int lane = threadIdx.x & 31;
        const int leader = __ffs(dmask) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(&ctl->ndefer, __popc(dmask));
        base = __shfl_sync(dmask, base, leader);
        L.defer[base + __popc(dmask & ((1u << lane) - 1u))] = i;
    }
}

// The step of particle i without pair force and torque: F = ext (added to zero), the
// post-force hooks, stage3 of this step and stage1 + stage2 of the next (u in place, x to the
// next buffer), or F and tau stored after the run's last step.
__device__ __forceinline__ void stream_free_step(const Particles &P, const ForceConsts &fc, const StreamCtl &c,
                                                 double *vc, int i, const D4 &pi, double m, double ui0, double ui1,
                                                 double ui2, double &vmax2) {
    const int cap = P.cap;
    double F0 = 0., F1 = 0., F2 = 0.;
    if (fc.has_ext) {
        F0 += P.ext[i];
        F1 += P.ext[cap + i];
        F2 += P.ext[2 * cap + i];
    }
    if (fc.has_gravity) {
        F0 += m * fc.g[0];
        F1 += m * fc.g[1];
        F2 += m * fc.g[2];
    }
    if (fc.has_fix && (P.fix[i] & DEM_FIX_FORCE)) F0 = F1 = F2 = 0.;
    const double m_inverse = 1. / m;
    const double h = fc.half_dt;
    ui0 += h * F0 * m_inverse;
    ui1 += h * F1 * m_inverse;
    ui2 += h * F2 * m_inverse;
    D4 pn = pi;
    if (c.last) {
        P.force[i] = F0;
        P.force[cap + i] = F1;
        P.force[2 * cap + i] = F2;
        P.torque[i] = 0.;
        P.torque[cap + i] = 0.;
        P.torque[2 * cap + i] = 0.;
    } else {
        ui0 += h * F0 * m_inverse;
        ui1 += h * F1 * m_inverse;
        ui2 += h * F2 * m_inverse;
        pn.x += fc.dt * ui0;
        pn.y += fc.dt * ui1;
        pn.z += fc.dt * ui2;
        vmax2 = fmax(vmax2, ui0 * ui0 + ui1 * ui1 + ui2 * ui2);
    }
    st4(P.pos[c.cur ^ 1], i, pn);
    vc[i] = ui0;
    vc[cap + i] = ui1;
    vc[2 * cap + i] = ui2;
}

// A particle whose only contact candidates are the walls (and the mesh): defer when it has
// tracked contacts, mesh candidates or a wall overlap.
__device__ __forceinline__ bool wall_defer(const Particles &P, const ForceConsts &fc,
                                           const WallGeom *__restrict__ walls, int i, const D4 &pi, bool defer) {
    // a particle near the mesh (candidates) or with a tracked triangle contact takes the full step
    if (!defer && fc.mesh.nt) defer = (fc.mesh.ncand[i] | fc.mesh.cnt[i]) != 0;
    const int scene_i = P.scene ? P.scene[i] : 0;
    const int wall0 = fc.wps ? scene_i * fc.wps : 0;
    const int wall1 = fc.wps ? wall0 + fc.wps : fc.nwall;
    for (int w = wall0; w < wall1 && !defer; ++w) {
        const WallGeom &g = walls[w];   // point and normal only (the velocity is not needed here)
        const double tmp = (pi.x - __ldg(&g.x[0])) * __ldg(&g.n[0]) + (pi.y - __ldg(&g.x[1])) * __ldg(&g.n[1]) +
                           (pi.z - __ldg(&g.x[2])) * __ldg(&g.n[2]);
        defer = (pi.w - tmp) > 0.;
    }
    return defer;
}

// Wall-gap flags after a build: wfar[i] = 1 when every wall of particle i's scene is farther
// than half_skin (the overlap r_i - (x_i - x_w).n_w of wall_defer below -half_skin).  While
// twice the displacement bound stays below half_skin (walls static) such a particle cannot
// reach a wall, so the staged streaming kernel skips its wall test -- the same rule as the
// clear class of the re-sort for listed neighbours.  Non-finite positions give 0.
__global__ void k_wall_far(Particles P, NbrList L, Ctl *ctl, ForceConsts fc, const WallGeom *__restrict__ walls,
                           double half_skin) {
    const double4 *__restrict__ pc = P.pos[ctl->cur];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += gridDim.x * blockDim.x) {
        const D4 pi = ld4(pc, i);
        const int scene_i = P.scene ? P.scene[i] : 0;
        const int wall0 = fc.wps ? scene_i * fc.wps : 0;
        const int wall1 = fc.wps ? wall0 + fc.wps : fc.nwall;
        bool far = true;
        for (int w = wall0; w < wall1; ++w) {
            const WallGeom &g = walls[w];
            const double tmp = (pi.x - g.x[0]) * g.n[0] + (pi.y - g.x[1]) * g.n[1] + (pi.z - g.x[2]) * g.n[2];
            far = far && (pi.w - tmp) < -half_skin;
        }
        L.wfar[i] = far ? 1 : 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) ctl->wfar_build = ctl->rebuilds;
}

void launch_wall_far(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc, const WallGeom *walls,
                     double half_skin, cudaStream_t s) {
    if (!L.wfar || fc.mwalls || fc.mesh.nt || !(half_skin > 0.0) || P.n <= 0) return;
    k_wall_far<<<148 * 8, 256, 0, s>>>(P, L, ctl, fc, walls, half_skin);
}

// Streaming body for one particle i (any class); returns whether it is deferred.
__device__ __forceinline__ bool stream_particle(const Particles &P, const NbrList &L, const ForceConsts &fc,
                                                const WallGeom *__restrict__ walls, const StreamCtl &c, int i,
                                                double &vmax2) {
    const int cap = P.cap;
    const double4 *__restrict__ pc = P.pos[c.cur];
    double *vc = P.vel[c.vcur];
    // all own-state loads first (one memory round trip per particle)
    const D4 pi = ld4_early(pc, i);
    const int cs = ld_early_i(P.cstate + i);
    // the re-sort placed particles without listed neighbours first: their lists stay empty
    // until the next build, so neither the list nor a partner is read (one round trip)
    const bool lone = i < c.nlone;
    const int nn = lone ? 0 : ld_early_i(L.nn + i);
    const double m = ld_early(&P.mI[i]);
    const double ui0 = ld_early(vc + i), ui1 = ld_early(vc + cap + i), ui2 = ld_early(vc + 2 * cap + i);
    // the first two list slots are read with the own state (in bounds for every i; the
    // value is only used below the list length), so that most warps need one more
    // round trip (the partners' positions) instead of two per neighbour
    const int j0 = (!lone && L.maxnb > 0) ? ld_early_i(L.idx + i) : 0;
    const int j1 = (!lone && L.maxnb > 1) ? ld_early_i(L.idx + cap + i) : 0;
    bool defer = cs != 0;
    if (!defer && nn > 0 && i >= c.nclear_end) {
        const D4 pa = ld4(pc, j0);
        D4 pb = pa;
        if (nn > 1) pb = ld4(pc, j1);
        const double ax = pi.x - pa.x, ay = pi.y - pa.y, az = pi.z - pa.z;
        const double sa = pi.w + pa.w;
        defer = !(ax * ax + ay * ay + az * az >= sa * sa * 1.0000000001);
        if (nn > 1) {
            const double bx = pi.x - pb.x, by = pi.y - pb.y, bz = pi.z - pb.z;
            const double sb = pi.w + pb.w;
            defer = defer || !(bx * bx + by * by + bz * bz >= sb * sb * 1.0000000001);
        }
    }
    for (int kk = 2; kk < nn && !defer && i >= c.nclear_end; ++kk) {
        const int j = L.idx[(long)kk * cap + i];
        const D4 pj = ld4(pc, j);
        const double px = pi.x - pj.x, py = pi.y - pj.y, pz = pi.z - pj.z;
        const double r2ij = px * px + py * py + pz * pz;
        const double sr = pi.w + pj.w;
        defer = !(r2ij >= sr * sr * 1.0000000001);
    }
    defer = wall_defer(P, fc, walls, i, pi, defer);
    if (!defer) stream_free_step(P, fc, c, vc, i, pi, m, ui0, ui1, ui2, vmax2);
    return defer;
}

// Block size is a run-time choice (dem_solver_params.stream_block): 64 x 16, 128 x 10 or
// 256 x 4 blocks per SM (register caps 64, 48, 64).  On the 2M lattice 128 x 10 was fastest in a
// B200 sweep; the autotuner picks per workload.  One thread per particle, every particle.
template <int BS, int MINB>
__global__ void __launch_bounds__(BS, MINB) k_stream(Particles P, NbrList L, Ctl *ctl, ForceConsts fc,
                                                     const WallGeom *__restrict__ walls) {
    grid_dep_wait();   // launched as a dependent (launch_k): the kernel before has completed
    grid_dep_release();
    if (!step_gate(ctl)) return;
    const StreamCtl c = stream_ctl(ctl, P.n);
    double vmax2 = 0.0;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    bool defer = false;
    if (i < P.n) defer = stream_particle(P, L, fc, walls, c, i, vmax2);
    defer_append(ctl, L, defer, i);
    warp_vmax(ctl, P.vslots, vmax2, 0);
}

// Split streaming pass, part 1: the particles [0, nlone) the last re-sort placed first (no
// listed neighbour until the next build).  Persistent grid-stride loop over that range; per
// particle only the own state is read (position, radius, contact word, mass, velocity), so
// the kernel is compiled for the full 64 warps per SM.
template <int BS>
__global__ void __launch_bounds__(BS, 1536 / BS) k_stream_lone(Particles P, NbrList L, Ctl *ctl, ForceConsts fc,
                                                               const WallGeom *__restrict__ walls) {
    if (!step_gate(ctl)) return;
    const StreamCtl c = stream_ctl(ctl, P.n);
    const int cap = P.cap;
    const double4 *__restrict__ pc = P.pos[c.cur];
    double *vc = P.vel[c.vcur];
    double vmax2 = 0.0;
    for (int base = blockIdx.x * BS; base < c.nlone; base += gridDim.x * BS) {   // block-uniform
        const int i = base + threadIdx.x;
        bool defer = false;
        if (i < c.nlone) {
            const D4 pi = ld4_early(pc, i);
            const int cs = ld_early_i(P.cstate + i);
            const double m = ld_early(&P.mI[i]);
            const double ui0 = ld_early(vc + i), ui1 = ld_early(vc + cap + i), ui2 = ld_early(vc + 2 * cap + i);
            defer = wall_defer(P, fc, walls, i, pi, cs != 0);
            if (!defer) stream_free_step(P, fc, c, vc, i, pi, m, ui0, ui1, ui2, vmax2);
        }
        defer_append(ctl, L, defer, i);
    }
    warp_vmax(ctl, P.vslots, vmax2, 0);
}

// Split streaming pass, part 2: the particles [nlone, n), persistent grid-stride loop, the
// body of k_stream.
template <int BS, int MINB>
__global__ void __launch_bounds__(BS, MINB) k_stream_rest(Particles P, NbrList L, Ctl *ctl, ForceConsts fc,
                                                          const WallGeom *__restrict__ walls) {
    if (!step_gate(ctl)) return;
    const StreamCtl c = stream_ctl(ctl, P.n);
    double vmax2 = 0.0;
    for (int base = c.nlone + blockIdx.x * BS; base < P.n; base += gridDim.x * BS) {   // block-uniform
        const int i = base + threadIdx.x;
        bool defer = false;
        if (i < P.n) defer = stream_particle(P, L, fc, walls, c, i, vmax2);
        defer_append(ctl, L, defer, i);
    }
    warp_vmax(ctl, P.vslots, vmax2, 0);
}

// Staged streaming pass (split 4): the body of k_stream over tiles of T consecutive particles,
// their own state brought into shared memory by bulk asynchronous copies.  A persistent block
// walks the tiles blockIdx.x, blockIdx.x + gridDim.x, ...; thread 0 keeps S tiles in flight
// (each tile's rows -- position, velocity x/y/z, mass, contact word and, where the tile
// reaches past the clear class, list length and the first two list rows -- as one copy per
// row completing on the tile's barrier), so the HBM reads of the next tiles overlap the
// partner loads and stores of the current one instead of waiting on per-thread loads.
// Waits are bounded: a wait that gives up sets DEM_ERR_TIMEOUT, waits (bounded again) for
// the block's copies still in flight and leaves the step unfinished.
constexpr int kBulkWaitLimit = 1 << 18;

template <int T>
struct BulkTile {
    static constexpr int POS = 0;                 // double4 [T]
    static constexpr int VEL = POS + 32 * T;      // double [3][T]
    static constexpr int MASS = VEL + 24 * T;     // double [T]
    static constexpr int CS = MASS + 8 * T;       // int [T]
    static constexpr int NN = CS + 4 * T;         // int [T]
    static constexpr int IDX = NN + 4 * T;        // int [2][T]
    static constexpr int WFAR = IDX + 8 * T;      // uint8 [T]
    static constexpr int BYTES = WFAR + T;
};

#ifndef STREAM_BULK_MINB
#define STREAM_BULK_MINB 9
#endif
template <int T, int S>
__global__ void __launch_bounds__(T, STREAM_BULK_MINB) k_stream_bulk(Particles P, NbrList L, Ctl *ctl, ForceConsts fc,
                                                   const WallGeom *__restrict__ walls) {
    grid_dep_wait();   // launched as a dependent (launch_k): the kernel before has completed
    grid_dep_release();
    using B = BulkTile<T>;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t full[S];
    __shared__ int s_fail;
    if (!step_gate(ctl)) return;
    const StreamCtl c = stream_ctl(ctl, P.n);
    const int cap = P.cap;
    const double4 *__restrict__ pc = P.pos[c.cur];
    double *vc = P.vel[c.vcur];
    const int ntiles = (P.n + T - 1) / T;
    const int mine = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    if (threadIdx.x == 0) {
        for (int k = 0; k < S; ++k) bulk::bar_init(&full[k], 1);
        bulk::bar_init_fence();
        s_fail = 0;
    }
    __syncthreads();
    // thread 0: the copies of this block's k-th tile into stage k % S
    auto issue = [&](int k) {
        const int i0 = (blockIdx.x + k * gridDim.x) * T;
        const int m = min(T, cap - i0);   // cap is a multiple of 64, i0 of T: m is 64 or T
        const bool lists = i0 + m > c.nclear_end;
        const int rows = lists ? (L.maxnb > 1 ? 2 : L.maxnb) : 0;
        unsigned char *sb = smem + (k % S) * B::BYTES;
        uint64_t *bar = &full[k % S];
        bulk::bar_arrive_expect(bar, (uint32_t)m * (32u + 24u + 8u + 4u + (lists ? 4u : 0u) + 4u * rows + (c.wfar ? 1u : 0u)));
        if (fc.drop_copies) return;   // testing the bounded waits: nothing will arrive
        bulk::copy_g2s(sb + B::POS, pc + i0, 32u * m, bar);
        for (int d = 0; d < 3; ++d) bulk::copy_g2s(sb + B::VEL + 8 * T * d, vc + (long)d * cap + i0, 8u * m, bar);
        // rows every step reads again and (between builds) hardly anything writes: kept in L2 across
        // steps (at most 25 bytes per particle, 50 MB on the 2M lattice; the velocities kept as well
        // measured slower)
        const uint64_t keep = bulk::policy_keep();
        bulk::copy_g2s_hint(sb + B::MASS, P.mI + i0, 8u * m, bar, keep);
        bulk::copy_g2s_hint(sb + B::CS, P.cstate + i0, 4u * m, bar, keep);
        if (lists) bulk::copy_g2s_hint(sb + B::NN, L.nn + i0, 4u * m, bar, keep);
        for (int r = 0; r < rows; ++r)
            bulk::copy_g2s_hint(sb + B::IDX + 4 * T * r, L.idx + (long)r * cap + i0, 4u * m, bar, keep);
        if (c.wfar) bulk::copy_g2s_hint(sb + B::WFAR, L.wfar + i0, (uint32_t)m, bar, keep);
    };
    if (threadIdx.x == 0)
        for (int k = 0; k < S && k < mine; ++k) issue(k);
    const int limit = fc.wait_polls > 0 ? fc.wait_polls : kBulkWaitLimit;
    double vmax2 = 0.0;
    int k = 0;
    for (; k < mine; ++k) {
        if (!bulk::bar_wait(&full[k % S], (k / S) & 1, limit)) s_fail = 1;
        __syncthreads();
        if (s_fail) break;
        const unsigned char *sb = smem + (k % S) * B::BYTES;
        const int t = threadIdx.x;
        const int i = (blockIdx.x + k * gridDim.x) * T + t;
        bool defer = false;
        if (i < P.n) {
            const D4 pi = reinterpret_cast<const D4 *>(sb + B::POS)[t];
            const double *sv = reinterpret_cast<const double *>(sb + B::VEL);
            const double ui0 = sv[t], ui1 = sv[T + t], ui2 = sv[2 * T + t];
            const double m = reinterpret_cast<const double *>(sb + B::MASS)[t];
            defer = reinterpret_cast<const int *>(sb + B::CS)[t] != 0;
            // lone and clear particles: no listed neighbour can touch them this step
            const int nn = i >= c.nclear_end ? reinterpret_cast<const int *>(sb + B::NN)[t] : 0;
            if (!defer && nn > 0) {
                const int *sidx = reinterpret_cast<const int *>(sb + B::IDX);
                const D4 pa = ld4(pc, sidx[t]);
                D4 pb = pa;
                if (nn > 1) pb = ld4(pc, sidx[T + t]);
                const double ax = pi.x - pa.x, ay = pi.y - pa.y, az = pi.z - pa.z;
                const double sa = pi.w + pa.w;
                defer = !(ax * ax + ay * ay + az * az >= sa * sa * 1.0000000001);
                if (nn > 1) {
                    const double bx = pi.x - pb.x, by = pi.y - pb.y, bz = pi.z - pb.z;
                    const double sb2 = pi.w + pb.w;
                    defer = defer || !(bx * bx + by * by + bz * bz >= sb2 * sb2 * 1.0000000001);
                }
            }
            for (int kk = 2; kk < nn && !defer; ++kk) {
                const int j = L.idx[(long)kk * cap + i];
                const D4 pj = ld4(pc, j);
                const double px = pi.x - pj.x, py = pi.y - pj.y, pz = pi.z - pj.z;
                const double r2ij = px * px + py * py + pz * pz;
                const double sr = pi.w + pj.w;
                defer = !(r2ij >= sr * sr * 1.0000000001);
            }
            // the wall test, unless the last build found every wall beyond reach
            if (!(c.wfar && sb[B::WFAR + t])) defer = wall_defer(P, fc, walls, i, pi, defer);
            if (!defer) stream_free_step(P, fc, c, vc, i, pi, m, ui0, ui1, ui2, vmax2);
        }
        defer_append(ctl, L, defer, i);
        __syncthreads();   // stage k % S consumed: thread 0 refills it
        if (threadIdx.x == 0 && k + S < mine) issue(k + S);
    }
    if (k < mine) {   // a wait gave up: report, and let the copies in flight land before exiting
        if (threadIdx.x == 0) {
            atomicOr(&ctl->status, DEM_ERR_TIMEOUT);
            for (int q = k; q < k + S && q < mine; ++q) bulk::bar_wait(&full[q % S], (q / S) & 1, limit);
        }
        return;
    }
    warp_vmax(ctl, P.vslots, vmax2, 0);
}

// Fused step, kernel 2 of 3: the full arithmetic for the deferred particles.  New u and
// omega go to scratch slot t (their current values are still read by contact partners).
template <int MINB, bool MESH = false>
__global__ void __launch_bounds__(kBlock, MINB) k_contact(Particles P, NbrList L, Ctl *ctl, ForceConsts fc,
                                                    const PairConst *__restrict__ pp, const PairConst *__restrict__ pw,
                                                    const WallGeom *__restrict__ walls) {
    grid_dep_wait();   // launched as a dependent (launch_k): the kernel before has completed
    grid_dep_release();
    if (!step_gate(ctl)) return;
    const int nd = ctl->ndefer;
    if ((long)blockIdx.x * blockDim.x >= nd) return;
    const int cur = ctl->cur, vcur = ctl->vcur;
    const int last = ctl->steps_done + 1 >= ctl->target;
    double vmax2 = 0.0;
    int status = 0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nd; t += gridDim.x * blockDim.x) {
        double v2 = 0.0;
        particle_full<MODE_FUSED, false, MESH>(P, L, fc, pp, pw, walls, cur, cur ^ 1, vcur, last, L.defer[t], t, v2,
                                         status);
        vmax2 = fmax(vmax2, v2);
    }
    block_vmax(ctl, P.vslots, vmax2, status);
}

// One-kernel step for dense flows (most particles in contact): every particle takes the
// full arithmetic, positions and velocities go to the other buffers, and the last block
// finalises the step.  Same results as the three-kernel step.
template <int MINB, bool MESH = false>
__global__ void __launch_bounds__(kBlock, MINB) k_contact_all(Particles P, NbrList L, Ctl *ctl, ForceConsts fc,
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
        particle_full<MODE_FUSED_DIRECT, false, MESH>(P, L, fc, pp, pw, walls, c.cur, c.cur ^ 1, vcur, c.last, i, i, v2,
                                                status, &a);
        vmax2 = fmax(vmax2, v2);
        active += a;
    }
    finish_step_counted(ctl, P.vslots, vmax2, fc.dt, status, active, fc, !c.last);
}

// Fused step, kernel 3 of 3: commit the deferred particles' u and omega, then the last
// block to take a ticket finalises the step (displacement bound, position-buffer flip,
// step counter, deferred-list reset).  Each block copies ndefer before its ticket, so the
// reset cannot cut another block's copy short.  With at most kApplyOneBlock deferred particles
// (a sparse step: tens on the 2M lattice) block 0 alone commits and finalises, and the other
// blocks leave at once: no ticket chain on the step's path.
constexpr int kApplyOneBlock = 8 * kApplyBlock;
__global__ void __launch_bounds__(kApplyBlock) k_apply(Particles P, NbrList L, Ctl *ctl, ForceConsts fc) {
    grid_dep_wait();   // launched as a dependent (launch_k): the kernel before has completed
    grid_dep_release();
    __shared__ int s_nd, s_go, s_last;
    if (threadIdx.x == 0) {
        s_go = step_gate(ctl);
        s_nd = ctl->ndefer;
    }
    __syncthreads();
    if (!s_go) return;
    const int nd = s_nd, cap = P.cap, vcur = ctl->vcur;
    const bool one = nd <= kApplyOneBlock;   // the same in every block
    if (one && blockIdx.x != 0) return;
    double *vc = P.vel[vcur], *wc = P.omg[vcur];
    const int stride = one ? blockDim.x : gridDim.x * blockDim.x;
    for (int t = (one ? 0 : blockIdx.x * blockDim.x) + threadIdx.x; t < nd; t += stride) {
        const int i = L.defer[t];
        for (int d = 0; d < 3; ++d) {
            vc[d * cap + i] = L.defer_v[d * cap + t];
            wc[d * cap + i] = L.defer_w[d * cap + t];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (one) {
            s_last = 1;
        } else {
            const unsigned tk = take_ticket(&ctl->ticket);
            s_last = (tk == gridDim.x - 1);
        }
    }
    __syncthreads();
    if (s_last && threadIdx.x < 32) {   // every block has taken its ticket: the slots are quiescent
        const double v2 = fmax(vmax_collect_warp(P.vslots), mesh_speed2(fc));
        // walls and mesh drift with the particles' stage2 of the next step (none after a run's last step)
        if (ctl->steps_done + 1 < ctl->target) advance_kinematics(fc);
        if (threadIdx.x == 0) {
            ctl->disp = ctl->disp + fc.dt * sqrt(v2) * (1.0 + 1e-9);
            ctl->last_ndefer = nd;
            ctl->ndefer = 0;
            ctl->cur ^= 1;
            ctl->steps_done += 1;
            ctl->total_steps += 1;
            ctl->ticket = 0u;
        }
    }
}

// Prologue of a run: stage1 + stage2 of its first step with the stored F, tau
// (src/CabanaDEM_Integrator.hpp:31-74).  u and omega in place; positions to the next
// buffer, which becomes current.
// Persistent grid-stride form: the step finalisation takes one ticket per block, so a grid of
// one block per 128 particles (15,625 on the 2M lattice) would queue as many atomics on one word.
__global__ void __launch_bounds__(kBlock) k_prologue(Particles P, Ctl *ctl, ForceConsts fc) {
    const int cur = ctl->cur, nxt = cur ^ 1, vcur = ctl->vcur;
    const int cap = P.cap;
    double vmax2 = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += gridDim.x * blockDim.x) {
        const double m_inverse = 1. / P.mI[i], h = fc.half_dt;
        double *vc = P.vel[vcur], *wc = P.omg[vcur];
        double u[3];
        for (int d = 0; d < 3; ++d) {
            u[d] = vc[d * cap + i] + h * P.force[d * cap + i] * m_inverse;
            vc[d * cap + i] = u[d];
        }
        // zero torque leaves omega as it is (the streaming kernel's rule for particles without
        // pair or wall contacts): omega and I are read only for particles with a torque
        const double t0 = P.torque[i], t1 = P.torque[cap + i], t2 = P.torque[2 * cap + i];
        if (t0 != 0. || t1 != 0. || t2 != 0.) {
            const double I_inverse = 1. / P.mI[cap + i];
            wc[i] = wc[i] + h * t0 * I_inverse;
            wc[cap + i] = wc[cap + i] + h * t1 * I_inverse;
            wc[2 * cap + i] = wc[2 * cap + i] + h * t2 * I_inverse;
        }
        D4 p = ld4(P.pos[cur], i);
        p.x += fc.dt * u[0];
        p.y += fc.dt * u[1];
        p.z += fc.dt * u[2];
        vmax2 = fmax(vmax2, u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        st4(P.pos[nxt], i, p);
    }
    finish_step(ctl, P.vslots, vmax2, fc.dt, 0, false, false, &fc);
}

// Unfused Integrator stages, in place on the current buffer.
__global__ void k_stage(Particles P, Ctl *ctl, ForceConsts fc, int stage) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (stage == 2 && i < 32) advance_kinematics(fc);   // block 0's first warp
    if (i >= P.n) return;
    const int cur = ctl->cur, vcur = ctl->vcur, cap = P.cap;
    double *vc = P.vel[vcur], *wc = P.omg[vcur];
    if (stage == 2) {
        D4 p = ld4(P.pos[cur], i);
        p.x += fc.dt * vc[i];
        p.y += fc.dt * vc[cap + i];
        p.z += fc.dt * vc[2 * cap + i];
        st4(P.pos[cur], i, p);
        return;
    }
    const double2 mIi = load_mI(P, i);
    const double m_inverse = 1. / mIi.x, I_inverse = 1. / mIi.y, h = fc.half_dt;
    for (int d = 0; d < 3; ++d) {
        vc[d * cap + i] += h * P.force[d * cap + i] * m_inverse;
        wc[d * cap + i] += h * P.torque[d * cap + i] * I_inverse;
    }
}

// Energy totals: per-block partial sums in a fixed tree order, then one thread sums
// the block partials in block order (deterministic).
__global__ void __launch_bounds__(kBlock) k_energy_partials(Particles P, NbrList L, ForceConsts fc,
                                                            const PairConst *__restrict__ pp,
                                                            const PairConst *__restrict__ pw,
                                                            const WallGeom *__restrict__ walls, const Ctl *ctl,
                                                            double *partials) {
    const int cur = ctl->cur, vcur = ctl->vcur;
    __shared__ double red[4][kBlock];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int cap = P.cap;
    double e[4] = {0., 0., 0., 0.};
    if (i < P.n) {
        const double2 mIi = load_mI(P, i);
        const double *vc = P.vel[vcur], *wc = P.omg[vcur];
        const double u0 = vc[i], u1 = vc[cap + i], u2 = vc[2 * cap + i];
        const double w0 = wc[i], w1 = wc[cap + i], w2 = wc[2 * cap + i];
        e[0] = 0.5 * mIi.x * (u0 * u0 + u1 * u1 + u2 * u2);
        e[1] = 0.5 * mIi.y * (w0 * w0 + w1 * w1 + w2 * w2);
        const D4 pi = ld4(P.pos[cur], i);
        const int mi = fc.nmat > 1 ? (int)P.mat[i] : 0;
        for (int kk = 0; kk < L.nn[i]; ++kk) {
            const int j = L.idx[(long)kk * cap + i];
            const D4 pj = ld4(P.pos[cur], j);
            const double px = pi.x - pj.x, py = pi.y - pj.y, pz = pi.z - pj.z;
            const double ov = pi.w + pj.w - sqrt(px * px + py * py + pz * pz);
            if (ov > 0.) {
                const int mj = fc.nmat > 1 ? (int)P.mat[j] : 0;
                const double R_eff = 1. / (1. / pi.w + 1. / pj.w);
                const double kn = pp[mi * fc.nmat + mj].c_kn * sqrt(R_eff);
                e[2] += 0.5 * 0.4 * kn * ov * ov * sqrt(ov);  // half of each pair (full list)
            }
        }
        const int scene_i = P.scene ? P.scene[i] : 0;
        const int wall0 = fc.wps ? scene_i * fc.wps : 0;
        const int wall1 = fc.wps ? wall0 + fc.wps : fc.nwall;
        for (int w = wall0; w < wall1; ++w) {
            const WallGeom g = walls[w];
            const double ov = pi.w - ((pi.x - g.x[0]) * g.n[0] + (pi.y - g.x[1]) * g.n[1] + (pi.z - g.x[2]) * g.n[2]);
            if (ov > 0.) {
                const double kn = pw[mi * fc.nwall + w].c_kn * sqrt(1. / (1. / pi.w + 0.));
                e[3] += 0.4 * kn * ov * ov * sqrt(ov);
            }
        }
    }
    for (int k = 0; k < 4; ++k) red[k][threadIdx.x] = e[k];
    __syncthreads();
    for (int s = kBlock / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int k = 0; k < 4; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x < 4) partials[(long)blockIdx.x * 4 + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void k_energy_final(const double *partials, int nparts, double *out) {
    if (threadIdx.x < 4) {
        double s = 0.;
        for (int b = 0; b < nparts; ++b) s += partials[(long)b * 4 + threadIdx.x];
        out[threadIdx.x] = s;
    }
}

// Mesh candidates of each particle at a neighbour build: every triangle whose closest point lies
// within the list cutoff (delta, or r_i + skin), ascending id, by brute force over the mesh.
// More than kMeshCand candidates: DEM_ERR_MESH_OVERFLOW (the extra triangles are not seen).
__global__ void __launch_bounds__(kBlock) k_mesh_cand(Particles P, MeshDev M, Ctl *ctl, double delta, double skin) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    if (ctl->status & DEM_ERR_NAN) {
        M.ncand[i] = 0;
        return;
    }
    const D4 pi = ld4(P.pos[ctl->cur], i);
    const double x[3] = {pi.x, pi.y, pi.z};
    const double D[3] = {M.D[0], M.D[1], M.D[2]};
    const double reach = delta > 0.0 ? delta : pi.w + skin;
    int k = 0;
    bool over = false;
    for (int t = 0; t < M.nt; ++t) {
        double a[3], b[3], c[3], q[3];
        int f;
        mesh_vertices(M, t, D, a, b, c);
        tri_closest(x, a, b, c, q, f);
        const double dx = x[0] - q[0], dy = x[1] - q[1], dz = x[2] - q[2];
        if (dx * dx + dy * dy + dz * dz <= reach * reach) {
            if (k < kMeshCand)
                M.cand[(long)k++ * P.cap + i] = t;
            else
                over = true;
        }
    }
    M.ncand[i] = (unsigned char)k;
    if (over) atomicOr(&ctl->status, DEM_ERR_MESH_OVERFLOW);
}

// Re-sort: the tracked triangle contacts move with their particles (new p <- old items[p]).
__global__ void k_permute_mesh(MeshDev M, MeshDev A, int n, int cap, const int *items) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const int q = items[p];
        A.cnt[p] = M.cnt[q];
        for (int s2 = 0; s2 < M.mt; ++s2) A.tid[(long)s2 * cap + p] = M.tid[(long)s2 * cap + q];
        for (long k = 0; k < 3L * M.mt; ++k) A.th[k * cap + p] = M.th[k * cap + q];
    }
}

// ---------------------------------------------------------------------------------------
static inline int nblocks(int n) { return (n + kBlock - 1) / kBlock; }

void launch_mesh_candidates(const Particles &P, const MeshDev &M, Ctl *ctl, double delta, double skin, cudaStream_t s) {
    k_mesh_cand<<<nblocks(P.n), kBlock, 0, s>>>(P, M, ctl, delta, skin);
}

void launch_permute_mesh(const MeshDev &M, const MeshDev &A, int n, int cap, const int *items, cudaStream_t s) {
    k_permute_mesh<<<148 * 4, 256, 0, s>>>(M, A, n, cap, items);
}

void launch_prologue(const Particles &P, Ctl *ctl, const ForceConsts &fc, cudaStream_t s) {
    const int g = nblocks(P.n) < 148 * 12 ? nblocks(P.n) : 148 * 12;
    k_prologue<<<g > 0 ? g : 1, kBlock, 0, s>>>(P, ctl, fc);
}

int kernels_per_step(const ForceConsts &fc) {
    if (fc.all) return fc.all == 2 ? 3 : 1;
    return fc.split == 2 || fc.split == 3 ? 4 : 3;
}

#ifndef STREAM_BULK_STAGES
#define STREAM_BULK_STAGES 2
#endif
#ifndef STREAM_BULK_T
#define STREAM_BULK_T 128
#endif
constexpr int kBulkT = STREAM_BULK_T, kBulkS = STREAM_BULK_STAGES;

// Persistent grid of the staged streaming kernel: every block the SMs hold at its shared
// memory, at most one per tile.
static int bulk_blocks(int n) {
    static thread_local int per = -1, sms = 0;
    if (per < 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
        const int smem = kBulkS * BulkTile<kBulkT>::BYTES;
        cudaFuncSetAttribute((const void *)k_stream_bulk<kBulkT, kBulkS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_stream_bulk<kBulkT, kBulkS>, kBulkT, smem);
        if (per <= 0) per = 1;
    }
    const int tiles = (n + kBulkT - 1) / kBulkT;
    return std::max(1, std::min(tiles, sms * per));
}

static int persistent_blocks(const void *kernel, int block, int n) {
    static thread_local int sms = 0;   // per host thread: solvers run concurrently from threads
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    int per = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, block, 0);
    if (per <= 0) per = 1;
    const int need = (n + block - 1) / block;
    return need < sms * per ? (need > 0 ? need : 1) : sms * per;
}

template <bool MESH>
static void launch_step_t(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc, const PairConst *pp,
                 const PairConst *pw, const WallGeom *walls, int mode, cudaStream_t s, const AuxStream &aux) {
    if (mode == MODE_FUSED && fc.all == 2) {
        if (fc.mixed) {
            launch_pairs_mixed(P, L, ctl, fc, pp, pw, walls, MESH, s);
        } else {
            static thread_local int g2 = 0, g3 = 0, sms = 0, last_np = -1;
            if (last_np != P.n) {
                g2 = persistent_blocks((const void *)k_pairs_eval<false>, kPairsBlock, 8 * P.n);
                g3 = persistent_blocks((const void *)k_pairs_sum<false, MESH>, kPairsBlock, P.n);
                int dev = 0;
                cudaGetDevice(&dev);
                cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
                if (sms <= 0) sms = 148;
                last_np = P.n;
            }
            launch_pairs_find<false>(P, L, ctl, fc, walls, sms, s);
            launch_k(k_pairs_eval<false>, g2, kPairsBlock, 0, s, fc.pdl, P, L, ctl, fc, pp, pw, walls);
            launch_k(k_pairs_sum<false, MESH>, g3, kPairsBlock, 0, s, fc.pdl, P, L, ctl, fc);
        }
    } else if (mode == MODE_FUSED && fc.all) {
        static thread_local int ga = 0, gma = 0, last_na = -1;
        if (last_na != P.n) {
            ga = persistent_blocks((const void *)k_contact_all<kContactMinBlocksDense, MESH>, kBlock, P.n);
            gma = persistent_blocks(contact_mixed_all_kernel(MESH), kBlock, P.n);
            last_na = P.n;
        }
        if (fc.mixed)
            launch_contact_mixed_all(P, L, ctl, fc, pp, pw, walls, gma, MESH, s);
        else
            launch_k(k_contact_all<kContactMinBlocksDense, MESH>, ga, kBlock, 0, s, fc.pdl, P, L, ctl, fc, pp, pw, walls);
    } else if (mode == MODE_FUSED) {
        static thread_local int gc = 0, gm = 0, gcd = 0, gmd = 0, gk4 = 0, gk8 = 0, gkm4 = 0, gkm8 = 0, last_n = -1;
        if (last_n != P.n) {
            // contact kernels: every block the SMs hold (a dense packing defers nearly every
            // particle; blocks past the deferred count exit at once); the apply kernel copies
            // 48 B per deferred particle and takes one ticket per block: one block per SM
            gc = persistent_blocks((const void *)k_contact<1, MESH>, kBlock, P.n);
            gm = persistent_blocks(contact_mixed_kernel(0, 0, MESH), kBlock, P.n);
            gcd = persistent_blocks((const void *)k_contact<kContactMinBlocksDense, MESH>, kBlock, P.n);
            gmd = persistent_blocks(contact_mixed_kernel(1, 0, MESH), kBlock, P.n);
            // cooperative kernels: a block serves kBlock / NL particles per pass
            gk4 = persistent_blocks((const void *)k_contact_coop<4, kCoopMinBlocks, false, MESH>, kBlock, 4 * P.n);
            gk8 = persistent_blocks((const void *)k_contact_coop<8, kCoopMinBlocks, false, MESH>, kBlock, 8 * P.n);
            gkm4 = persistent_blocks(contact_mixed_kernel(0, 4, MESH), kBlock, 4 * P.n);
            gkm8 = persistent_blocks(contact_mixed_kernel(0, 8, MESH), kBlock, 8 * P.n);
            last_n = P.n;
        }
        if (fc.split == 2 || fc.split == 3) {
            // lone particles and the rest in two persistent kernels; with the concurrent form
            // (split 3, an aux stream given) as two graph branches whose grids share the SMs
            static thread_local int sms = 0;
            if (!sms) {
                int dev = 0;
                cudaGetDevice(&dev);
                cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
                if (sms <= 0) sms = 148;
            }
            const bool conc = fc.split == 3 && aux.stream;
            const int glone = sms * (conc ? 7 : 12), grest = sms * (conc ? 5 : 9);
            if (conc) {
                cudaEventRecord(aux.fork, s);
                cudaStreamWaitEvent(aux.stream, aux.fork, 0);
                k_stream_rest<128, 9><<<grest, 128, 0, aux.stream>>>(P, L, ctl, fc, walls);
                k_stream_lone<128><<<glone, 128, 0, s>>>(P, L, ctl, fc, walls);
                cudaEventRecord(aux.join, aux.stream);
                cudaStreamWaitEvent(s, aux.join, 0);
            } else {
                k_stream_lone<128><<<glone, 128, 0, s>>>(P, L, ctl, fc, walls);
                k_stream_rest<128, 9><<<grest, 128, 0, s>>>(P, L, ctl, fc, walls);
            }
        } else if (fc.split == 4) {
            launch_k(k_stream_bulk<kBulkT, kBulkS>, bulk_blocks(P.n), kBulkT, kBulkS * BulkTile<kBulkT>::BYTES, s,
                     fc.pdl, P, L, ctl, fc, walls);
        } else if (fc.stream_block == 64)
            launch_k(k_stream<64, 16>, (P.n + 63) / 64, 64, 0, s, fc.pdl, P, L, ctl, fc, walls);
        else if (fc.stream_block == 256)
            launch_k(k_stream<256, 4>, (P.n + 255) / 256, 256, 0, s, fc.pdl, P, L, ctl, fc, walls);
        else
            launch_k(k_stream<128, 10>, (P.n + 127) / 128, 128, 0, s, fc.pdl, P, L, ctl, fc, walls);
        // the contact and apply kernels follow the streaming pass as its dependents, except after
        // the concurrent form's join (a kernel after two branches)
        const bool dep = fc.pdl && fc.split != 3;
        if (fc.mixed)
            launch_contact_mixed(P, L, ctl, fc, pp, pw, walls, MESH,
                                 fc.coop == 8 ? gkm8 : fc.coop == 4 ? gkm4 : fc.dense ? gmd : gm, s);
        else if (fc.coop == 8)
            launch_k(k_contact_coop<8, kCoopMinBlocks, false, MESH>, gk8, kBlock, 0, s, dep, P, L, ctl, fc, pp, pw, walls);
        else if (fc.coop == 4)
            launch_k(k_contact_coop<4, kCoopMinBlocks, false, MESH>, gk4, kBlock, 0, s, dep, P, L, ctl, fc, pp, pw, walls);
        else if (fc.dense)
            launch_k(k_contact<kContactMinBlocksDense, MESH>, gcd, kBlock, 0, s, dep, P, L, ctl, fc, pp, pw, walls);
        else
            launch_k(k_contact<1, MESH>, gc, kBlock, 0, s, dep, P, L, ctl, fc, pp, pw, walls);
        launch_k(k_apply, fc.dense ? 4 * 148 : 148, kApplyBlock, 0, s, fc.pdl, P, L, ctl, fc);
    } else if (fc.mixed) {
        launch_force_mixed(P, L, ctl, fc, pp, pw, walls, MESH, s);
    } else {
        k_force<MESH><<<nblocks(P.n), kBlock, 0, s>>>(P, L, ctl, fc, pp, pw, walls);
    }
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

cudaError_t launch_steps_coop(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc, const PairConst *pp,
                              const PairConst *pw, const WallGeom *walls, int max_steps, unsigned long long *scratch,
                              cudaStream_t s) {
    if (fc.mixed) return launch_steps_coop_mixed(P, L, ctl, fc, pp, pw, walls, max_steps, scratch, s);
    return fc.mesh.nt ? steps_coop_t<false, true>(P, L, ctl, fc, pp, pw, walls, max_steps, scratch, s)
                      : steps_coop_t<false, false>(P, L, ctl, fc, pp, pw, walls, max_steps, scratch, s);
}

void launch_step(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc, const PairConst *pp,
                 const PairConst *pw, const WallGeom *walls, int mode, cudaStream_t s, const AuxStream &aux) {
    if (fc.mesh.nt)
        launch_step_t<true>(P, L, ctl, fc, pp, pw, walls, mode, s, aux);
    else
        launch_step_t<false>(P, L, ctl, fc, pp, pw, walls, mode, s, aux);
}

void launch_stage(const Particles &P, Ctl *ctl, const ForceConsts &fc, int stage, cudaStream_t s) {
    k_stage<<<nblocks(P.n), kBlock, 0, s>>>(P, ctl, fc, stage);
}

void launch_energy(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc, const PairConst *pp,
                   const PairConst *pw, const WallGeom *walls, double *partials, int nparts, double *out,
                   cudaStream_t s) {
    k_energy_partials<<<nparts, kBlock, 0, s>>>(P, L, fc, pp, pw, walls, ctl, partials);
    k_energy_final<<<1, 32, 0, s>>>(partials, nparts, out);
}

bool launch_scene_table(const Particles &P, int nscenes, int2 *table, int *counts, int *bad, cudaStream_t s) {
    if (!P.scene || nscenes <= 0) return false;
    cudaMemsetAsync(counts, 0, sizeof(int) * nscenes, s);
    cudaMemsetAsync(bad, 0, sizeof(int), s);
    const int g = (P.n + 255) / 256 < 148 * 8 ? (P.n + 255) / 256 : 148 * 8;
    k_scene_hist<<<g > 0 ? g : 1, 256, 0, s>>>(P.scene, P.n, counts);
    k_scene_bounds<<<g > 0 ? g : 1, 256, 0, s>>>(P.scene, P.n, table);
    k_scene_check<<<(nscenes + 255) / 256, 256, 0, s>>>(nscenes, table, counts, bad);
    int h = 1;
    if (cudaMemcpyAsync(&h, bad, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) return false;
    if (cudaStreamSynchronize(s) != cudaSuccess) return false;
    return h == 0;
}

void launch_scene_steps(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc, const PairConst *pp,
                        const PairConst *pw, const WallGeom *walls, const int2 *table, int nscenes, int nsteps,
                        double delta, double skin, cudaStream_t s) {
    if (fc.mixed) {
        launch_scene_steps_mixed(P, L, ctl, fc, pp, pw, walls, table, nscenes, nsteps, delta, skin, s);
        return;
    }
    const SceneSmem o = scene_smem(P.mc, P.mw, P.ext != nullptr, P.fix != nullptr, fc.nmat > 1);
    if (o.bytes <= kSceneSmemMax &&
        cudaFuncSetAttribute(k_scene_steps_smem<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, o.bytes) ==
            cudaSuccess)
        k_scene_steps_smem<false><<<nscenes, kSceneBlock, o.bytes, s>>>(P, L, ctl, fc, pp, pw, walls, table, nsteps,
                                                                        delta, skin);
    else
        k_scene_steps<false><<<nscenes, kSceneBlock, 0, s>>>(P, L, ctl, fc, pp, pw, walls, table, nsteps, delta, skin);
    k_scene_run_end<<<1, 32, 0, s>>>(ctl, nsteps);
}

}  // namespace b200dem
