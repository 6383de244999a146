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

namespace b200dem {

template <int MODE>
__global__ void __launch_bounds__(kBlock) k_step(Particles P, NbrList L, Ctl *ctl, ForceConsts fc,
                                                 const PairConst *__restrict__ pp, const PairConst *__restrict__ pw,
                                                 const WallGeom *__restrict__ walls) {
    const CtlSnap cs_ = read_ctl(ctl, MODE == MODE_FUSED);
    if (!cs_.go) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double vmax2 = 0.0;
    int status = 0;
    if (i < P.n) particle_full<MODE, false>(P, L, fc, pp, pw, walls, cs_.cur, cs_.cur ^ 1, cs_.last, i, vmax2, status);
    if (MODE == MODE_FUSED) {
        finish_step(ctl, vmax2, fc.dt, status, true);
    } else if (status) {
        atomicOr(&ctl->status, status);
    }
}

// ---------------------------------------------------------------------------------------
// Fused step, part 1: streaming kernel.  A particle with no tracked contact, no active
// wall history, no neighbour within r_i + r_j (1 + 5e-11) and no wall overlap has zero
// pair force; its step reduces to hooks + integration, done here with few registers so
// the kernel runs at high occupancy.  Every other particle is appended to L.defer and
// handled by the contact kernel with the full arithmetic.  Persistent grid-stride loop;
// each thread reads the control word itself (no block barrier before the work).
// ---------------------------------------------------------------------------------------
#ifndef STREAM_MIN_BLOCKS
#define STREAM_MIN_BLOCKS 1
#endif
__global__ void __launch_bounds__(kStreamBlock, STREAM_MIN_BLOCKS) k_stream(Particles P, NbrList L, Ctl *ctl, ForceConsts fc,
                                                        const WallGeom *__restrict__ walls) {
    const int cur = ctl->cur;
    const bool stale = !(ctl->disp < ctl->half_skin);
    const int steps_done = ctl->steps_done, target = ctl->target;
    if (steps_done >= target || (ctl->status & DEM_ERR_NEIGHBOR_OVERFLOW) || stale) return;
    const bool last = steps_done + 1 >= target;
    const int nxt = cur ^ 1, cap = P.cap;
    const double4 *__restrict__ pc = P.pos[cur];
    const double *__restrict__ vc = P.vel[cur];
    const double *__restrict__ wc = P.omg[cur];
    double vmax2 = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += gridDim.x * blockDim.x) {
        // all own-state loads first (one memory round trip per particle)
        const D4 pi = ld4_early(pc, i);
        const int cs = ld_early_i(P.cstate + i);
        const int nn = ld_early_i(L.nn + i);
        const double2 mIi = ld_early2(P.mI + i);
        double ui0 = ld_early(vc + i), ui1 = ld_early(vc + cap + i), ui2 = ld_early(vc + 2 * cap + i);
        double wi0 = ld_early(wc + i), wi1 = ld_early(wc + cap + i), wi2 = ld_early(wc + 2 * cap + i);
        bool defer = cs != 0;
        for (int kk = 0; kk < nn && !defer; ++kk) {
            const int j = L.idx[(long)kk * cap + i];
            const D4 pj = ld4(pc, j);
            const double px = pi.x - pj.x, py = pi.y - pj.y, pz = pi.z - pj.z;
            const double r2ij = px * px + py * py + pz * pz;
            const double sr = pi.w + pj.w;
            defer = !(r2ij >= sr * sr * 1.0000000001);
        }
        for (int w = 0; w < fc.nwall && !defer; ++w) {
            const WallGeom g = walls[w];
            const double tmp = (pi.x - g.x[0]) * g.n[0] + (pi.y - g.x[1]) * g.n[1] + (pi.z - g.x[2]) * g.n[2];
            defer = (pi.w - tmp) > 0.;
        }
        const unsigned dmask = __ballot_sync(__activemask(), defer);
        if (defer) {
            const int lane = threadIdx.x & 31;
            const int leader = __ffs(dmask) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(&ctl->ndefer, __popc(dmask));
            base = __shfl_sync(dmask, base, leader);
            L.defer[base + __popc(dmask & ((1u << lane) - 1u))] = i;
            continue;
        }
        // no pair force: F = ext (added to zero), then the post-force hooks
        double F0 = 0., F1 = 0., F2 = 0., T0 = 0., T1 = 0., T2 = 0.;
        if (fc.has_ext) {
            F0 += P.ext[i];
            F1 += P.ext[cap + i];
            F2 += P.ext[2 * cap + i];
        }
        if (fc.has_gravity) {
            F0 += mIi.x * fc.g[0];
            F1 += mIi.x * fc.g[1];
            F2 += mIi.x * fc.g[2];
        }
        if (fc.has_fix) {
            const int f = P.fix[i];
            if (f & DEM_FIX_FORCE) F0 = F1 = F2 = 0.;
            if (f & DEM_FIX_TORQUE) T0 = T1 = T2 = 0.;
        }
        const double m_inverse = 1. / mIi.x;
        const double I_inverse = 1. / mIi.y;
        const double h = fc.half_dt;
        ui0 += h * F0 * m_inverse;
        ui1 += h * F1 * m_inverse;
        ui2 += h * F2 * m_inverse;
        wi0 += h * T0 * I_inverse;
        wi1 += h * T1 * I_inverse;
        wi2 += h * T2 * I_inverse;
        D4 pn = pi;
        if (last) {
            P.force[i] = F0;
            P.force[cap + i] = F1;
            P.force[2 * cap + i] = F2;
            P.torque[i] = T0;
            P.torque[cap + i] = T1;
            P.torque[2 * cap + i] = T2;
        } else {
            ui0 += h * F0 * m_inverse;
            ui1 += h * F1 * m_inverse;
            ui2 += h * F2 * m_inverse;
            wi0 += h * T0 * I_inverse;
            wi1 += h * T1 * I_inverse;
            wi2 += h * T2 * I_inverse;
            pn.x += fc.dt * ui0;
            pn.y += fc.dt * ui1;
            pn.z += fc.dt * ui2;
            vmax2 = fmax(vmax2, ui0 * ui0 + ui1 * ui1 + ui2 * ui2);
        }
        st4(P.pos[nxt], i, pn);
        double *vn = P.vel[nxt], *wn = P.omg[nxt];
        vn[i] = ui0;
        vn[cap + i] = ui1;
        vn[2 * cap + i] = ui2;
        wn[i] = wi0;
        wn[cap + i] = wi1;
        wn[2 * cap + i] = wi2;
    }
    // one atomic per block
    __shared__ double red[kStreamBlock / 32];
    for (int o = 16; o > 0; o >>= 1) vmax2 = fmax(vmax2, __shfl_xor_sync(0xffffffffu, vmax2, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = vmax2;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = red[0];
        for (int w = 1; w < kStreamBlock / 32; ++w) m = fmax(m, red[w]);
        if (m > 0.0) atomicMax(&ctl->vmax2, (unsigned long long)__double_as_longlong(m));
    }
}

// Fused step, part 2: the full arithmetic for the deferred particles, then the last block
// finalises the step (displacement bound, buffer flip, step counter, list reset).
__global__ void __launch_bounds__(kBlock) k_contact(Particles P, NbrList L, Ctl *ctl, ForceConsts fc,
                                                    const PairConst *__restrict__ pp, const PairConst *__restrict__ pw,
                                                    const WallGeom *__restrict__ walls) {
    // gate read by every thread (no barrier); a block with no deferred particle only votes
    if (ctl->steps_done >= ctl->target || (ctl->status & DEM_ERR_NEIGHBOR_OVERFLOW) || !(ctl->disp < ctl->half_skin))
        return;
    const int nd = ctl->ndefer;
    if ((long)blockIdx.x * blockDim.x >= nd) {
        finish_step_idle(ctl, fc.dt);
        return;
    }
    CtlSnap cs_;
    cs_.cur = ctl->cur;
    cs_.last = ctl->steps_done + 1 >= ctl->target;
    double vmax2 = 0.0;
    int status = 0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nd; t += gridDim.x * blockDim.x) {
        double v2 = 0.0;
        particle_full<MODE_FUSED, false>(P, L, fc, pp, pw, walls, cs_.cur, cs_.cur ^ 1, cs_.last, L.defer[t], v2, status);
        vmax2 = fmax(vmax2, v2);
    }
    finish_step(ctl, vmax2, fc.dt, status, true);
}

// Prologue of a run: stage1 + stage2 of its first step with the stored F, tau
// (src/CabanaDEM_Integrator.hpp:31-74).  Writes the next buffer and flips.
__global__ void __launch_bounds__(kBlock) k_prologue(Particles P, Ctl *ctl, ForceConsts fc) {
    const CtlSnap cs_ = read_ctl(ctl, false);
    const int cur = cs_.cur, nxt = cur ^ 1;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int cap = P.cap;
    double vmax2 = 0.0;
    if (i < P.n) {
        const double2 mIi = P.mI[i];
        const double m_inverse = 1. / mIi.x, I_inverse = 1. / mIi.y, h = fc.half_dt;
        const double *vc = P.vel[cur], *wc = P.omg[cur];
        double u[3], w[3];
        for (int d = 0; d < 3; ++d) {
            u[d] = vc[d * cap + i] + h * P.force[d * cap + i] * m_inverse;
            w[d] = wc[d * cap + i] + h * P.torque[d * cap + i] * I_inverse;
        }
        D4 p = ld4(P.pos[cur], i);
        p.x += fc.dt * u[0];
        p.y += fc.dt * u[1];
        p.z += fc.dt * u[2];
        vmax2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
        st4(P.pos[nxt], i, p);
        for (int d = 0; d < 3; ++d) {
            P.vel[nxt][d * cap + i] = u[d];
            P.omg[nxt][d * cap + i] = w[d];
        }
    }
    finish_step(ctl, vmax2, fc.dt, 0, false);
}

// Unfused Integrator stages, in place on the current buffer.
__global__ void k_stage(Particles P, Ctl *ctl, ForceConsts fc, int stage) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const int cur = ctl->cur, cap = P.cap;
    if (stage == 2) {
        D4 p = ld4(P.pos[cur], i);
        p.x += fc.dt * P.vel[cur][i];
        p.y += fc.dt * P.vel[cur][cap + i];
        p.z += fc.dt * P.vel[cur][2 * cap + i];
        st4(P.pos[cur], i, p);
        return;
    }
    const double2 mIi = P.mI[i];
    const double m_inverse = 1. / mIi.x, I_inverse = 1. / mIi.y, h = fc.half_dt;
    for (int d = 0; d < 3; ++d) {
        P.vel[cur][d * cap + i] += h * P.force[d * cap + i] * m_inverse;
        P.omg[cur][d * cap + i] += h * P.torque[d * cap + i] * I_inverse;
    }
}

// Energy totals: per-block partial sums in a fixed tree order, then one thread sums
// the block partials in block order (deterministic).
__global__ void __launch_bounds__(kBlock) k_energy_partials(Particles P, NbrList L, ForceConsts fc,
                                                            const PairConst *__restrict__ pp,
                                                            const PairConst *__restrict__ pw,
                                                            const WallGeom *__restrict__ walls, int cur,
                                                            double *partials) {
    __shared__ double red[4][kBlock];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int cap = P.cap;
    double e[4] = {0., 0., 0., 0.};
    if (i < P.n) {
        const double2 mIi = P.mI[i];
        const double *vc = P.vel[cur], *wc = P.omg[cur];
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
        for (int w = 0; w < fc.nwall; ++w) {
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

// ---------------------------------------------------------------------------------------
static inline int nblocks(int n) { return (n + kBlock - 1) / kBlock; }

void launch_prologue(const Particles &P, Ctl *ctl, const ForceConsts &fc, cudaStream_t s) {
    k_prologue<<<nblocks(P.n), kBlock, 0, s>>>(P, ctl, fc);
}

int kernels_per_step() { return 2; }

static int persistent_blocks(const void *kernel, int block, int n) {
    static int sms = 0;
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

void launch_step(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc, const PairConst *pp,
                 const PairConst *pw, const WallGeom *walls, int mode, cudaStream_t s) {
    if (mode == MODE_FUSED) {
        static int gs = 0, gc = 0, gm = 0, last_n = -1;
        if (last_n != P.n) {
            gs = persistent_blocks((const void *)k_stream, kStreamBlock, P.n);
            gc = persistent_blocks((const void *)k_contact, kBlock, P.n);
            gm = persistent_blocks(contact_mixed_kernel(), kBlock, P.n);
            last_n = P.n;
        }
        k_stream<<<gs, kStreamBlock, 0, s>>>(P, L, ctl, fc, walls);
        if (fc.mixed)
            launch_contact_mixed(P, L, ctl, fc, pp, pw, walls, gm, s);
        else
            k_contact<<<gc, kBlock, 0, s>>>(P, L, ctl, fc, pp, pw, walls);
    } else if (fc.mixed) {
        launch_force_mixed(P, L, ctl, fc, pp, pw, walls, s);
    } else {
        k_step<MODE_FORCE_ONLY><<<nblocks(P.n), kBlock, 0, s>>>(P, L, ctl, fc, pp, pw, walls);
    }
}

void launch_stage(const Particles &P, Ctl *ctl, const ForceConsts &fc, int stage, cudaStream_t s) {
    k_stage<<<nblocks(P.n), kBlock, 0, s>>>(P, ctl, fc, stage);
}

void launch_energy(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc, const PairConst *pp,
                   const PairConst *pw, const WallGeom *walls, double *partials, int nparts, double *out,
                   cudaStream_t s) {
    (void)ctl;
    // `cur` is read on the host by the caller and passed through fc-independent path
    int cur = 0;
    cudaMemcpyAsync(&cur, &ctl->cur, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    k_energy_partials<<<nparts, kBlock, 0, s>>>(P, L, fc, pp, pw, walls, cur, partials);
    k_energy_final<<<1, 32, 0, s>>>(partials, nparts, out);
}

}  // namespace b200dem
