// dem_particle.cuh -- per-particle DEM step shared by the FP64 and mixed-precision
// translation units.  dem_step.cu (built with --fmad=false) instantiates the FP64 body,
// whose every expression keeps the reference's order; dem_mixed.cu (built with FMA)
// instantiates the mixed body: contact geometry (pair distance and overlap) in FP64 on the
// FP64 positions, normal/tangential forces in FP32 on the resulting offsets, tangential
// history accumulation, force sums and integration in FP64.
#pragma once
#include "b200dem.h"
#include "dem_internal.cuh"

namespace b200dem {

namespace {

constexpr int kBlock = 128;
// Resident blocks per SM the contact kernels are compiled for (a register cap).  A sparse step
// defers few particles and prefers the uncapped kernel; when most particles are in contact the
// kernel is latency-bound and more resident warps win (B200 sweep on a dense 200k flow: FP64
// 177 -> 133 us per step at 5 blocks, mixed 120 -> 99 us at 4; the 2M lattice loses 1-3 %).
constexpr int kContactMinBlocksDense = 5;
constexpr int kContactMixedMinBlocksDense = 4;
// Resident blocks per SM of the cooperative contact kernel (register cap 128 at 128 threads).
constexpr int kCoopMinBlocks = 4;
constexpr int kApplyBlock = 256;

struct __align__(32) D4 {
    double x, y, z, w;
};

__device__ __forceinline__ D4 ld4(const double4 *p, int i) {
    const D4 *q = reinterpret_cast<const D4 *>(p);
    return q[i];
}
__device__ __forceinline__ void st4(double4 *p, int i, D4 v) { reinterpret_cast<D4 *>(p)[i] = v; }

// Read-only loads issued where they are written: volatile asm is neither sunk into a later
// branch nor merged, so all of a particle's loads are in flight together.
__device__ __forceinline__ double ld_early(const double *p) {
    double v;
    asm volatile("ld.global.nc.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ double2 ld_early2(const void *p) {
    double2 v;
    asm volatile("ld.global.nc.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
    return v;
}
__device__ __forceinline__ int ld_early_i(const int *p) {
    int v;
    asm volatile("ld.global.nc.b32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ D4 ld4_early(const double4 *p, int i) {
    const double2 a = ld_early2(reinterpret_cast<const double2 *>(p) + 2 * (long)i);
    const double2 b = ld_early2(reinterpret_cast<const double2 *>(p) + 2 * (long)i + 1);
    D4 r;
    r.x = a.x;
    r.y = a.y;
    r.z = b.x;
    r.w = b.y;
    return r;
}

// Round-to-nearest add and multiply that the compiler never contracts into an FMA: the
// gravity hook and the velocity-Verlet updates of a particle give the same bits in the FP64
// translation unit (built without contraction) and in the mixed one (built with it), so a
// particle's step does not depend on which kernel form stepped it.
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }

// L2 prefetch of a contiguous range with the TMA bulk-prefetch instruction (no registers,
// no completion to wait for).  The range is clipped to 16-byte granules inside [p, p+bytes).
__device__ __forceinline__ void prefetch_l2(const void *p, long bytes) {
    const unsigned long long a = (unsigned long long)p;
    const unsigned long long a0 = (a + 15ull) & ~15ull;
    const unsigned long long e = (a + (unsigned long long)bytes) & ~15ull;
    if (e > a0) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a0), "r"((unsigned)(e - a0)) : "memory");
}

struct CtlSnap {
    int cur, go, last;
};

// Block-uniform gate on the device control word.  Every block evaluates the same
// condition from values finalised by the previous launch.
__device__ __forceinline__ CtlSnap read_ctl(const Ctl *ctl, bool gated) {
    __shared__ CtlSnap s;
    if (threadIdx.x == 0) {
        CtlSnap c;
        c.cur = ctl->cur;
        if (gated) {
            const bool stale = !(ctl->disp < ctl->half_skin);
            c.go = (ctl->steps_done < ctl->target) && !(ctl->status & kStopBits) && !stale;
            c.last = (ctl->steps_done + 1 >= ctl->target);
        } else {
            c.go = !(ctl->status & DEM_ERR_NEIGHBOR_OVERFLOW);
            c.last = 1;
        }
        s = c;
    }
    __syncthreads();
    return s;
}

// Last-block election of a kernel: each block's thread 0 takes a ticket once the block's
// writes are done (a block barrier before it); the block with ticket gridDim.x - 1 finalises.
// The ticket is an acq_rel atomic at GPU scope: it orders the block's earlier memory
// operations before the ticket (release; the barrier extends that to the block's other
// threads), and the last block's later reads after it (acquire; its other threads follow
// through a block barrier).  The finalising block's own writes reach the next kernel at the
// kernel boundary, so neither side needs a separate fence.
__device__ __forceinline__ unsigned take_ticket(unsigned *ticket) {
    unsigned old;
    asm volatile("atom.acq_rel.gpu.add.u32 %0, [%1], 1;" : "=r"(old) : "l"(ticket) : "memory");
    return old;
}

__device__ __forceinline__ void vmax_fold(unsigned long long *slots, double m) {
    if (m > 0.0) atomicMax(&slots[(blockIdx.x % kVmaxSlots) * 32], (unsigned long long)__double_as_longlong(m));
}

// Max over the slots, clearing them for the next step: one warp, lane s takes slot s
// (kVmaxSlots == 32), one round trip.
__device__ __forceinline__ double vmax_collect_warp(unsigned long long *slots) {
    const int lane = threadIdx.x & 31;
    unsigned long long v = atomicExch(&slots[lane * 32], 0ull);
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return __longlong_as_double((long long)v);
}

// Kinematic walls and mesh: x_w += dt u_w and D += dt u (their stage2), by one full warp of the
// block that finalises a step, after every particle of the step has used the current positions.
__device__ __forceinline__ void advance_kinematics(const ForceConsts &fc) {
    if (fc.mwalls)
        for (int w = threadIdx.x & 31; w < fc.nwall; w += 32)
            for (int d = 0; d < 3; ++d) fc.mwalls[w].x[d] = dadd(fc.mwalls[w].x[d], dmul(fc.dt, fc.mwalls[w].u[d]));
    if (fc.mesh_moving && (threadIdx.x & 31) == 0)
        for (int d = 0; d < 3; ++d) fc.mesh.D[d] = dadd(fc.mesh.D[d], dmul(fc.dt, fc.mesh.u[d]));
}

// |u|^2 of the moving mesh (0 otherwise): its motion enters the displacement bound, since the
// mesh candidates of a particle are fixed between neighbour builds.
__device__ __forceinline__ double mesh_speed2(const ForceConsts &fc) {
    if (!fc.mesh_moving) return 0.0;
    return dadd(dadd(dmul(fc.mesh.u[0], fc.mesh.u[0]), dmul(fc.mesh.u[1], fc.mesh.u[1])),
                dmul(fc.mesh.u[2], fc.mesh.u[2]));
}

// Block max of |u|^2 folded into its slot, then the last block to finish advances the
// control word: disp += dt*|u|max (conservative displacement bound), flips the position
// buffer (and the velocity buffer when the kernel wrote the other one).
__device__ __forceinline__ void finish_step(Ctl *ctl, unsigned long long *slots, double vmax2, double dt, int status,
                                            bool count_step, bool flip_v = false, const ForceConsts *kin = nullptr) {
    __shared__ double red[32];
    __shared__ bool am_last;
    for (int o = 16; o > 0; o >>= 1) vmax2 = fmax(vmax2, __shfl_xor_sync(0xffffffffu, vmax2, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (status) atomicOr(&ctl->status, status);
    if (lane == 0) red[warp] = vmax2;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = red[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
        vmax_fold(slots, m);
        const unsigned t = take_ticket(&ctl->ticket);
        am_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (am_last && threadIdx.x < 32) {
        double v2 = vmax_collect_warp(slots);
        if (kin) {
            advance_kinematics(*kin);
            v2 = fmax(v2, mesh_speed2(*kin));
        }
        if (threadIdx.x == 0) {
            ctl->disp = ctl->disp + dt * sqrt(v2) * (1.0 + 1e-9);
            ctl->ndefer = 0;
            ctl->cur ^= 1;
            if (flip_v) ctl->vcur ^= 1;
            if (count_step) {
                ctl->steps_done += 1;
                ctl->total_steps += 1;
            }
            ctl->ticket = 0u;
        }
    }
}

// finish_step for the one-kernel dense step: also counts the particles in contact (`active`
// per thread; one atomic per block, added before the block's ticket) and leaves the count in last_ndefer,
// where the host reads the step's density.  Flips the position and velocity buffers.
__device__ __forceinline__ void finish_step_counted(Ctl *ctl, unsigned long long *slots, double vmax2, double dt,
                                                    int status, int active, const ForceConsts &fc, bool advance) {
    __shared__ int cnt_s[32];
    __shared__ double red[32];
    __shared__ bool am_last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int c = active;   // particles in contact among this thread's
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
    }
    __syncthreads();
    if (am_last && threadIdx.x < 32) {
        const double v2 = fmax(vmax_collect_warp(slots), mesh_speed2(fc));
        if (advance) advance_kinematics(fc);   // not on the last step of a run (no next drift)
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
        }
    }
}

// Fold the warp's largest |u|^2 into a slot chosen by the global warp index (and OR its
// status bits): no block barrier, one atomic per warp spread over the 32 slots.
__device__ __forceinline__ void warp_vmax(Ctl *ctl, unsigned long long *slots, double vmax2, int status) {
    for (int o = 16; o > 0; o >>= 1) vmax2 = fmax(vmax2, __shfl_xor_sync(0xffffffffu, vmax2, o));
    if (status) atomicOr(&ctl->status, status);
    if ((threadIdx.x & 31) == 0 && vmax2 > 0.0) {
        const unsigned w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
        atomicMax(&slots[(w % kVmaxSlots) * 32], (unsigned long long)__double_as_longlong(vmax2));
    }
}

// Fold the block's largest |u|^2 into its slot (and OR its status bits).
__device__ __forceinline__ void block_vmax(Ctl *ctl, unsigned long long *slots, double vmax2, int status) {
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) vmax2 = fmax(vmax2, __shfl_xor_sync(0xffffffffu, vmax2, o));
    if (status) atomicOr(&ctl->status, status);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = vmax2;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = red[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
        vmax_fold(slots, m);
    }
}


// One particle-particle contact of i with partner j at overlap > 0 (Force.hpp:73-329): Hertz
// normal force with damping, Mindlin tangential force with the Coulomb limit.  h is the
// tangential history (in and out); cf receives the contribution to F (0..2) and tau (3..5) of i,
// added by the caller in list order.  Shared by the per-thread and the cooperative contact
// kernels, so both evaluate every expression identically.
template <bool MIXED>
__device__ __forceinline__ void pp_pair(const double *__restrict__ mrow, const double *__restrict__ vc,
                                        const double *__restrict__ wc, const int cap, const unsigned q, const D4 &pi,
                                        const D4 &pj, const int j, const double px, const double py, const double pz,
                                        const double rij, const double overlap, const double ui0, const double ui1,
                                        const double ui2, const double wi0, const double wi1, const double wi2,
                                        const double m_i, const PairConst &c, const double K_n_pp,
                                        const double K_t_pp, const double mu_pp, const double dt, double &h0,
                                        double &h1, double &h2, double (&cf)[6]) {
    if constexpr (MIXED) {
        // Kinematics in FP64 (multiplies and adds only: the normal, the relative contact
        // velocity and its normal/tangential split, where cancellation would cost FP32 its
        // accuracy); force magnitudes -- square roots, divisions, x^1.5, Coulomb limit --
        // in FP32; history accumulation and force sums in FP64.
        const float ov = (float)overlap;
        const double inv_r = 1.0 / rij;
        const double dnx = px * inv_r, dny = py * inv_r, dnz = pz * inv_r;
        const double da_i = pi.w - 0.5 * overlap, da_j = pj.w - 0.5 * overlap;
        const double uj0 = vc[j];
        const double uj1 = (q & DEM_Q1_VELJ_USES_UI) ? ui1 : vc[cap + j];
        const double uj2 = (q & DEM_Q1_VELJ_USES_UI) ? ui2 : vc[2 * cap + j];
        const double wj0 = wc[j], wj1 = wc[cap + j], wj2 = wc[2 * cap + j];
        const double dv0 = (ui0 + (wi1 * dnz - wi2 * dny) * da_i) - (uj0 + (-wj1 * dnz + wj2 * dny) * da_j);
        const double dv1 = (ui1 + (wi2 * dnx - wi0 * dnz) * da_i) - (uj1 + (-wj2 * dnx + wj0 * dnz) * da_j);
        const double dv2 = (ui2 + (wi0 * dny - wi1 * dnx) * da_i) - (uj2 + (-wj0 * dny + wj1 * dnx) * da_j);
        const double dvdn = dv0 * dnx + dv1 * dny + dv2 * dnz;
        const float fnx = (float)dnx, fny = (float)dny, fnz = (float)dnz;
        const float fa_i = (float)da_i;
        const float ri = (float)pi.w, rj = (float)pj.w;
        const float v0 = (float)dv0, v1 = (float)dv1, v2 = (float)dv2;
        const float vdn = (float)dvdn;
        const float vt0 = (float)(dv0 - dvdn * dnx), vt1 = (float)(dv1 - dvdn * dny), vt2 = (float)(dv2 - dvdn * dnz);
        const float R_eff = 1.f / (1.f / ri + 1.f / rj);
        const float m_eff = 1.f / (1.f / (float)m_i + 1.f / (float)mrow[j]);
        const float sro = sqrtf(R_eff * ov);
        const float kn = (float)c.c_kn * sqrtf(R_eff);
        const float S_n = (float)c.c_Sn * sro;
        const float eta_n = (float)K_n_pp * sqrtf(S_n * m_eff);
        const float kt = (float)c.c_kt * sro;
        const float eta_t = (float)K_t_pp * sqrtf(kt * m_eff);
        const float fn = kn * ov * sqrtf(ov);
        const float fn0 = fn * fnx - eta_n * (vdn * fnx);
        const float fn1 = fn * fny - eta_n * (vdn * fny);
        const float fn2 = fn * fnz - eta_n * (vdn * fnz);
        float tf0 = 0.f, tf1 = 0.f, tf2 = 0.f;
        const float vij_magn = sqrtf(v0 * v0 + v1 * v1 + v2 * v2);
        if (vij_magn < 1e-12f) {
            h0 = 0.;
            h1 = 0.;
            h2 = 0.;
        } else {
            const float ti_magn = sqrtf(vt0 * vt0 + vt1 * vt1 + vt2 * vt2);
            float ti0 = 0.f, ti1 = 0.f, ti2 = 0.f;
            if (ti_magn > 1e-12f) {
                const float inv_t = 1.f / ti_magn;
                ti0 = vt0 * inv_t;
                ti1 = vt1 * inv_t;
                ti2 = vt2 * inv_t;
            }
            const double dl0 = h0 + dv0 * dt, dl1 = h1 + dv1 * dt, dl2 = h2 + dv2 * dt;
            const double dld = dl0 * (double)ti0 + dl1 * (double)ti1 + dl2 * (double)ti2;
            h0 = dld * (double)ti0;
            h1 = dld * (double)ti1;
            h2 = dld * (double)ti2;
            const float ft0 = -kt * (float)h0 - eta_t * vt0;
            const float ft1 = -kt * (float)h1 - eta_t * vt1;
            const float ft2 = -kt * (float)h2 - eta_t * vt2;
            const float ft_magn = sqrtf(ft0 * ft0 + ft1 * ft1 + ft2 * ft2);
            const float fn_magn = sqrtf(fn0 * fn0 + fn1 * fn1 + fn2 * fn2);
            const float lim = (float)mu_pp * fn_magn;
            const float fms = ft_magn > lim ? lim : ft_magn;
            tf0 = -fms * ti0;
            tf1 = -fms * ti1;
            tf2 = -fms * ti2;
            const float md0 = -tf0 / kt, md1 = -tf1 / kt, md2 = -tf2 / kt;
            if (q & DEM_Q4_UNIT_HISTORY) {
                const float lt = sqrtf(md0 * md0 + md1 * md1 + md2 * md2);
                if (lt > 1e-12f) {
                    h0 = (double)(md0 / lt);
                    h1 = (double)(md1 / lt);
                    h2 = (double)(md2 / lt);
                } else {
                    h0 = 0.;
                    h1 = 0.;
                    h2 = 0.;
                }
            } else {
                h0 = (double)md0;
                h1 = (double)md1;
                h2 = (double)md2;
            }
        }
        cf[0] = (double)(fn0 + tf0);
        cf[1] = (double)(fn1 + tf1);
        cf[2] = (double)(fn2 + tf2);
        cf[3] = (double)((fny * tf2 - fnz * tf1) * fa_i);
        cf[4] = (double)((fnz * tf0 - fnx * tf2) * fa_i);
        cf[5] = (double)((fnx * tf1 - fny * tf0) * fa_i);
    } else {
        const double a_i = pi.w - overlap / 2.;
        const double a_j = pj.w - overlap / 2.;
        const double nx = px / rij, ny = py / rij, nz = pz / rij;
        const double uj0 = vc[j];
        const double uj1 = (q & DEM_Q1_VELJ_USES_UI) ? ui1 : vc[cap + j];
        const double uj2 = (q & DEM_Q1_VELJ_USES_UI) ? ui2 : vc[2 * cap + j];
        const double wj0 = wc[j], wj1 = wc[cap + j], wj2 = wc[2 * cap + j];
        const double vi0 = ui0 + (wi1 * nz - wi2 * ny) * a_i;
        const double vi1 = ui1 + (wi2 * nx - wi0 * nz) * a_i;
        const double vi2 = ui2 + (wi0 * ny - wi1 * nx) * a_i;
        const double vj0 = uj0 + (-wj1 * nz + wj2 * ny) * a_j;
        const double vj1 = uj1 + (-wj2 * nx + wj0 * nz) * a_j;
        const double vj2 = uj2 + (-wj0 * ny + wj1 * nx) * a_j;
        const double v0 = vi0 - vj0, v1 = vi1 - vj1, v2 = vi2 - vj2;
        const double vdn = v0 * nx + v1 * ny + v2 * nz;
        const double vn0 = vdn * nx, vn1 = vdn * ny, vn2 = vdn * nz;
        const double vt0 = v0 - vn0, vt1 = v1 - vn1, vt2 = v2 - vn2;
        const double tmp_3 = 1. / pi.w;
        const double tmp_4 = 1. / pj.w;
        const double R_eff = 1. / (tmp_3 + tmp_4);
        const double kn = c.c_kn * sqrt(R_eff);
        const double S_n = c.c_Sn * sqrt(R_eff * overlap);
        const double m_eff = 1. / (1. / m_i + 1. / mrow[j]);
        const double eta_n = K_n_pp * sqrt(S_n * m_eff);
        const double kt = c.c_kt * sqrt(R_eff * overlap);
        const double eta_t = K_t_pp * sqrt(kt * m_eff);
        const double fn = kn * (overlap * sqrt(overlap));
        const double fn0 = fn * nx - eta_n * vn0;
        const double fn1 = fn * ny - eta_n * vn1;
        const double fn2 = fn * nz - eta_n * vn2;
        double tf0 = 0., tf1 = 0., tf2 = 0.;
        const double vij_magn = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
        if (vij_magn < 1e-12) {
            h0 = 0.;
            h1 = 0.;
            h2 = 0.;
        } else {
            const double tx = v0 - nx * vdn, ty = v1 - ny * vdn, tz = v2 - nz * vdn;
            const double ti_magn = sqrt(tx * tx + ty * ty + tz * tz);
            double ti0 = 0., ti1 = 0., ti2 = 0.;
            if (ti_magn > 1e-12) {
                ti0 = tx / ti_magn;
                ti1 = ty / ti_magn;
                ti2 = tz / ti_magn;
            }
            const double dl0 = h0 + v0 * dt, dl1 = h1 + v1 * dt, dl2 = h2 + v2 * dt;
            const double dld = (dl0 * ti0 + dl1 * ti1 + dl2 * ti2);
            h0 = dld * ti0;
            h1 = dld * ti1;
            h2 = dld * ti2;
            const double ft0 = -kt * h0 - eta_t * vt0;
            const double ft1 = -kt * h1 - eta_t * vt1;
            const double ft2 = -kt * h2 - eta_t * vt2;
            const double ft_magn = sqrt(ft0 * ft0 + ft1 * ft1 + ft2 * ft2);
            const double fn_magn = sqrt(fn0 * fn0 + fn1 * fn1 + fn2 * fn2);
            double fms = ft_magn;
            if (fms > mu_pp * fn_magn) fms = mu_pp * fn_magn;
            tf0 = -fms * ti0;
            tf1 = -fms * ti1;
            tf2 = -fms * ti2;
            const double md0 = -tf0 / kt, md1 = -tf1 / kt, md2 = -tf2 / kt;
            if (q & DEM_Q4_UNIT_HISTORY) {
                const double lt = sqrt(md0 * md0 + md1 * md1 + md2 * md2);
                if (lt > 1e-12) {
                    h0 = md0 / lt;
                    h1 = md1 / lt;
                    h2 = md2 / lt;
                } else {
                    h0 = 0.;
                    h1 = 0.;
                    h2 = 0.;
                }
            } else {
                h0 = md0;
                h1 = md1;
                h2 = md2;
            }
        }
        cf[0] = fn0 + tf0;
        cf[1] = fn1 + tf1;
        cf[2] = fn2 + tf2;
        cf[3] = (ny * tf2 - nz * tf1) * a_i;
        cf[4] = (nz * tf0 - nx * tf2) * a_i;
        cf[5] = (nx * tf1 - ny * tf0) * a_i;
    }
}

// One particle-wall contact at overlap > 0 (Force.hpp:475-673): forces of the infinite wall with
// normal (nx, ny, nz) on i, the wall history (swx, swy, swz) read when has_hist and written;
// cf as for pp_pair.
template <bool MIXED>
__device__ __forceinline__ void pw_wall(const unsigned q, const D4 &pi, const double nx, const double ny,
                                        const double nz, const double overlap, const double ui0, const double ui1,
                                        const double ui2, const double wi0, const double wi1, const double wi2,
                                        const double uw0, const double uw1, const double uw2,
                                        const double m_i, const PairConst &c, const double K_n_pw,
                                        const double K_t_pw, const double mu_pw, const double dt,
                                        const bool has_hist, double *swx, double *swy, double *swz,
                                        double (&cf)[6]) {
    if constexpr (MIXED) {
        const float ov = (float)overlap;
        const double da_i = pi.w - 0.5 * overlap;
        const double dv0 = ui0 + (wi1 * nz - wi2 * ny) * da_i - uw0;
        const double dv1 = ui1 + (wi2 * nx - wi0 * nz) * da_i - uw1;
        const double dv2 = ui2 + (wi0 * ny - wi1 * nx) * da_i - uw2;
        const double dvdn = dv0 * nx + dv1 * ny + dv2 * nz;
        const float fa_i = (float)da_i;
        const float gx = (float)nx, gy = (float)ny, gz = (float)nz;
        const float v0 = (float)dv0, v1 = (float)dv1, v2 = (float)dv2;
        const float vdn = (float)dvdn;
        const float vt0 = (float)(dv0 - dvdn * nx), vt1 = (float)(dv1 - dvdn * ny), vt2 = (float)(dv2 - dvdn * nz);
        const float R_eff = (float)pi.w;
        const float m_eff = (float)m_i;
        const float sro = sqrtf(R_eff * ov);
        const float kn = (float)c.c_kn * sqrtf(R_eff);
        const float S_n = (float)c.c_Sn * sro;
        const float eta_n = (float)K_n_pw * sqrtf(S_n * m_eff);
        const float fn = kn * ov * sqrtf(ov);
        const float fn0 = fn * gx - eta_n * (vdn * gx);
        const float fn1 = fn * gy - eta_n * (vdn * gy);
        const float fn2 = fn * gz - eta_n * (vdn * gz);
        float ft0 = 0.f, ft1 = 0.f, ft2 = 0.f;
        const float vij_magn = sqrtf(v0 * v0 + v1 * v1 + v2 * v2);
        if (vij_magn < 1e-12f) {
            *swx = 0.;
            *swy = 0.;
            *swz = 0.;
        } else {
            double s0 = 0., s1 = 0., s2 = 0.;
            if (has_hist) {
                s0 = *swx;
                s1 = *swy;
                s2 = *swz;
            }
            s0 += (dv0 - dvdn * nx) * dt;
            s1 += (dv1 - dvdn * ny) * dt;
            s2 += (dv2 - dvdn * nz) * dt;
            const float kt = (float)c.c_kt * sro;
            const float eta_t = (float)K_t_pw * sqrtf(kt * m_eff);
            const float fx = -kt * (float)s0 - eta_t * vt0;
            const float fy = -kt * (float)s1 - eta_t * vt1;
            const float fz = -kt * (float)s2 - eta_t * vt2;
            const float ft_magn = (q & DEM_Q5_WALL_FT_TYPO) ? sqrtf(fx * fx + fy * fy + fz * fy)
                                                             : sqrtf(fx * fx + fy * fy + fz * fz);
            float ti0 = 0.f, ti1 = 0.f, ti2 = 0.f;
            if (ft_magn > 1e-12f) {
                ti0 = fx / ft_magn;
                ti1 = fy / ft_magn;
                ti2 = fz / ft_magn;
            }
            const float fn_magn = sqrtf(fn0 * fn0 + fn1 * fn1 + fn2 * fn2);
            const float lim = (float)mu_pw * fn_magn;
            const float fms = (ft_magn < lim) ? ft_magn : lim;
            ft0 = fms * ti0 + eta_t * vt0;
            ft1 = fms * ti1 + eta_t * vt1;
            ft2 = fms * ti2 + eta_t * vt2;
            *swx = (double)(-ft0 / kt);
            *swy = (double)(-ft1 / kt);
            *swz = (double)(-ft2 / kt);
            if (!(q & DEM_Q2_ETA_T_ZERO)) {   // as the FP64 branch: the limited force acts
                ft0 = __fmul_rn(fms, ti0);
                ft1 = __fmul_rn(fms, ti1);
                ft2 = __fmul_rn(fms, ti2);
            }
        }
        cf[0] = (double)(fn0 + ft0);
        cf[1] = (double)(fn1 + ft1);
        cf[2] = (double)(fn2 + ft2);
        cf[3] = (double)((gy * ft2 - gz * ft1) * fa_i);
        cf[4] = (double)((gz * ft0 - gx * ft2) * fa_i);
        cf[5] = (double)((gx * ft1 - gy * ft0) * fa_i);
    } else {
        const double a_i = pi.w - overlap / 2.;
        // contact-point velocity minus the wall's (vel_i - vel_j, Force.hpp:529-533)
        const double v0 = ui0 + (wi1 * nz - wi2 * ny) * a_i - uw0;
        const double v1 = ui1 + (wi2 * nx - wi0 * nz) * a_i - uw1;
        const double v2 = ui2 + (wi0 * ny - wi1 * nx) * a_i - uw2;
        const double vdn = v0 * nx + v1 * ny + v2 * nz;
        const double vt0 = v0 - vdn * nx, vt1 = v1 - vdn * ny, vt2 = v2 - vdn * nz;
        const double R_eff = 1. / (1. / pi.w + 0.);
        const double kn = c.c_kn * sqrt(R_eff);
        const double S_n = c.c_Sn * sqrt(R_eff * overlap);
        const double m_eff = 1. / (1. / m_i + 0.);
        const double eta_n = K_n_pw * sqrt(S_n * m_eff);
        const double fn = kn * (overlap * sqrt(overlap));
        const double fn0 = fn * nx - eta_n * (vdn * nx);
        const double fn1 = fn * ny - eta_n * (vdn * ny);
        const double fn2 = fn * nz - eta_n * (vdn * nz);
        double ft0 = 0., ft1 = 0., ft2 = 0.;
        const double vij_magn = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
        if (vij_magn < 1e-12) {
            *swx = 0.;
            *swy = 0.;
            *swz = 0.;
        } else {
            double s0 = 0., s1 = 0., s2 = 0.;
            if (has_hist) {
                s0 = *swx;
                s1 = *swy;
                s2 = *swz;
            }
            s0 += vt0 * dt;
            s1 += vt1 * dt;
            s2 += vt2 * dt;
            const double kt = c.c_kt * sqrt(R_eff * overlap);
            const double eta_t = K_t_pw * sqrt(kt * m_eff);
            const double fx = -kt * s0 - eta_t * vt0;
            const double fy = -kt * s1 - eta_t * vt1;
            const double fz = -kt * s2 - eta_t * vt2;
            const double ft_magn = (q & DEM_Q5_WALL_FT_TYPO) ? sqrt(fx * fx + fy * fy + fz * fy)
                                                              : sqrt(fx * fx + fy * fy + fz * fz);
            double ti0 = 0., ti1 = 0., ti2 = 0.;
            if (ft_magn > 1e-12) {
                ti0 = fx / ft_magn;
                ti1 = fy / ft_magn;
                ti2 = fz / ft_magn;
            }
            const double fn_magn = sqrt(fn0 * fn0 + fn1 * fn1 + fn2 * fn2);
            const double lim = mu_pw * fn_magn;
            const double fms = (ft_magn < lim) ? ft_magn : lim;  // std::min(lim, ft_magn)
            ft0 = fms * ti0;
            ft1 = fms * ti1;
            ft2 = fms * ti2;
            ft0 += eta_t * vt0;
            ft1 += eta_t * vt1;
            ft2 += eta_t * vt2;
            *swx = -ft0 / kt;
            *swy = -ft1 / kt;
            *swz = -ft2 / kt;
            if (!(q & DEM_Q2_ETA_T_ZERO)) {
                // with eta_t live (Q2 clear) the limited force is what acts; the damping is
                // added back (Force.hpp:640-643) only to reset the spring above.  The reference
                // applies the sum, which pushes a sliding contact along its sliding direction.
                ft0 = fms * ti0;
                ft1 = fms * ti1;
                ft2 = fms * ti2;
            }
        }
        cf[0] = fn0 + ft0;
        cf[1] = fn1 + ft1;
        cf[2] = fn2 + ft2;
        cf[3] = (ny * ft2 - nz * ft1) * a_i;
        cf[4] = (nz * ft0 - nx * ft2) * a_i;
        cf[5] = (nx * ft1 - ny * ft0) * a_i;
    }
}

// ---------------------------------------------------------------------------------------
// Triangle-mesh wall (no reference counterpart).  Closest point of triangle (a, b, c) to p:
// the Voronoi-region method of Ericson, Real-Time Collision Detection (2005), sec. 5.1.5;
// feature 0 face interior, 1 edge, 2 vertex.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void tri_closest(const double p[3], const double a[3], const double b[3], const double c[3],
                                            double out[3], int &feature) {
    double ab[3], ac[3], ap[3];
    for (int d = 0; d < 3; ++d) {
        ab[d] = b[d] - a[d];
        ac[d] = c[d] - a[d];
        ap[d] = p[d] - a[d];
    }
    const double d1 = ab[0] * ap[0] + ab[1] * ap[1] + ab[2] * ap[2];
    const double d2 = ac[0] * ap[0] + ac[1] * ap[1] + ac[2] * ap[2];
    if (d1 <= 0. && d2 <= 0.) {
        for (int d = 0; d < 3; ++d) out[d] = a[d];
        feature = 2;
        return;
    }
    double bp[3];
    for (int d = 0; d < 3; ++d) bp[d] = p[d] - b[d];
    const double d3 = ab[0] * bp[0] + ab[1] * bp[1] + ab[2] * bp[2];
    const double d4 = ac[0] * bp[0] + ac[1] * bp[1] + ac[2] * bp[2];
    if (d3 >= 0. && d4 <= d3) {
        for (int d = 0; d < 3; ++d) out[d] = b[d];
        feature = 2;
        return;
    }
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0. && d1 >= 0. && d3 <= 0.) {
        const double v = d1 / (d1 - d3);
        for (int d = 0; d < 3; ++d) out[d] = a[d] + v * ab[d];
        feature = 1;
        return;
    }
    double cp[3];
    for (int d = 0; d < 3; ++d) cp[d] = p[d] - c[d];
    const double d5 = ab[0] * cp[0] + ab[1] * cp[1] + ab[2] * cp[2];
    const double d6 = ac[0] * cp[0] + ac[1] * cp[1] + ac[2] * cp[2];
    if (d6 >= 0. && d5 <= d6) {
        for (int d = 0; d < 3; ++d) out[d] = c[d];
        feature = 2;
        return;
    }
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0. && d2 >= 0. && d6 <= 0.) {
        const double w = d2 / (d2 - d6);
        for (int d = 0; d < 3; ++d) out[d] = a[d] + w * ac[d];
        feature = 1;
        return;
    }
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0. && (d4 - d3) >= 0. && (d5 - d6) >= 0.) {
        const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        for (int d = 0; d < 3; ++d) out[d] = b[d] + w * (c[d] - b[d]);
        feature = 1;
        return;
    }
    const double denom = 1. / (va + vb + vc);
    const double v = vb * denom, w = vc * denom;
    for (int d = 0; d < 3; ++d) out[d] = a[d] + ab[d] * v + ac[d] * w;
    feature = 0;
}

__device__ __forceinline__ void mesh_vertices(const MeshDev &M, int t, const double D[3], double a[3], double b[3],
                                              double c[3]) {
    const double *v = M.tri + 9L * t;
    for (int d = 0; d < 3; ++d) {
        a[d] = v[d] + D[d];
        b[d] = v[3 + d] + D[d];
        c[d] = v[6 + d] + D[d];
    }
}

// Contacts of particle i with the mesh, over its candidates in triangle order: contacts at
// 0 < d < r (d = distance to the closest point); face contacts kept, an edge or vertex
// contact dropped when its point coincides (1e-9 r) with a kept contact's or lies on a
// triangle with a face contact; tracked slots: the still-live slots in their order, then the
// new contacts with zero history; each kept contact acts as a plane through its point with
// normal (x - c)/d (pw_wall), added in triangle order.  Returns the tracked count.  Not
// inlined: particles away from the mesh never enter it.
template <bool MIXED>
__device__ __noinline__ int mesh_pass(const Particles &P, const ForceConsts &fc, const int i, const D4 pi,
                                      const double ui0, const double ui1, const double ui2, const double wi0,
                                      const double wi1, const double wi2, const double m_i, const int mi,
                                      const double K_n_pw, const double K_t_pw, const double mu_pw, double *FT,
                                      int *status) {
    const MeshDev &M = fc.mesh;
    const int cap = P.cap, mt = M.mt;
    const int nc = M.ncand[i], cnt0 = M.cnt[i];
    if (nc == 0 && cnt0 == 0) return 0;
    const double r = pi.w;
    const double x[3] = {pi.x, pi.y, pi.z};
    const double D[3] = {M.D[0], M.D[1], M.D[2]};
    int ht[kMeshCand], hf[kMeshCand];
    double hc[kMeshCand][3], hd[kMeshCand], ho[kMeshCand];
    bool keep[kMeshCand];
    int nh = 0;
    for (int k = 0; k < nc; ++k) {
        const int t = M.cand[(long)k * cap + i];
        double a[3], b[3], c[3], q[3];
        int f;
        mesh_vertices(M, t, D, a, b, c);
        tri_closest(x, a, b, c, q, f);
        const double dx = x[0] - q[0], dy = x[1] - q[1], dz = x[2] - q[2];
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (!(d2 < r * r) || !(d2 > 0.)) continue;
        const double d = sqrt(d2);
        const double overlap = r - d;
        if (!(overlap > 0.)) continue;
        ht[nh] = t;
        hf[nh] = f;
        hc[nh][0] = q[0];
        hc[nh][1] = q[1];
        hc[nh][2] = q[2];
        hd[nh] = d;
        ho[nh] = overlap;
        ++nh;
    }
    const double eps = 1e-9 * r, eps2 = eps * eps;
    for (int h = 0; h < nh; ++h) keep[h] = hf[h] == 0;
    for (int h = 0; h < nh; ++h) {
        if (hf[h] == 0) continue;
        bool drop = false;
        for (int k = 0; k < nh && !drop; ++k) {
            if (k == h || !keep[k]) continue;
            const double ex = hc[h][0] - hc[k][0], ey = hc[h][1] - hc[k][1], ez = hc[h][2] - hc[k][2];
            if (ex * ex + ey * ey + ez * ez <= eps2) drop = true;
            if (!drop && hf[k] == 0) {
                double a[3], b[3], c[3], q[3];
                int f;
                mesh_vertices(M, ht[k], D, a, b, c);
                tri_closest(hc[h], a, b, c, q, f);
                const double fx = hc[h][0] - q[0], fy = hc[h][1] - q[1], fz = hc[h][2] - q[2];
                if (fx * fx + fy * fy + fz * fz <= eps2) drop = true;
            }
        }
        keep[h] = !drop;
    }
    // tracked slots: live slots in order, then new contacts in triangle order
    int *tid = M.tid + i;
    double *thx = M.th + i, *thy = M.th + (long)mt * cap + i, *thz = M.th + 2L * mt * cap + i;
    int ntid[kMeshMaxContacts];
    double n0[kMeshMaxContacts], n1[kMeshMaxContacts], n2[kMeshMaxContacts];
    int cnt1 = 0;
    for (int s2 = 0; s2 < cnt0; ++s2) {
        const int t = tid[(long)s2 * cap];
        bool live = false;
        for (int h = 0; h < nh; ++h)
            if (keep[h] && ht[h] == t) live = true;
        if (live) {
            ntid[cnt1] = t;
            n0[cnt1] = thx[(long)s2 * cap];
            n1[cnt1] = thy[(long)s2 * cap];
            n2[cnt1] = thz[(long)s2 * cap];
            ++cnt1;
        }
    }
    const int kept_old = cnt1;
    for (int h = 0; h < nh; ++h) {
        if (!keep[h]) continue;
        bool found = false;
        for (int s2 = 0; s2 < cnt1; ++s2)
            if (ntid[s2] == ht[h]) found = true;
        if (found) continue;
        if (cnt1 < mt) {
            ntid[cnt1] = ht[h];
            n0[cnt1] = n1[cnt1] = n2[cnt1] = 0.;
            ++cnt1;
        } else {
            *status |= DEM_ERR_CONTACT_OVERFLOW;
        }
    }
    for (int s2 = 0; s2 < mt; ++s2) {
        const long a = (long)s2 * cap;
        tid[a] = s2 < cnt1 ? ntid[s2] : -1;
        thx[a] = s2 < cnt1 ? n0[s2] : 0.;
        thy[a] = s2 < cnt1 ? n1[s2] : 0.;
        thz[a] = s2 < cnt1 ? n2[s2] : 0.;
    }
    M.cnt[i] = (unsigned char)cnt1;
    // forces, in triangle order
    const PairConst c = M.pm[mi];
    for (int h = 0; h < nh; ++h) {
        if (!keep[h]) continue;
        int slot = -1;
        for (int s2 = 0; s2 < cnt1; ++s2)
            if (ntid[s2] == ht[h]) slot = s2;
        double dummy[3] = {0., 0., 0.};
        double *sx = slot >= 0 ? thx + (long)slot * cap : dummy, *sy = slot >= 0 ? thy + (long)slot * cap : dummy + 1,
               *sz = slot >= 0 ? thz + (long)slot * cap : dummy + 2;
        const double d = hd[h];
        const double nx = (x[0] - hc[h][0]) / d, ny = (x[1] - hc[h][1]) / d, nz = (x[2] - hc[h][2]) / d;
        double cf[6];
        pw_wall<MIXED>(fc.quirks, pi, nx, ny, nz, ho[h], ui0, ui1, ui2, wi0, wi1, wi2, M.u[0], M.u[1], M.u[2], m_i, c,
                       K_n_pw, K_t_pw, mu_pw, fc.dt, slot >= 0 && slot < kept_old, sx, sy, sz, cf);
        for (int k = 0; k < 6; ++k) FT[k] += cf[k];
    }
    return cnt1;
}

// ---------------------------------------------------------------------------------------
// Full per-particle step (contact compaction, pp and wall forces, hooks, integration).
// MODE_FORCE_ONLY writes F and tau in place and leaves x, u, omega untouched (the
// unfused reference-order path); MODE_FUSED integrates into the next buffer.
// ---------------------------------------------------------------------------------------
// MESH: the solver has a triangle mesh (a separate build, so that meshless steps carry no call).
// GLOBAL: the particle arrays are in global memory (the early list and slot loads take the
// read-only path); false when they are a scene's copy in shared memory (generic loads).
template <int MODE, bool MIXED, bool MESH = false, bool GLOBAL = true>
__device__ __forceinline__ void particle_full(const Particles &P, const NbrList &L, const ForceConsts &fc,
                                              const PairConst *__restrict__ pp, const PairConst *__restrict__ pw,
                                              const WallGeom *__restrict__ walls, const int cur, const int nxt,
                                              const int vcur, const int last, const int i, const int slot,
                                              double &vmax2, int &status, int *active = nullptr) {
    const int cap = P.cap;
    const unsigned q = fc.quirks;
    // batched scenes: this particle's scene supplies damping, friction and its walls
    const int scene_i = P.scene ? P.scene[i] : 0;
    const SceneConst *scn = fc.scenes ? fc.scenes + scene_i : nullptr;
    const double K_n_pp = scn ? scn->K_n_pp : fc.K_n_pp, K_t_pp = scn ? scn->K_t_pp : fc.K_t_pp;
    const double K_n_pw = scn ? scn->K_n_pw : fc.K_n_pw, K_t_pw = scn ? scn->K_t_pw : fc.K_t_pw;
    const double mu_pp = scn ? scn->mu_pp : fc.mu_pp, mu_pw = scn ? scn->mu_pw : fc.mu_pw;
    const int wall0 = fc.wps ? scene_i * fc.wps : 0;
    const int wall1 = fc.wps ? wall0 + fc.wps : fc.nwall;
    const double4 *__restrict__ pc = P.pos[cur];
    const double *__restrict__ vc = P.vel[vcur];
    const double *__restrict__ wc = P.omg[vcur];
    // Speculative partner prefetch, issued with the particle's own loads: the first two
    // neighbour-list slots and the first two contact-history slots, then those partners'
    // positions.  Slots past the list length or count hold stale values; an index outside
    // [0, n) falls back to i, and a prefetched position is used only while its slot still
    // holds the same partner, so the arithmetic is that of the plain loop.
    int lpf0 = L.maxnb > 0 ? (GLOBAL ? ld_early_i(L.idx + i) : L.idx[i]) : i;
    int lpf1 = L.maxnb > 1 ? (GLOBAL ? ld_early_i(L.idx + cap + i) : L.idx[cap + i]) : i;
    int tpf0 = P.mc > 0 ? (GLOBAL ? ld_early_i(P.tidx + i) : P.tidx[i]) : i;
    int tpf1 = P.mc > 1 ? (GLOBAL ? ld_early_i(P.tidx + cap + i) : P.tidx[cap + i]) : i;
    lpf0 = (unsigned)lpf0 < (unsigned)P.n ? lpf0 : i;
    lpf1 = (unsigned)lpf1 < (unsigned)P.n ? lpf1 : i;
    tpf0 = (unsigned)tpf0 < (unsigned)P.n ? tpf0 : i;
    tpf1 = (unsigned)tpf1 < (unsigned)P.n ? tpf1 : i;
    const D4 lpp0 = ld4(pc, lpf0), lpp1 = ld4(pc, lpf1), tpp0 = ld4(pc, tpf0), tpp1 = ld4(pc, tpf1);
    const D4 pi = ld4(pc, i);
    double ui0 = vc[i], ui1 = vc[cap + i], ui2 = vc[2 * cap + i];
    double wi0 = wc[i], wi1 = wc[cap + i], wi2 = wc[2 * cap + i];
    const double2 mIi = load_mI(P, i);
    const int mi = fc.nmat > 1 ? (int)P.mat[i] : 0;
    const int cs0 = P.cstate[i];
    int cnt = cs0 & 0xff;
    unsigned wmask = (unsigned)cs0 >> 8;
    int *tidx = P.tidx + i;
    double *thx = P.th + i;
    double *thy = P.th + (long)P.mc * cap + i;
    double *thz = P.th + 2L * P.mc * cap + i;
    double F0 = 0., F1 = 0., F2 = 0., T0 = 0., T1 = 0., T2 = 0.;
    if (fc.has_ext) {
        F0 += P.ext[i];
        F1 += P.ext[cap + i];
        F2 += P.ext[2 * cap + i];
    }
    // ---- update_tangential_contacts (Force.hpp:364-441)
    if (cnt > 0) {
        int count = 0, k = 0;
        const int total = cnt;
        int last_idx_tmp = cnt - 1;
        while (count < total) {
            const int sidx = tidx[(long)k * cap];
            if (sidx == -1) break;
            const D4 pj = (k == 0 && sidx == tpf0) ? tpp0 : (k == 1 && sidx == tpf1) ? tpp1 : ld4(pc, sidx);
            const double px = pi.x - pj.x, py = pi.y - pj.y, pz = pi.z - pj.z;
            const double r2ij = px * px + py * py + pz * pz;
            const double rij = sqrt(r2ij);
            const double overlap = pi.w + pj.w - rij;
            if (overlap <= 0.) {
                const long a = (long)k * cap, b = (long)last_idx_tmp * cap;
                if (k == last_idx_tmp) {
                    tidx[a] = -1;
                    thx[a] = 0.;
                    thy[a] = 0.;
                    thz[a] = 0.;
                } else {
                    tidx[a] = tidx[b];
                    tidx[b] = -1;
                    thx[a] = thx[b];
                    thx[b] = 0.;
                    thy[a] = thy[b];
                    thy[b] = 0.;
                    thz[a] = thz[b];
                    thz[b] = 0.;
                    last_idx_tmp -= 1;
                }
                cnt -= 1;
            } else {
                k = k + 1;
            }
            count += 1;
        }
    }
    // ---- particle-particle (Force.hpp:73-329), list in ascending caller index
    const int nn = L.nn[i];
    const int *__restrict__ lidx = L.idx + i;
    for (int kk = 0; kk < nn; ++kk) {
        const int j = lidx[(long)kk * cap];
        const D4 pj = (kk == 0 && j == lpf0) ? lpp0 : (kk == 1 && j == lpf1) ? lpp1 : ld4(pc, j);
        const double px = pi.x - pj.x, py = pi.y - pj.y, pz = pi.z - pj.z;
        const double r2ij = px * px + py * py + pz * pz;
        const double sr = pi.w + pj.w;
        // exact early-out: r2 >= s^2 (1 + 1e-10) implies sqrt(r2) >= s, overlap <= 0
        if (r2ij >= sr * sr * 1.0000000001) continue;
        const double rij = sqrt(r2ij);
        const double overlap = sr - rij;
        if (!(overlap > 0.)) continue;
        // slot lookup / insert (Force.hpp:166-192)
        int found_at = -1;
        for (int s = 0; s < cnt; ++s)
            if (tidx[(long)s * cap] == j) found_at = s;
        double h0 = 0., h1 = 0., h2 = 0.;
        if (found_at < 0) {
            if (cnt < P.mc) {
                found_at = cnt;
                cnt += 1;
                const long a = (long)found_at * cap;
                tidx[a] = j;
                thx[a] = 0.;
                thy[a] = 0.;
                thz[a] = 0.;
            } else {
                status |= DEM_ERR_CONTACT_OVERFLOW;
            }
        } else {
            const long a = (long)found_at * cap;
            h0 = thx[a];
            h1 = thy[a];
            h2 = thz[a];
        }
        const int mj = fc.nmat > 1 ? (int)P.mat[j] : 0;
        const PairConst c = pp[mi * fc.nmat + mj];
        double cf[6];
        pp_pair<MIXED>(P.mI, vc, wc, cap, q, pi, pj, j, px, py, pz, rij, overlap, ui0, ui1, ui2, wi0, wi1, wi2, mIi.x, c,
                       K_n_pp, K_t_pp, mu_pp, fc.dt, h0, h1, h2, cf);
        if (found_at >= 0) {
            const long a = (long)found_at * cap;
            thx[a] = h0;
            thy[a] = h1;
            thz[a] = h2;
        }
        F0 += cf[0];
        F1 += cf[1];
        F2 += cf[2];
        if (!(q & DEM_Q3_NO_PP_TORQUE)) {
            T0 += cf[3];
            T1 += cf[4];
            T2 += cf[5];
        }
    }
    // ---- particle-infinite wall (Force.hpp:475-673)
    for (int w = wall0; w < wall1; ++w) {
        const WallGeom g = walls[w];
        const int lw = w - wall0;   // this particle's wall slot
        const double px = pi.x - g.x[0], py = pi.y - g.x[1], pz = pi.z - g.x[2];
        const double nx = g.n[0], ny = g.n[1], nz = g.n[2];
        const double tmp = px * nx + py * ny + pz * nz;
        const double overlap = pi.w - tmp;
        const unsigned bit = 1u << lw;
        double *swx = P.sw + (long)lw * cap + i;
        double *swy = P.sw + (long)(P.mw + lw) * cap + i;
        double *swz = P.sw + (long)(2 * P.mw + lw) * cap + i;
        if (overlap > 0.) {
            double cf[6];
            pw_wall<MIXED>(q, pi, nx, ny, nz, overlap, ui0, ui1, ui2, wi0, wi1, wi2, g.u[0], g.u[1], g.u[2], mIi.x,
                           pw[mi * fc.nwall + w], K_n_pw, K_t_pw, mu_pw, fc.dt, (wmask & bit) != 0u, swx, swy, swz, cf);
            wmask |= bit;
            F0 += cf[0];
            F1 += cf[1];
            F2 += cf[2];
            T0 += cf[3];
            T1 += cf[4];
            T2 += cf[5];
        } else if (wmask & bit) {
            *swx = 0.;
            *swy = 0.;
            *swz = 0.;
            wmask &= ~bit;
        }
    }
    int mcnt = 0;
    if constexpr (MESH) {
        double FT[6] = {F0, F1, F2, T0, T1, T2};
        mcnt = mesh_pass<MIXED>(P, fc, i, pi, ui0, ui1, ui2, wi0, wi1, wi2, mIi.x, mi, K_n_pw, K_t_pw, mu_pw, FT,
                                &status);
        F0 = FT[0];
        F1 = FT[1];
        F2 = FT[2];
        T0 = FT[3];
        T1 = FT[4];
        T2 = FT[5];
    }
    const int cs1 = cnt | (int)(wmask << 8);
    if (cs1 != cs0) P.cstate[i] = cs1;
    if (active) *active = (cs0 | cs1) != 0 || mcnt != 0;
    // ---- hooks after the pair forces
    if (fc.has_gravity) {
        F0 = dadd(F0, dmul(mIi.x, fc.g[0]));
        F1 = dadd(F1, dmul(mIi.x, fc.g[1]));
        F2 = dadd(F2, dmul(mIi.x, fc.g[2]));
    }
    if (fc.has_fix) {
        const int f = P.fix[i];
        if (f & DEM_FIX_FORCE) F0 = F1 = F2 = 0.;
        if (f & DEM_FIX_TORQUE) T0 = T1 = T2 = 0.;
    }
    if (MODE == MODE_FORCE_ONLY) {
        P.force[i] = F0;
        P.force[cap + i] = F1;
        P.force[2 * cap + i] = F2;
        P.torque[i] = T0;
        P.torque[cap + i] = T1;
        P.torque[2 * cap + i] = T2;
    } else {
        const double m_inverse = 1. / mIi.x;
        const double I_inverse = 1. / mIi.y;
        const double h = fc.half_dt;
        // stage3 of this step
        ui0 = dadd(ui0, dmul(dmul(h, F0), m_inverse));
        ui1 = dadd(ui1, dmul(dmul(h, F1), m_inverse));
        ui2 = dadd(ui2, dmul(dmul(h, F2), m_inverse));
        wi0 = dadd(wi0, dmul(dmul(h, T0), I_inverse));
        wi1 = dadd(wi1, dmul(dmul(h, T1), I_inverse));
        wi2 = dadd(wi2, dmul(dmul(h, T2), I_inverse));
        D4 pn = pi;
        if (last) {
            P.force[i] = F0;
            P.force[cap + i] = F1;
            P.force[2 * cap + i] = F2;
            P.torque[i] = T0;
            P.torque[cap + i] = T1;
            P.torque[2 * cap + i] = T2;
        } else {
            // stage1 + stage2 of the next step
            ui0 = dadd(ui0, dmul(dmul(h, F0), m_inverse));
            ui1 = dadd(ui1, dmul(dmul(h, F1), m_inverse));
            ui2 = dadd(ui2, dmul(dmul(h, F2), m_inverse));
            wi0 = dadd(wi0, dmul(dmul(h, T0), I_inverse));
            wi1 = dadd(wi1, dmul(dmul(h, T1), I_inverse));
            wi2 = dadd(wi2, dmul(dmul(h, T2), I_inverse));
            pn.x = dadd(pn.x, dmul(fc.dt, ui0));
            pn.y = dadd(pn.y, dmul(fc.dt, ui1));
            pn.z = dadd(pn.z, dmul(fc.dt, ui2));
            vmax2 = dadd(dadd(dmul(ui0, ui0), dmul(ui1, ui1)), dmul(ui2, ui2));
        }
        // positions go to the next buffer; u and omega to this particle's scratch slot,
        // committed by the apply kernel once no thread reads the current values any more
        // (MODE_FUSED), or straight to the other velocity buffer when one kernel steps every
        // particle (MODE_FUSED_DIRECT, slot = i)
        st4(P.pos[nxt], i, pn);
        double *vn = MODE == MODE_FUSED_DIRECT ? P.vel[vcur ^ 1] : L.defer_v;
        double *wn = MODE == MODE_FUSED_DIRECT ? P.omg[vcur ^ 1] : L.defer_w;
        vn[slot] = ui0;
        vn[cap + slot] = ui1;
        vn[2 * cap + slot] = ui2;
        wn[slot] = wi0;
        wn[cap + slot] = wi1;
        wn[2 * cap + slot] = wi2;
    }
    }


}  // namespace
}  // namespace b200dem
