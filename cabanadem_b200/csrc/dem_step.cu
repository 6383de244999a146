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

namespace b200dem {

namespace {

constexpr int kBlock = 128;
constexpr int kStreamBlock = 256;

struct __align__(32) D4 {
    double x, y, z, w;
};

__device__ __forceinline__ D4 ld4(const double4 *p, int i) {
    const D4 *q = reinterpret_cast<const D4 *>(p);
    return q[i];
}
__device__ __forceinline__ void st4(double4 *p, int i, D4 v) { reinterpret_cast<D4 *>(p)[i] = v; }

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
            c.go = (ctl->steps_done < ctl->target) && !(ctl->status & DEM_ERR_NEIGHBOR_OVERFLOW) && !stale;
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

// Block max of |u|^2, then the last block to finish advances the control word:
// disp += dt*|u|max (conservative displacement bound), flips the ping-pong buffer.
__device__ __forceinline__ void finish_step(Ctl *ctl, double vmax2, double dt, int status, bool count_step) {
    __shared__ double red[kBlock / 32];
    __shared__ bool am_last;
    for (int o = 16; o > 0; o >>= 1) vmax2 = fmax(vmax2, __shfl_xor_sync(0xffffffffu, vmax2, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (status) atomicOr(&ctl->status, status);
    if (lane == 0) red[warp] = vmax2;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = red[0];
        for (int w = 1; w < kBlock / 32; ++w) m = fmax(m, red[w]);
        atomicMax(&ctl->vmax2, (unsigned long long)__double_as_longlong(m));
        __threadfence();
        const unsigned t = atomicAdd(&ctl->ticket, 1u);
        am_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (am_last && threadIdx.x == 0) {
        __threadfence();
        const double v2 = __longlong_as_double((long long)atomicAdd(&ctl->vmax2, 0ull));
        ctl->disp = ctl->disp + dt * sqrt(v2) * (1.0 + 1e-9);
        ctl->vmax2 = 0ull;
        ctl->ndefer = 0;
        ctl->cur ^= 1;
        if (count_step) {
            ctl->steps_done += 1;
            ctl->total_steps += 1;
        }
        __threadfence();
        ctl->ticket = 0u;
    }
}

}  // namespace

// ---------------------------------------------------------------------------------------
// Full per-particle step (contact compaction, pp and wall forces, hooks, integration).
// MODE_FORCE_ONLY writes F and tau in place and leaves x, u, omega untouched (the
// unfused reference-order path); MODE_FUSED integrates into the next buffer.
// ---------------------------------------------------------------------------------------
template <int MODE>
__device__ __forceinline__ void particle_full(const Particles &P, const NbrList &L, const ForceConsts &fc,
                                              const PairConst *__restrict__ pp, const PairConst *__restrict__ pw,
                                              const WallGeom *__restrict__ walls, const int cur, const int nxt,
                                              const int last, const int i, double &vmax2, int &status) {
    const int cap = P.cap;
    const unsigned q = fc.quirks;
    const double4 *__restrict__ pc = P.pos[cur];
    const double *__restrict__ vc = P.vel[cur];
    const double *__restrict__ wc = P.omg[cur];
    const D4 pi = ld4(pc, i);
    double ui0 = vc[i], ui1 = vc[cap + i], ui2 = vc[2 * cap + i];
    double wi0 = wc[i], wi1 = wc[cap + i], wi2 = wc[2 * cap + i];
    const double2 mIi = P.mI[i];
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
            const D4 pj = ld4(pc, sidx);
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
        const D4 pj = ld4(pc, j);
        const double px = pi.x - pj.x, py = pi.y - pj.y, pz = pi.z - pj.z;
        const double r2ij = px * px + py * py + pz * pz;
        const double sr = pi.w + pj.w;
        // exact early-out: r2 >= s^2 (1 + 1e-10) implies sqrt(r2) >= s, overlap <= 0
        if (r2ij >= sr * sr * 1.0000000001) continue;
        const double rij = sqrt(r2ij);
        const double overlap = sr - rij;
        if (!(overlap > 0.)) continue;
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
        const double tmp_3 = 1. / pi.w;
        const double tmp_4 = 1. / pj.w;
        const double R_eff = 1. / (tmp_3 + tmp_4);
        const double kn = c.c_kn * sqrt(R_eff);
        const double S_n = c.c_Sn * sqrt(R_eff * overlap);
        const double m_eff = 1. / (1. / mIi.x + 1. / P.mI[j].x);
        const double eta_n = fc.K_n_pp * sqrt(S_n * m_eff);
        const double kt = c.c_kt * sqrt(R_eff * overlap);
        const double eta_t = fc.K_t_pp * sqrt(kt * m_eff);
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
            const double dl0 = h0 + v0 * fc.dt, dl1 = h1 + v1 * fc.dt, dl2 = h2 + v2 * fc.dt;
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
            if (fms > fc.mu_pp * fn_magn) fms = fc.mu_pp * fn_magn;
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
        if (found_at >= 0) {
            const long a = (long)found_at * cap;
            thx[a] = h0;
            thy[a] = h1;
            thz[a] = h2;
        }
        F0 += fn0 + tf0;
        F1 += fn1 + tf1;
        F2 += fn2 + tf2;
        if (!(q & DEM_Q3_NO_PP_TORQUE)) {
            T0 += (ny * tf2 - nz * tf1) * a_i;
            T1 += (nz * tf0 - nx * tf2) * a_i;
            T2 += (nx * tf1 - ny * tf0) * a_i;
        }
    }
    // ---- particle-infinite wall (Force.hpp:475-673)
    for (int w = 0; w < fc.nwall; ++w) {
        const WallGeom g = walls[w];
        const double px = pi.x - g.x[0], py = pi.y - g.x[1], pz = pi.z - g.x[2];
        const double nx = g.n[0], ny = g.n[1], nz = g.n[2];
        const double tmp = px * nx + py * ny + pz * nz;
        const double overlap = pi.w - tmp;
        const unsigned bit = 1u << w;
        double *swx = P.sw + (long)w * cap + i;
        double *swy = P.sw + (long)(P.mw + w) * cap + i;
        double *swz = P.sw + (long)(2 * P.mw + w) * cap + i;
        if (overlap > 0.) {
            const double a_i = pi.w - overlap / 2.;
            const double v0 = ui0 + (wi1 * nz - wi2 * ny) * a_i;
            const double v1 = ui1 + (wi2 * nx - wi0 * nz) * a_i;
            const double v2 = ui2 + (wi0 * ny - wi1 * nx) * a_i;
            const double vdn = v0 * nx + v1 * ny + v2 * nz;
            const double vt0 = v0 - vdn * nx, vt1 = v1 - vdn * ny, vt2 = v2 - vdn * nz;
            const PairConst c = pw[mi * fc.nwall + w];
            const double R_eff = 1. / (1. / pi.w + 0.);
            const double kn = c.c_kn * sqrt(R_eff);
            const double S_n = c.c_Sn * sqrt(R_eff * overlap);
            const double m_eff = 1. / (1. / mIi.x + 0.);
            const double eta_n = fc.K_n_pw * sqrt(S_n * m_eff);
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
                if (wmask & bit) {
                    s0 = *swx;
                    s1 = *swy;
                    s2 = *swz;
                }
                s0 += vt0 * fc.dt;
                s1 += vt1 * fc.dt;
                s2 += vt2 * fc.dt;
                const double kt = c.c_kt * sqrt(R_eff * overlap);
                const double eta_t = fc.K_t_pw * sqrt(kt * m_eff);
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
                const double lim = fc.mu_pw * fn_magn;
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
            }
            wmask |= bit;
            F0 += fn0 + ft0;
            F1 += fn1 + ft1;
            F2 += fn2 + ft2;
            T0 += (ny * ft2 - nz * ft1) * a_i;
            T1 += (nz * ft0 - nx * ft2) * a_i;
            T2 += (nx * ft1 - ny * ft0) * a_i;
        } else if (wmask & bit) {
            *swx = 0.;
            *swy = 0.;
            *swz = 0.;
            wmask &= ~bit;
        }
    }
    const int cs1 = cnt | (int)(wmask << 8);
    if (cs1 != cs0) P.cstate[i] = cs1;
    // ---- hooks after the pair forces
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
            // stage1 + stage2 of the next step
            ui0 += h * F0 * m_inverse;
            ui1 += h * F1 * m_inverse;
            ui2 += h * F2 * m_inverse;
            wi0 += h * T0 * I_inverse;
            wi1 += h * T1 * I_inverse;
            wi2 += h * T2 * I_inverse;
            pn.x += fc.dt * ui0;
            pn.y += fc.dt * ui1;
            pn.z += fc.dt * ui2;
            vmax2 = ui0 * ui0 + ui1 * ui1 + ui2 * ui2;
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
    }

template <int MODE>
__global__ void __launch_bounds__(kBlock) k_step(Particles P, NbrList L, Ctl *ctl, ForceConsts fc,
                                                 const PairConst *__restrict__ pp, const PairConst *__restrict__ pw,
                                                 const WallGeom *__restrict__ walls) {
    const CtlSnap cs_ = read_ctl(ctl, MODE == MODE_FUSED);
    if (!cs_.go) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double vmax2 = 0.0;
    int status = 0;
    if (i < P.n) particle_full<MODE>(P, L, fc, pp, pw, walls, cs_.cur, cs_.cur ^ 1, cs_.last, i, vmax2, status);
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
__global__ void __launch_bounds__(kStreamBlock) k_stream(Particles P, NbrList L, Ctl *ctl, ForceConsts fc,
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
        const D4 pi = ld4(pc, i);
        const int cs = P.cstate[i];
        const int nn = L.nn[i];
        const double2 mIi = P.mI[i];
        double ui0 = vc[i], ui1 = vc[cap + i], ui2 = vc[2 * cap + i];
        double wi0 = wc[i], wi1 = wc[cap + i], wi2 = wc[2 * cap + i];
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
    const CtlSnap cs_ = read_ctl(ctl, true);
    if (!cs_.go) return;
    const int nd = ctl->ndefer;
    double vmax2 = 0.0;
    int status = 0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nd; t += gridDim.x * blockDim.x) {
        double v2 = 0.0;
        particle_full<MODE_FUSED>(P, L, fc, pp, pw, walls, cs_.cur, cs_.cur ^ 1, cs_.last, L.defer[t], v2, status);
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
        static int gs = 0, gc = 0, last_n = -1;
        if (last_n != P.n) {
            gs = persistent_blocks((const void *)k_stream, kStreamBlock, P.n);
            gc = persistent_blocks((const void *)k_contact, kBlock, P.n);
            last_n = P.n;
        }
        k_stream<<<gs, kStreamBlock, 0, s>>>(P, L, ctl, fc, walls);
        k_contact<<<gc, kBlock, 0, s>>>(P, L, ctl, fc, pp, pw, walls);
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
