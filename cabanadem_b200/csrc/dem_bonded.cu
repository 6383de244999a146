// dem_bonded.cu -- bonded-DEM bond build and fused bond-force step on sm_100a (FP64,
// built with --fmad=false; the expressions follow the reference's order).
//
//   k_bond_setup   setupBonds (src/CabanaBondedDEM_Particles.hpp:118-137): over the
//                  neighbour list (ascending caller index) bond every j with
//                  rij < factor * rad(i), rest length = rij
//   k_bond_step    one bonded step in the order of tst_01_BDEM:295-306: force reset, external
//                  force, computeBondedForce (src/CabanaBondedDEM_Force.hpp:86-341), boundary
//                  hook, stage3, then stage1 + stage2 of the next step (ping-pong buffers)
//   k_bond_force   computeBondedForce alone, for callers that drive the bonded loop phase by
//                  phase (with k_add_ext_force and k_post_hooks for the example's hooks)
//
// Bond slots are slot-major per particle: partner (sorted index), rest length, and the 9 live
// history components (tangential force, normal and tangential moments; the reference's
// bond_fn_* arrays are never written, :69-71).  Breakage (no reference counterpart): a bond
// whose FP64 strain (rij - L0) / L0 exceeds the threshold is flagged and skipped from then on;
// both ends compute the same strain bit for bit, so they break in the same step.
#include "dem_particle.cuh"

namespace b200dem {

namespace {

constexpr int kBondBlock = 128;

__global__ void k_bond_setup(Particles P, NbrList L, Bonds B, Ctl *ctl, double factor) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const int cur = ctl->cur, cap = P.cap;
    const D4 pi = ld4(P.pos[cur], i);
    int cnt = 0;
    int status = 0;
    for (int kk = 0; kk < L.nn[i]; ++kk) {
        const int j = L.idx[(long)kk * cap + i];
        const D4 pj = ld4(P.pos[cur], j);
        const double px = pi.x - pj.x, py = pi.y - pj.y, pz = pi.z - pj.z;
        const double r2ij = px * px + py * py + pz * pz;
        const double rij = sqrt(r2ij);
        const double bond_cond = factor * pi.w;
        if (rij < bond_cond) {
            if (cnt >= B.mb) {
                status |= DEM_ERR_BOND_OVERFLOW;
                continue;
            }
            B.idx[(long)cnt * cap + i] = j;
            B.init_len[(long)cnt * cap + i] = rij;
            ++cnt;
        }
    }
    B.count[i] = cnt;
    for (int k = cnt; k < B.mb; ++k) B.idx[(long)k * cap + i] = -1;
    if (status) atomicOr(&ctl->status, status);
}

// R = double: the reference's FP64 arithmetic (bitwise parity with the oracle).  R = float
// (mixed precision): strain, geometry and relative kinematics stay FP64 (rij - L0 and the
// breakage test are exact), the bond force/moment history is stored and updated in FP32
// (half the history traffic), per-particle sums and integration are FP64.
template <typename R>
__device__ __forceinline__ R *bond_hist(const Bonds &B);
template <>
__device__ __forceinline__ double *bond_hist<double>(const Bonds &B) { return B.hist; }
template <>
__device__ __forceinline__ float *bond_hist<float>(const Bonds &B) { return B.hist32; }

// One bond, slot k of particle i (BondedDEM_Force.hpp:53-348): strain and breakage, normal
// force, incremental shear force, twisting and bending moments with their histories.
// Returns false when the slot holds no live bond (empty, broken now or before, or its
// partner-indexed history slot overflows); else cf receives the bond's contribution to F
// (0..2) and tau (3..5) of i, which the caller adds in slot order.
template <typename R>
__device__ __forceinline__ bool bond_term(const Particles &P, const Bonds &B, const BondConsts &bc, R *__restrict__ hist,
                                          const double4 *__restrict__ pc, const double *__restrict__ vc,
                                          const double *__restrict__ wc, const int cap, const int i, const int k,
                                          const D4 &pi, const double ui0, const double ui1, const double ui2,
                                          const double wi0, const double wi1, const double wi2, const double Ei,
                                          const double Gi, const double dt, int &status, double (&cf)[6]) {
    const long slot = (long)k * cap + i;
    const int j = B.idx[slot];
    if (j < 0 || B.broken[slot]) return false;
    long hs = slot;
    if (bc.quirks & BQ10_INDEX_BY_J) {
        const int jc = P.perm[j];
        if (jc >= B.mb) {
            status |= DEM_ERR_BOND_OVERFLOW;
            return false;
        }
        hs = (long)jc * cap + i;
    }
    const D4 pj = ld4(pc, j);
    const double px = pi.x - pj.x, py = pi.y - pj.y, pz = pi.z - pj.z;
    const double r2ij = px * px + py * py + pz * pz;
    const double rij = sqrt(r2ij);
    const double L0 = B.init_len[hs];
    if (bc.break_strain > 0.0) {
        const double strain = (rij - L0) / L0;
        if (strain > bc.break_strain) {
            B.broken[slot] = 1;
            return false;
        }
    }
    const double g_c = rij - pi.w - pj.w;
    const double a_i = pi.w + g_c / 2.;
    const double a_j = pj.w + g_c / 2.;
    const double n0 = px / rij, n1 = py / rij, n2 = pz / rij;
    const double uj0 = vc[j];
    const double uj1 = (bc.quirks & BQ1_VELJ_USES_UI) ? ui1 : vc[cap + j];
    const double uj2 = (bc.quirks & BQ1_VELJ_USES_UI) ? ui2 : vc[2 * cap + j];
    const double wj0 = wc[j], wj1 = wc[cap + j], wj2 = wc[2 * cap + j];
    const double vi0 = ui0 + (wi1 * n2 - wi2 * n1) * a_i;
    const double vi1 = ui1 + (wi2 * n0 - wi0 * n2) * a_i;
    const double vi2 = ui2 + (wi0 * n1 - wi1 * n0) * a_i;
    const double vj0 = uj0 + (-wj1 * n2 + wj2 * n1) * a_j;
    const double vj1 = uj1 + (-wj2 * n0 + wj0 * n2) * a_j;
    const double vj2 = uj2 + (-wj0 * n1 + wj1 * n0) * a_j;
    const double vr0 = vi0 - vj0, vr1 = vi1 - vj1, vr2 = vi2 - vj2;
    const double vdp = vr0 * n0 + vr1 * n1 + vr2 * n2;
    const double vn0 = vdp * n0, vn1 = vdp * n1, vn2 = vdp * n2;
    const double vt0 = vr0 - vn0, vt1 = vr1 - vn1, vt2 = vr2 - vn2;
    const double wr0 = wi0 - wj0, wr1 = wi1 - wj1, wr2 = wi2 - wj2;
    const double wdp = wr0 * n0 + wr1 * n1 + wr2 * n2;
    const double wn0 = wdp * n0, wn1 = wdp * n1, wn2 = wdp * n2;
    const double wt0 = wr0 - wn0, wt1 = wr1 - wn1, wt2 = wr2 - wn2;
    const double rad_sum = pi.w + pj.w;
    const double beta_bond = bc.beta;
    const double bond_rad = (pi.w < pj.w ? pi.w : pj.w) * bc.radius_factor;
    const double A_bond = M_PI * (bond_rad * bond_rad);
    const double I_bond = M_PI * ((bond_rad * bond_rad) * (bond_rad * bond_rad)) / 4.0;
    const double I_p_bond = I_bond * 2.0;
    double k_n_bond, k_t_bond, k_tor_bond, k_ben_bond;
    if (bc.quirks & BQ11_HARDCODED_K) {
        k_n_bond = Ei * A_bond / rad_sum;
        k_t_bond = Gi * A_bond / rad_sum;
        k_tor_bond = Gi * I_p_bond / rad_sum;
        k_ben_bond = Ei * I_bond / rad_sum;
    } else {
        k_n_bond = bc.kn;
        k_t_bond = bc.kt;
        k_tor_bond = bc.kt * I_p_bond / A_bond;
        k_ben_bond = bc.kn * I_bond / A_bond;
    }
    // normal bond force (:205-222)
    const double overlap_n = rij - L0;
    const R rn0 = (R)n0, rn1 = (R)n1, rn2 = (R)n2;
    const R fn0 = -(R)k_n_bond * (R)overlap_n * rn0;
    const R fn1 = -(R)k_n_bond * (R)overlap_n * rn1;
    const R fn2 = -(R)k_n_bond * (R)overlap_n * rn2;
    const R beta_b = (R)beta_bond;
    R mX = (vn0 >= 0.0) ? (R)1 : (R)-1;
    R mY = (vn1 >= 0.0) ? (R)1 : (R)-1;
    R mZ = (vn2 >= 0.0) ? (R)1 : (R)-1;
    const R fd0 = fn0 + beta_b * fabs(fn0) * mX;
    const R fd1 = fn1 + beta_b * fabs(fn1) * mY;
    const R fd2 = fn2 + beta_b * fabs(fn2) * mZ;
    // tangential bond force (:231-260)
    R ft0 = hist[(0L * B.mb) * cap + hs], ft1 = hist[(1L * B.mb) * cap + hs], ft2 = hist[(2L * B.mb) * cap + hs];
    const R fdp = ft0 * rn0 + ft1 * rn1 + ft2 * rn2;
    ft0 -= fdp * rn0;
    ft1 -= fdp * rn1;
    ft2 -= fdp * rn2;
    R tmp = (R)k_t_bond * (R)dt;
    ft0 += -(R)vt0 * tmp;
    ft1 += -(R)vt1 * tmp;
    ft2 += -(R)vt2 * tmp;
    mX = (vt0 >= 0.0) ? (R)1 : (R)-1;
    mY = (vt1 >= 0.0) ? (R)1 : (R)-1;
    mZ = (vt2 >= 0.0) ? (R)1 : (R)-1;
    const R ftd0 = ft0 - beta_b * fabs(ft0) * mX;
    const R ftd1 = ft1 - beta_b * fabs(ft1) * mY;
    const R ftd2 = ft2 - beta_b * fabs(ft2) * mZ;
    hist[(0L * B.mb) * cap + hs] = ftd0;
    hist[(1L * B.mb) * cap + hs] = ftd1;
    hist[(2L * B.mb) * cap + hs] = ftd2;
    // twisting moment (:267-291)
    R tn0 = hist[(3L * B.mb) * cap + hs], tn1 = hist[(4L * B.mb) * cap + hs], tn2 = hist[(5L * B.mb) * cap + hs];
    R tdp = tn0 * rn0 + tn1 * rn1 + tn2 * rn2;
    tn0 = tdp * rn0;
    tn1 = tdp * rn1;
    tn2 = tdp * rn2;
    tmp = (R)k_tor_bond * (R)dt;
    tn0 += -(R)wn0 * tmp;
    tn1 += -(R)wn1 * tmp;
    tn2 += -(R)wn2 * tmp;
    mX = (wn0 >= 0.0) ? (R)1 : (R)-1;
    mY = (wn1 >= 0.0) ? (R)1 : (R)-1;
    mZ = (wn2 >= 0.0) ? (R)1 : (R)-1;
    const R nd0 = tn0 - beta_b * fabs(tn0) * mX;
    const R nd1 = tn1 - beta_b * fabs(tn1) * mY;
    const R nd2 = tn2 - beta_b * fabs(tn2) * mZ;
    hist[(3L * B.mb) * cap + hs] = nd0;
    hist[(4L * B.mb) * cap + hs] = nd1;
    hist[(5L * B.mb) * cap + hs] = nd2;
    // bending moment (:298-322)
    R tt0 = hist[(6L * B.mb) * cap + hs], tt1 = hist[(7L * B.mb) * cap + hs], tt2 = hist[(8L * B.mb) * cap + hs];
    tdp = tt0 * rn0 + tt1 * rn1 + tt2 * rn2;
    tt0 -= tdp * rn0;
    tt1 -= tdp * rn1;
    tt2 -= tdp * rn2;
    tmp = (R)k_ben_bond * (R)dt;
    tt0 += -(R)wt0 * tmp;
    tt1 += -(R)wt1 * tmp;
    tt2 += -(R)wt2 * tmp;
    mX = (wt0 >= 0.0) ? (R)1 : (R)-1;
    mY = (wt1 >= 0.0) ? (R)1 : (R)-1;
    mZ = (wt2 >= 0.0) ? (R)1 : (R)-1;
    const R td0 = tt0 - beta_b * fabs(tt0) * mX;
    const R td1 = tt1 - beta_b * fabs(tt1) * mY;
    const R td2 = tt2 - beta_b * fabs(tt2) * mZ;
    hist[(6L * B.mb) * cap + hs] = td0;
    hist[(7L * B.mb) * cap + hs] = td1;
    hist[(8L * B.mb) * cap + hs] = td2;
    const double cri = rij * 1. / pi.w * 1. / (pi.w + pj.w);
    cf[0] = (double)(fd0 + ftd0);
    cf[1] = (double)(fd1 + ftd1);
    cf[2] = (double)(fd2 + ftd2);
    cf[3] = (double)(nd0 + td0) - cri * 0.0;
    cf[4] = (double)(nd1 + td1) - cri * 0.0;
    cf[5] = (double)(nd2 + td2) - cri * 0.0;
    return true;
}

// Hooks (gravity, applyBoundaryConditions of tst_01_BDEM:50-60) and the velocity-Verlet
// update of particle i after its bond pass; u, omega to the other velocity buffer.
__device__ __forceinline__ void bond_finish_particle(const Particles &P, const ForceConsts &fc, const int i,
                                                     const int nxt, const int vcur, const bool last, const D4 &pi,
                                                     double ui0, double ui1, double ui2, double wi0, double wi1,
                                                     double wi2, const double2 mIi, double F0, double F1, double F2,
                                                     double T0, double T1, double T2, double &vmax2) {
    const int cap = P.cap;
    if (fc.has_gravity) {
        F0 += mIi.x * fc.g[0];
        F1 += mIi.x * fc.g[1];
        F2 += mIi.x * fc.g[2];
    }
    if (fc.has_fix) {   // applyBoundaryConditions (tst_01_BDEM:50-60)
        const int f = P.fix[i];
        if (f & DEM_FIX_FORCE) F0 = F1 = F2 = 0.;
        if (f & DEM_FIX_TORQUE) T0 = T1 = T2 = 0.;
    }
    const double m_inverse = 1. / mIi.x, I_inverse = 1. / mIi.y, h = fc.half_dt;
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
        vmax2 = ui0 * ui0 + ui1 * ui1 + ui2 * ui2;
    }
    st4(P.pos[nxt], i, pn);
    double *vn = P.vel[vcur ^ 1], *wn = P.omg[vcur ^ 1];
    vn[i] = ui0;
    vn[cap + i] = ui1;
    vn[2 * cap + i] = ui2;
    wn[i] = wi0;
    wn[cap + i] = wi1;
    wn[2 * cap + i] = wi2;
}

template <typename R>
__global__ void __launch_bounds__(kBondBlock) k_bond_step(Particles P, Bonds B, Ctl *ctl, ForceConsts fc, BondConsts bc) {
    grid_dep_wait();   // launched as a dependent (launch_k): the kernel before has completed
    grid_dep_release();
    R *__restrict__ hist = bond_hist<R>(B);
    const CtlSnap cs_ = read_ctl(ctl, true);
    if (!cs_.go) return;
    const int cur = cs_.cur, nxt = cur ^ 1, vcur = ctl->vcur;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int cap = P.cap;
    double vmax2 = 0.0;
    int status = 0;
    if (i < P.n) {
        const double4 *__restrict__ pc = P.pos[cur];
        const double *__restrict__ vc = P.vel[vcur];
        const double *__restrict__ wc = P.omg[vcur];
        const D4 pi = ld4(pc, i);
        double ui0 = vc[i], ui1 = vc[cap + i], ui2 = vc[2 * cap + i];
        double wi0 = wc[i], wi1 = wc[cap + i], wi2 = wc[2 * cap + i];
        const double2 mIi = load_mI(P, i);
        double F0 = 0., F1 = 0., F2 = 0., T0 = 0., T1 = 0., T2 = 0.;
        if (fc.has_ext) {   // applyTensileForce (tst_01_BDEM:101-111) before the bond pass
            F0 += P.ext[i];
            F1 += P.ext[cap + i];
            F2 += P.ext[2 * cap + i];
        }
        const double Ei = B.E[i], Gi = B.G[i];
        const int no_bonds_i = B.count[i];
        for (int k = 0; k < no_bonds_i; k++) {
            double cf[6];
            if (!bond_term<R>(P, B, bc, hist, pc, vc, wc, cap, i, k, pi, ui0, ui1, ui2, wi0, wi1, wi2, Ei, Gi, fc.dt,
                              status, cf))
                continue;
            F0 += cf[0];
            F1 += cf[1];
            F2 += cf[2];
            T0 += cf[3];
            T1 += cf[4];
            T2 += cf[5];
        }
        bond_finish_particle(P, fc, i, nxt, vcur, cs_.last, pi, ui0, ui1, ui2, wi0, wi1, wi2, mIi, F0, F1, F2, T0, T1,
                             T2, vmax2);
    }
    finish_step(ctl, P.vslots, vmax2, fc.dt, status, true, true);
}

// computeBondedForce as a phase of its own (src/CabanaBondedDEM_Force.hpp:53-348): for every
// particle, F and tau += the bond terms in slot order, starting from the F and tau the earlier
// phases left (resetForcesAndTorques, then the caller's hooks).  Same per-bond arithmetic as
// the fused step (bond_term), so a loop of phases equals the fused step bit for bit.
template <typename R>
__global__ void __launch_bounds__(kBondBlock) k_bond_force(Particles P, Bonds B, Ctl *ctl, BondConsts bc, double dt) {
    R *__restrict__ hist = bond_hist<R>(B);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const int cur = ctl->cur, vcur = ctl->vcur, cap = P.cap;
    const double4 *__restrict__ pc = P.pos[cur];
    const double *__restrict__ vc = P.vel[vcur];
    const double *__restrict__ wc = P.omg[vcur];
    const D4 pi = ld4(pc, i);
    const double ui0 = vc[i], ui1 = vc[cap + i], ui2 = vc[2 * cap + i];
    const double wi0 = wc[i], wi1 = wc[cap + i], wi2 = wc[2 * cap + i];
    double F0 = P.force[i], F1 = P.force[cap + i], F2 = P.force[2 * cap + i];
    double T0 = P.torque[i], T1 = P.torque[cap + i], T2 = P.torque[2 * cap + i];
    const double Ei = B.E[i], Gi = B.G[i];
    int status = 0;
    const int no_bonds_i = B.count[i];
    for (int k = 0; k < no_bonds_i; k++) {
        double cf[6];
        if (!bond_term<R>(P, B, bc, hist, pc, vc, wc, cap, i, k, pi, ui0, ui1, ui2, wi0, wi1, wi2, Ei, Gi, dt, status,
                          cf))
            continue;
        F0 += cf[0];
        F1 += cf[1];
        F2 += cf[2];
        T0 += cf[3];
        T1 += cf[4];
        T2 += cf[5];
    }
    P.force[i] = F0;
    P.force[cap + i] = F1;
    P.force[2 * cap + i] = F2;
    P.torque[i] = T0;
    P.torque[cap + i] = T1;
    P.torque[2 * cap + i] = T2;
    if (status) atomicOr(&ctl->status, status);
}

// The hook in the position of tst_01_BDEM's applyTensileForce (:101-111): F += the external
// force (DEM_F_EXT_FORCE).
__global__ void k_add_ext_force(Particles P) {
    const int cap = P.cap;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += gridDim.x * blockDim.x) {
        P.force[i] += P.ext[i];
        P.force[cap + i] += P.ext[cap + i];
        P.force[2 * cap + i] += P.ext[2 * cap + i];
    }
}

// The hooks in the position of tst_01_BDEM's applyBoundaryConditions (:19-67): gravity (m g
// added), then the DEM_FIX_* flags zero F and/or tau -- the order of the fused step.
__global__ void k_post_hooks(Particles P, ForceConsts fc) {
    const int cap = P.cap;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += gridDim.x * blockDim.x) {
        if (fc.has_gravity) {
            const double m = load_mI(P, i).x;
            P.force[i] += m * fc.g[0];
            P.force[cap + i] += m * fc.g[1];
            P.force[2 * cap + i] += m * fc.g[2];
        }
        if (fc.has_fix) {
            const int f = P.fix[i];
            if (f & DEM_FIX_FORCE) P.force[i] = P.force[cap + i] = P.force[2 * cap + i] = 0.;
            if (f & DEM_FIX_TORQUE) P.torque[i] = P.torque[cap + i] = P.torque[2 * cap + i] = 0.;
        }
    }
}

__global__ void k_bond_broken_count(Bonds B, int n, unsigned long long *out) {
    unsigned long long c = 0;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < (long)B.mb * B.cap; t += (long)gridDim.x * blockDim.x)
        c += B.broken[t] ? 1 : 0;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

}  // namespace

void launch_bond_setup(const Particles &P, const NbrList &L, const Bonds &B, Ctl *ctl, double factor, cudaStream_t s) {
    k_bond_setup<<<(P.n + 127) / 128, 128, 0, s>>>(P, L, B, ctl, factor);
}

void launch_bond_step(const Particles &P, const Bonds &B, Ctl *ctl, const ForceConsts &fc, const BondConsts &bc,
                      cudaStream_t s) {
    const int g = (P.n + kBondBlock - 1) / kBondBlock;
    if (B.hist32)
        launch_k(k_bond_step<float>, g, kBondBlock, 0, s, fc.pdl, P, B, ctl, fc, bc);
    else
        launch_k(k_bond_step<double>, g, kBondBlock, 0, s, fc.pdl, P, B, ctl, fc, bc);
}

void launch_bond_force(const Particles &P, const Bonds &B, Ctl *ctl, const BondConsts &bc, double dt, cudaStream_t s) {
    if (B.hist32)
        k_bond_force<float><<<(P.n + kBondBlock - 1) / kBondBlock, kBondBlock, 0, s>>>(P, B, ctl, bc, dt);
    else
        k_bond_force<double><<<(P.n + kBondBlock - 1) / kBondBlock, kBondBlock, 0, s>>>(P, B, ctl, bc, dt);
}

void launch_add_ext_force(const Particles &P, cudaStream_t s) {
    if (P.ext) k_add_ext_force<<<(P.n + 255) / 256, 256, 0, s>>>(P);
}

void launch_post_hooks(const Particles &P, const ForceConsts &fc, cudaStream_t s) {
    if (fc.has_gravity || fc.has_fix) k_post_hooks<<<(P.n + 255) / 256, 256, 0, s>>>(P, fc);
}

void launch_bond_broken_count(const Bonds &B, int n, unsigned long long *out, cudaStream_t s) {
    cudaMemsetAsync(out, 0, sizeof(unsigned long long), s);
    k_bond_broken_count<<<148 * 4, 256, 0, s>>>(B, n, out);
}

}  // namespace b200dem
