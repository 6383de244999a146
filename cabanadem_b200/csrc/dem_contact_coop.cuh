// dem_contact_coop.cuh -- cooperative contact step: NL lanes of a warp share one deferred
// particle.  Included after dem_particle.cuh by the FP64 and the mixed translation units.
//
// The per-thread step (particle_full) walks a particle's tracked contacts and neighbour list
// one entry at a time, so in a dense packing each particle is a chain of some fifteen
// dependent memory round trips.  Here the lanes of a group load the tracked slots, the list
// entries and the partners' state of one particle at once, so the chain is about five round
// trips long, and every sequential decision of the reference is reproduced exactly:
//
//  * compaction (Force.hpp:364-441) removes a slot by moving the last unexamined slot into
//    it.  Its outcome depends only on which slots still overlap: with K slots kept, the
//    kept slots below K stay in place and the removed slots below K receive the kept slots
//    at or above K, highest first.  Each lane evaluates that closed form for its slots.
//  * new contacts take slots in list order (Force.hpp:166-192): rank by a ballot prefix.
//  * F and tau are summed on the group's first lane in list order, then walls in wall order
//    (the reference's summation order), from per-contact terms computed by pp_pair/pw_wall,
//    the same functions the per-thread kernel uses.
// Results are therefore bit-identical to the per-thread step.  A particle's tracked slots are
// staged in shared memory (kCoopSlots per group), so the kernel serves MaxCnts <= 32.
#pragma once

namespace b200dem {
namespace {

// r-th highest set bit of b (r = 0: the highest); b has more than r bits set
__device__ __forceinline__ int nth_high_bit(unsigned b, int r) {
    for (int k = 0; k < r; ++k) b &= ~(0x80000000u >> __clz(b));
    return 31 - __clz(b);
}

// Warp-collective: all 32 lanes call it; the groups of lanes [g NL, g NL + NL) each take one
// particle i (i < 0: no particle, the group still takes part in the warp's shuffles).  t is
// the particle's deferred slot.  s_tidx / s_h are the group's shared slots.
template <int NL, bool MIXED, bool MESH = false>
__device__ __forceinline__ void particle_coop(const Particles &P, const NbrList &L, const ForceConsts &fc,
                                              const PairConst *__restrict__ pp, const PairConst *__restrict__ pw,
                                              const WallGeom *__restrict__ walls, const int cur, const int nxt,
                                              const int vcur, const int last, const int i, const int t,
                                              int *s_tidx, double *s_h, double &vmax2, int &status) {
    constexpr unsigned FULL = 0xffffffffu;
    constexpr unsigned GLOW = NL == 32 ? 0xffffffffu : ((1u << NL) - 1u);
    const int lane = threadIdx.x & 31, gl = lane % NL, gbase = lane - gl;
    const unsigned below = (1u << gl) - 1u;   // lanes of the group before this one
    const bool act = i >= 0;
    const int cap = P.cap;
    const unsigned q = fc.quirks;
    const int scene_i = (act && P.scene) ? P.scene[i] : 0;
    const SceneConst *scn = fc.scenes ? fc.scenes + scene_i : nullptr;
    const double K_n_pp = scn ? scn->K_n_pp : fc.K_n_pp, K_t_pp = scn ? scn->K_t_pp : fc.K_t_pp;
    const double K_n_pw = scn ? scn->K_n_pw : fc.K_n_pw, K_t_pw = scn ? scn->K_t_pw : fc.K_t_pw;
    const double mu_pp = scn ? scn->mu_pp : fc.mu_pp, mu_pw = scn ? scn->mu_pw : fc.mu_pw;
    const int wall0 = fc.wps ? scene_i * fc.wps : 0;
    const int nwall = act ? (fc.wps ? fc.wps : fc.nwall) : 0;
    const double4 *__restrict__ pc = P.pos[cur];
    const double *__restrict__ vc = P.vel[vcur];
    const double *__restrict__ wc = P.omg[vcur];
    D4 pi = {0., 0., 0., 0.};
    double ui0 = 0., ui1 = 0., ui2 = 0., wi0 = 0., wi1 = 0., wi2 = 0.;
    double2 mIi = make_double2(0., 0.);
    int mi = 0, cs0 = 0, nn = 0;
    if (act) {
        pi = ld4_early(pc, i);
        ui0 = ld_early(vc + i);
        ui1 = ld_early(vc + cap + i);
        ui2 = ld_early(vc + 2 * cap + i);
        wi0 = ld_early(wc + i);
        wi1 = ld_early(wc + cap + i);
        wi2 = ld_early(wc + 2 * cap + i);
        mIi = make_double2(ld_early(P.mI + i), ld_early(P.mI + cap + i));
        cs0 = ld_early_i(P.cstate + i);
        nn = ld_early_i(L.nn + i);
        mi = fc.nmat > 1 ? (int)P.mat[i] : 0;
    }
    const int cnt0 = cs0 & 0xff;
    const unsigned wmask0 = (unsigned)cs0 >> 8;
    const int ii = act ? i : 0;   // the pointers below are only dereferenced for a particle
    int *tidx = P.tidx + ii;
    double *thx = P.th + ii;
    double *thy = P.th + (long)P.mc * cap + ii;
    double *thz = P.th + 2L * P.mc * cap + ii;

    // ---- update_tangential_contacts (Force.hpp:364-441): which tracked slots still overlap
    constexpr int R = kCoopSlots / NL;
    const int rc = (int)__reduce_max_sync(FULL, (unsigned)((cnt0 + NL - 1) / NL));
    unsigned keep = 0u;
    for (int r = 0; r < rc; ++r) {
        const int s = gl + r * NL;
        bool kp = false;
        if (s < cnt0) {
            const long a = (long)s * cap;
            const int sidx = tidx[a];
            s_tidx[s] = sidx;
            s_h[s] = thx[a];
            s_h[kCoopSlots + s] = thy[a];
            s_h[2 * kCoopSlots + s] = thz[a];
            kp = true;   // an index outside [0, n) (not written by this library) stays in place
            if ((unsigned)sidx < (unsigned)P.n) {
                const D4 pj = ld4(pc, sidx);
                const double px = pi.x - pj.x, py = pi.y - pj.y, pz = pi.z - pj.z;
                const double r2ij = px * px + py * py + pz * pz;
                const double rij = sqrt(r2ij);
                const double overlap = pi.w + pj.w - rij;
                kp = !(overlap <= 0.);
            }
        }
        keep |= ((__ballot_sync(FULL, kp) >> gbase) & GLOW) << (r * NL);
    }
    __syncwarp();
    const int K = __popc(keep);
    if (rc > 0) {
        const unsigned lowK = K >= 32 ? FULL : ((1u << K) - 1u);
        const unsigned holes = ~keep & lowK;   // removed slots below K
        const unsigned back = keep & ~lowK;    // kept slots at or above K, moved down highest first
        int ft[R];
        double f0[R], f1[R], f2[R];
        bool mv[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int p = gl + r * NL;
            mv[r] = false;
            ft[r] = -1;
            f0[r] = f1[r] = f2[r] = 0.;
            if (r < rc && p < cnt0) {
                if (p < K) {
                    if (!((keep >> p) & 1u)) {
                        const int src = nth_high_bit(back, __popc(holes & ((1u << p) - 1u)));
                        ft[r] = s_tidx[src];
                        f0[r] = s_h[src];
                        f1[r] = s_h[kCoopSlots + src];
                        f2[r] = s_h[2 * kCoopSlots + src];
                        mv[r] = true;
                    }
                } else {
                    mv[r] = true;   // emptied: index -1, zero history
                }
            }
        }
        __syncwarp();
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int p = gl + r * NL;
            if (mv[r]) {
                const long a = (long)p * cap;
                s_tidx[p] = ft[r];
                s_h[p] = f0[r];
                s_h[kCoopSlots + p] = f1[r];
                s_h[2 * kCoopSlots + p] = f2[r];
                tidx[a] = ft[r];
                thx[a] = f0[r];
                thy[a] = f1[r];
                thz[a] = f2[r];
            }
        }
        __syncwarp();
    }

    // ---- particle-particle (Force.hpp:73-329): lanes over list entries, sums in list order
    double F0 = 0., F1 = 0., F2 = 0., T0 = 0., T1 = 0., T2 = 0.;
    if (act && fc.has_ext) {
        F0 += P.ext[i];
        F1 += P.ext[cap + i];
        F2 += P.ext[2 * cap + i];
    }
    int cnt = K;
    const int rn = (int)__reduce_max_sync(FULL, (unsigned)((nn + NL - 1) / NL));
    for (int r = 0; r < rn; ++r) {
        const int kk = gl + r * NL;
        bool con = false;
        int j = 0;
        D4 pj = {0., 0., 0., 0.};
        double px = 0., py = 0., pz = 0., rij = 0., overlap = 0.;
        if (kk < nn) {
            j = L.idx[(long)kk * cap + i];
            pj = ld4(pc, j);
            px = pi.x - pj.x;
            py = pi.y - pj.y;
            pz = pi.z - pj.z;
            const double r2ij = px * px + py * py + pz * pz;
            const double sr = pi.w + pj.w;
            if (!(r2ij >= sr * sr * 1.0000000001)) {
                rij = sqrt(r2ij);
                overlap = sr - rij;
                con = overlap > 0.;
            }
        }
        // slot lookup among the compacted slots (a partner appears once in a list, so the
        // slots inserted by earlier entries of this pass never match)
        int found_at = -1;
        if (con)
            for (int s = 0; s < K; ++s)
                if (s_tidx[s] == j) found_at = s;
        const bool isnew = con && found_at < 0;
        const unsigned nb = (__ballot_sync(FULL, isnew) >> gbase) & GLOW;
        if (isnew) {
            const int slot = cnt + __popc(nb & below);
            if (slot < P.mc)
                found_at = slot;
            else
                status |= DEM_ERR_CONTACT_OVERFLOW;
        }
        cnt = min(cnt + __popc(nb), P.mc);
        double cf[6] = {0., 0., 0., 0., 0., 0.};
        if (con) {
            double h0 = 0., h1 = 0., h2 = 0.;
            if (found_at >= 0 && !isnew) {
                h0 = s_h[found_at];
                h1 = s_h[kCoopSlots + found_at];
                h2 = s_h[2 * kCoopSlots + found_at];
            }
            const int mj = fc.nmat > 1 ? (int)P.mat[j] : 0;
            const PairConst c = pp[mi * fc.nmat + mj];
            pp_pair<MIXED>(P.mI, vc, wc, cap, q, pi, pj, j, px, py, pz, rij, overlap, ui0, ui1, ui2, wi0, wi1, wi2,
                           mIi.x, c, K_n_pp, K_t_pp, mu_pp, fc.dt, h0, h1, h2, cf);
            if (found_at >= 0) {
                const long a = (long)found_at * cap;
                if (isnew) tidx[a] = j;
                thx[a] = h0;
                thy[a] = h1;
                thz[a] = h2;
            }
        }
        const unsigned cball = __ballot_sync(FULL, con);
        unsigned col = 0u;
#pragma unroll
        for (int g = 0; g < 32 / NL; ++g) col |= (cball >> (g * NL)) & GLOW;
        const unsigned cb = (cball >> gbase) & GLOW;
        while (col) {
            const int qq = __ffs(col) - 1;
            col &= col - 1u;
            const double v0 = __shfl_sync(FULL, cf[0], gbase + qq), v1 = __shfl_sync(FULL, cf[1], gbase + qq);
            const double v2 = __shfl_sync(FULL, cf[2], gbase + qq), v3 = __shfl_sync(FULL, cf[3], gbase + qq);
            const double v4 = __shfl_sync(FULL, cf[4], gbase + qq), v5 = __shfl_sync(FULL, cf[5], gbase + qq);
            if ((cb >> qq) & 1u) {
                F0 += v0;
                F1 += v1;
                F2 += v2;
                if (!(q & DEM_Q3_NO_PP_TORQUE)) {
                    T0 += v3;
                    T1 += v4;
                    T2 += v5;
                }
            }
        }
    }

    // ---- particle-infinite wall (Force.hpp:475-673): lanes over walls, sums in wall order
    unsigned wset = 0u;
    const int rw = (int)__reduce_max_sync(FULL, (unsigned)((nwall + NL - 1) / NL));
    for (int r = 0; r < rw; ++r) {
        const int lw = gl + r * NL;
        bool con = false;
        double cf[6] = {0., 0., 0., 0., 0., 0.};
        if (lw < nwall) {
            const int w = wall0 + lw;
            const WallGeom g = walls[w];
            const double px = pi.x - g.x[0], py = pi.y - g.x[1], pz = pi.z - g.x[2];
            const double nx = g.n[0], ny = g.n[1], nz = g.n[2];
            const double tmp = px * nx + py * ny + pz * nz;
            const double overlap = pi.w - tmp;
            const unsigned bit = 1u << lw;
            double *swx = P.sw + (long)lw * cap + ii;
            double *swy = P.sw + (long)(P.mw + lw) * cap + ii;
            double *swz = P.sw + (long)(2 * P.mw + lw) * cap + ii;
            if (overlap > 0.) {
                pw_wall<MIXED>(q, pi, nx, ny, nz, overlap, ui0, ui1, ui2, wi0, wi1, wi2, g.u[0], g.u[1], g.u[2],
                               mIi.x, pw[mi * fc.nwall + w], K_n_pw, K_t_pw, mu_pw, fc.dt, (wmask0 & bit) != 0u, swx,
                               swy, swz, cf);
                con = true;
            } else if (wmask0 & bit) {
                *swx = 0.;
                *swy = 0.;
                *swz = 0.;
            }
        }
        const unsigned cball = __ballot_sync(FULL, con);
        const unsigned cb = (cball >> gbase) & GLOW;
        wset |= cb << (r * NL);
        unsigned col = 0u;
#pragma unroll
        for (int g = 0; g < 32 / NL; ++g) col |= (cball >> (g * NL)) & GLOW;
        while (col) {
            const int qq = __ffs(col) - 1;
            col &= col - 1u;
            const double v0 = __shfl_sync(FULL, cf[0], gbase + qq), v1 = __shfl_sync(FULL, cf[1], gbase + qq);
            const double v2 = __shfl_sync(FULL, cf[2], gbase + qq), v3 = __shfl_sync(FULL, cf[3], gbase + qq);
            const double v4 = __shfl_sync(FULL, cf[4], gbase + qq), v5 = __shfl_sync(FULL, cf[5], gbase + qq);
            if ((cb >> qq) & 1u) {
                F0 += v0;
                F1 += v1;
                F2 += v2;
                T0 += v3;
                T1 += v4;
                T2 += v5;
            }
        }
    }
    if (!act || gl != 0) return;

    // ---- the group's first lane: mesh contacts, contact state, hooks, integration (as particle_full)
    if constexpr (MESH) {
        double FT[6] = {F0, F1, F2, T0, T1, T2};
        mesh_pass<MIXED>(P, fc, i, pi, ui0, ui1, ui2, wi0, wi1, wi2, mIi.x, mi, K_n_pw, K_t_pw, mu_pw, FT, &status);
        F0 = FT[0];
        F1 = FT[1];
        F2 = FT[2];
        T0 = FT[3];
        T1 = FT[4];
        T2 = FT[5];
    }
    const unsigned wrange = nwall >= 32 ? FULL : ((1u << nwall) - 1u);
    const unsigned wmask = (wmask0 & ~wrange) | wset;
    const int cs1 = cnt | (int)(wmask << 8);
    if (cs1 != cs0) P.cstate[i] = cs1;
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
    const double m_inverse = 1. / mIi.x;
    const double I_inverse = 1. / mIi.y;
    const double h = fc.half_dt;
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
    st4(P.pos[nxt], i, pn);
    double *vn = L.defer_v, *wn = L.defer_w;
    vn[t] = ui0;
    vn[cap + t] = ui1;
    vn[2 * cap + t] = ui2;
    wn[t] = wi0;
    wn[cap + t] = wi1;
    wn[2 * cap + t] = wi2;
}

// Fused step, kernel 2 of 3 in its cooperative form: NL lanes per deferred particle, warps
// striding over the deferred list in groups of 32 / NL.  No block barrier: a warp past the
// list leaves at once, and the velocity bound is folded per warp.
template <int NL, int MINB, bool MIXED, bool MESH = false>
__global__ void __launch_bounds__(kBlock, MINB) k_contact_coop(Particles P, NbrList L, Ctl *ctl, ForceConsts fc,
                                                               const PairConst *__restrict__ pp,
                                                               const PairConst *__restrict__ pw,
                                                               const WallGeom *__restrict__ walls) {
    grid_dep_wait();   // launched as a dependent (launch_k): the kernel before has completed
    grid_dep_release();
    constexpr int G = 32 / NL;
    // one row per group, padded by one word so that the groups of a warp fall in different banks
    __shared__ int s_tidx[kBlock / NL][kCoopSlots + 1];
    __shared__ double s_h[kBlock / NL][3 * kCoopSlots + 1];
    if (ctl->steps_done >= ctl->target || (ctl->status & kStopBits) || !(ctl->disp < ctl->half_skin))
        return;
    const int nd = ctl->ndefer;
    const int warp = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
    const int nwarps = gridDim.x * (kBlock / 32);
    if ((long)warp * G >= nd) return;
    const int cur = ctl->cur, vcur = ctl->vcur;
    const int last = ctl->steps_done + 1 >= ctl->target;
    const int grp = (threadIdx.x & 31) / NL;
    const int sg = (threadIdx.x >> 5) * G + grp;
    double vmax2 = 0.0;
    int status = 0;
    for (int base = warp * G; base < nd; base += nwarps * G) {
        const int t = base + grp;
        const int i = t < nd ? L.defer[t] : -1;
        double v2 = 0.0;
        particle_coop<NL, MIXED, MESH>(P, L, fc, pp, pw, walls, cur, cur ^ 1, vcur, last, i, t, s_tidx[sg], s_h[sg], v2,
                                 status);
        vmax2 = fmax(vmax2, v2);
    }
    warp_vmax(ctl, P.vslots, vmax2, status);
}

}  // namespace
}  // namespace b200dem
