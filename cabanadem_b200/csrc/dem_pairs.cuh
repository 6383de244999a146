// dem_pairs.cuh -- pair-parallel form of the dense contact step (most particles in contact).
//
// The one-kernel dense step walks each particle's contacts in one thread: lists of different
// lengths and contacts of different counts leave most lanes idle while a few run the long
// FP64 pair law.  Here the step is three kernels, each with uniform work per thread:
//
//   k_pairs_find  one thread per particle: contact compaction of the tracked slots
//                 (src/CabanaDEM_Force.hpp:344-445), the overlap test over the list, and for
//                 each contact in list order its history slot (lookup, or the next free slot,
//                 Force.hpp:166-192) -- written as a packed work item (i, j, slot); then the
//                 wall overlaps (Force.hpp:475-673): one item (i, -1 - wall, local wall,
//                 history flag) per wall in contact, in wall order, and the history of a wall
//                 left behind cleared.  The items of a warp's particles are allocated with one
//                 atomic, in lane order, so each particle's items are contiguous and ordered.
//   k_pairs_eval  one thread per item: the Hertz-Mindlin pair law (pp_pair, the same function
//                 and arithmetic as the per-particle kernels) with the pair's history slot, or
//                 the wall law (pw_wall) with the wall's history; the force and torque terms
//                 are stored with the item.
//   k_pairs_sum   one thread per particle: F = ext + the terms of its pair items in list order
//                 + those of its wall items in wall order, the mesh, the hooks and the
//                 velocity-Verlet update (positions and velocities to the other buffers), the
//                 last block finalising the step.  No contact law is inlined here, so the pass
//                 runs at the occupancy of a streaming kernel.
//
// The per-particle sums run in the order of the per-particle kernel (external force, pair
// terms in list order, walls, mesh, gravity), so the results are the same bit for bit.
// Included by dem_step.cu (FP64, no contraction) and dem_mixed.cu (mixed precision).
#pragma once
#include "dem_particle.cuh"

namespace b200dem {
namespace {

constexpr int kPairsBlock = 128;
// List entries the contact search tests per round: their index loads, then their position
// loads, are issued together (B200, dam-break state, FP64 step: 79.2 us with one entry per round,
// 76.8 us with two, 81.9 us with four -- more registers, fewer resident warps; testing the
// tracked slots the same way before the compaction, or prefetching the first two tracked
// partners with the own state, cost more registers than they saved: 82.1 and 83.8 us).
constexpr int kFindBatch = 2;
// The three kernels are compiled without a register cap: on the dam-break state (B200) caps of
// 80 / 64 registers for the per-contact and summing kernels (more resident blocks, spills) ran
// the step in 102.3 us against 95.1 us, and a contact search with 4 or 8 lanes per particle
// (the closed-form compaction of dem_contact_coop.cuh) in 114-132 us.

template <bool MIXED>
__global__ void __launch_bounds__(kPairsBlock) k_pairs_find(Particles P, NbrList L, Ctl *ctl, ForceConsts fc,
                                                            const WallGeom *__restrict__ walls) {
    grid_dep_wait();   // launched as a dependent (launch_k): the kernel before has completed
    grid_dep_release();
    const CtlSnap c = read_ctl(ctl, true);
    if (!c.go) return;
    const int cap = P.cap, n = P.n;
    const double4 *__restrict__ pc = P.pos[c.cur];
    int status = 0;
    for (int b = blockIdx.x * kPairsBlock; b < n; b += gridDim.x * kPairsBlock) {   // block-uniform
        const int i = b + threadIdx.x;
        int ncont = 0, nwc = 0, cs0 = 0, cnt = 0, nn = 0, wall0 = 0;
        unsigned cm[4] = {0u, 0u, 0u, 0u};   // contact flags of list entries 0..127
        unsigned wmask = 0u, wtouch = 0u;    // wall history bits; walls in contact this step
        int *tidx = P.tidx + i;
        double *thx = P.th + i;
        double *thy = P.th + (long)P.mc * cap + i;
        double *thz = P.th + 2L * P.mc * cap + i;
        D4 pi{};
        if (i < n) {
            pi = ld4(pc, i);
            cs0 = P.cstate[i];
            cnt = cs0 & 0xff;
            nn = L.nn[i];
            // ---- update_tangential_contacts (Force.hpp:364-441), as in particle_full
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
                        const long a = (long)k * cap, bb = (long)last_idx_tmp * cap;
                        if (k == last_idx_tmp) {
                            tidx[a] = -1;
                            thx[a] = 0.;
                            thy[a] = 0.;
                            thz[a] = 0.;
                        } else {
                            tidx[a] = tidx[bb];
                            tidx[bb] = -1;
                            thx[a] = thx[bb];
                            thx[bb] = 0.;
                            thy[a] = thy[bb];
                            thy[bb] = 0.;
                            thz[a] = thz[bb];
                            thz[bb] = 0.;
                            last_idx_tmp -= 1;
                        }
                        cnt -= 1;
                    } else {
                        k = k + 1;
                    }
                    count += 1;
                }
            }
            // ---- overlap test over the list (the pair loop's early-outs of particle_full)
            // (kFindBatch list entries per round: their index loads, then their position loads)
#pragma unroll 1
            for (int k0 = 0; k0 < nn; k0 += kFindBatch) {
                int jj[kFindBatch];
                D4 pj[kFindBatch];
#pragma unroll
                for (int u = 0; u < kFindBatch; ++u) jj[u] = k0 + u < nn ? L.idx[(long)(k0 + u) * cap + i] : -1;
#pragma unroll
                for (int u = 0; u < kFindBatch; ++u)
                    if (jj[u] >= 0) pj[u] = ld4(pc, jj[u]);
#pragma unroll
                for (int u = 0; u < kFindBatch; ++u) {
                    if (jj[u] < 0) continue;
                    const int kk = k0 + u;
                    const double px = pi.x - pj[u].x, py = pi.y - pj[u].y, pz = pi.z - pj[u].z;
                    const double r2ij = px * px + py * py + pz * pz;
                    const double sr = pi.w + pj[u].w;
                    if (r2ij >= sr * sr * 1.0000000001) continue;
                    const double rij = sqrt(r2ij);
                    const double overlap = sr - rij;
                    if (!(overlap > 0.)) continue;
                    cm[kk >> 5] |= 1u << (kk & 31);
                    ++ncont;
                }
            }
            // ---- particle-infinite wall overlaps (Force.hpp:475-490, 664-673)
            const int scene_i = P.scene ? P.scene[i] : 0;
            wall0 = fc.wps ? scene_i * fc.wps : 0;
            const int wall1 = fc.wps ? wall0 + fc.wps : fc.nwall;
            wmask = (unsigned)cs0 >> 8;
            for (int w = wall0; w < wall1; ++w) {
                const WallGeom *g = walls + w;
                const int lw = w - wall0;
                const double px = pi.x - __ldg(&g->x[0]), py = pi.y - __ldg(&g->x[1]), pz = pi.z - __ldg(&g->x[2]);
                const double tmp = px * __ldg(&g->n[0]) + py * __ldg(&g->n[1]) + pz * __ldg(&g->n[2]);
                const double overlap = pi.w - tmp;
                const unsigned bit = 1u << lw;
                if (overlap > 0.) {
                    wtouch |= bit;
                    ++nwc;
                } else if (wmask & bit) {
                    P.sw[(long)lw * cap + i] = 0.;
                    P.sw[(long)(P.mw + lw) * cap + i] = 0.;
                    P.sw[(long)(2 * P.mw + lw) * cap + i] = 0.;
                    wmask &= ~bit;
                }
            }
        }
        // contiguous items for the warp's particles, in lane order
        const int lane = threadIdx.x & 31;
        int incl = ncont + nwc;
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        const int wtotal = __shfl_sync(0xffffffffu, incl, 31);
        int wbase = 0;
        if (lane == 31 && wtotal) wbase = atomicAdd(&ctl->npairs, wtotal);
        wbase = __shfl_sync(0xffffffffu, wbase, 31);
        if (i < n) {
            int t = wbase + incl - ncont - nwc;
            L.prec[i] = make_int4(t, ncont, cs0, nwc);
            for (int w = 0; w < 4; ++w) {
                unsigned bits = cm[w];
                while (bits) {
                    const int kk = 32 * w + __ffs(bits) - 1;
                    bits &= bits - 1u;
                    const int j = L.idx[(long)kk * cap + i];
                    // slot lookup / insert (Force.hpp:166-192)
                    int found_at = -1;
                    for (int s = 0; s < cnt; ++s)
                        if (tidx[(long)s * cap] == j) found_at = s;
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
                    }
                    L.pitem[t++] = make_int4(i, j, found_at, 0);
                }
            }
            // wall items in wall order; the history flag is the bit before this step
            for (unsigned bits = wtouch; bits; bits &= bits - 1u) {
                const int lw = __ffs(bits) - 1;
                L.pitem[t++] = make_int4(i, -1 - (wall0 + lw), lw, (wmask >> lw) & 1u);
            }
            const int cs1 = cnt | (int)((wmask | wtouch) << 8);
            if (cs1 != cs0) P.cstate[i] = cs1;
        }
    }
    if (status) atomicOr(&ctl->status, status);
}

// One work item (k_pairs_find): the pair law with the pair's history slot, or the wall law with
// the wall's history; cf receives the item's F (0..2) and tau (3..5) on particle i.
template <bool MIXED>
__device__ __forceinline__ void pairs_item(const Particles &P, const ForceConsts &fc, const PairConst *__restrict__ pp,
                                           const PairConst *__restrict__ pw, const WallGeom *__restrict__ walls,
                                           const double4 *__restrict__ pc, const double *__restrict__ vc,
                                           const double *__restrict__ wc, const int4 it, double (&cf)[6]) {
    const int cap = P.cap;
    const unsigned q = fc.quirks;
    const int i = it.x, j = it.y, slot = it.z;
    const D4 pi = ld4(pc, i);
    const double ui0 = vc[i], ui1 = vc[cap + i], ui2 = vc[2 * cap + i];
    const double wi0 = wc[i], wi1 = wc[cap + i], wi2 = wc[2 * cap + i];
    const double m_i = P.mI[i];
    const int scene_i = P.scene ? P.scene[i] : 0;
    const SceneConst *scn = fc.scenes ? fc.scenes + scene_i : nullptr;
    const int mi = fc.nmat > 1 ? (int)P.mat[i] : 0;
    if (j < 0) {
        // wall item: j = -1 - wall, slot = the scene-local wall, it.w = wall history flag
        // (Force.hpp:475-673, pw_wall)
        const int w = -1 - j;
        const WallGeom *g = walls + w;
        const double px = pi.x - __ldg(&g->x[0]), py = pi.y - __ldg(&g->x[1]), pz = pi.z - __ldg(&g->x[2]);
        const double nx = __ldg(&g->n[0]), ny = __ldg(&g->n[1]), nz = __ldg(&g->n[2]);
        const double tmp = px * nx + py * ny + pz * nz;
        const double overlap = pi.w - tmp;
        const double K_n_pw = scn ? scn->K_n_pw : fc.K_n_pw, K_t_pw = scn ? scn->K_t_pw : fc.K_t_pw;
        const double mu_pw = scn ? scn->mu_pw : fc.mu_pw;
        double *swx = P.sw + (long)slot * cap + i;
        double *swy = P.sw + (long)(P.mw + slot) * cap + i;
        double *swz = P.sw + (long)(2 * P.mw + slot) * cap + i;
        pw_wall<MIXED>(q, pi, nx, ny, nz, overlap, ui0, ui1, ui2, wi0, wi1, wi2, __ldg(&g->u[0]), __ldg(&g->u[1]),
                       __ldg(&g->u[2]), m_i, pw[mi * fc.nwall + w], K_n_pw, K_t_pw, mu_pw, fc.dt, it.w != 0, swx,
                       swy, swz, cf);
    } else {
        const D4 pj = ld4(pc, j);
        const double K_n_pp = scn ? scn->K_n_pp : fc.K_n_pp, K_t_pp = scn ? scn->K_t_pp : fc.K_t_pp;
        const double mu_pp = scn ? scn->mu_pp : fc.mu_pp;
        const int mj = fc.nmat > 1 ? (int)P.mat[j] : 0;
        const double px = pi.x - pj.x, py = pi.y - pj.y, pz = pi.z - pj.z;
        const double r2ij = px * px + py * py + pz * pz;
        const double sr = pi.w + pj.w;
        const double rij = sqrt(r2ij);
        const double overlap = sr - rij;
        double *hx = P.th + (long)slot * cap + i;
        double *hy = P.th + ((long)P.mc + slot) * cap + i;
        double *hz = P.th + (2L * P.mc + slot) * cap + i;
        double h0 = 0., h1 = 0., h2 = 0.;
        if (slot >= 0) {
            h0 = *hx;
            h1 = *hy;
            h2 = *hz;
        }
        pp_pair<MIXED>(P.mI, vc, wc, cap, q, pi, pj, j, px, py, pz, rij, overlap, ui0, ui1, ui2, wi0, wi1, wi2,
                       m_i, pp[mi * fc.nmat + mj], K_n_pp, K_t_pp, mu_pp, fc.dt, h0, h1, h2, cf);
        if (slot >= 0) {
            *hx = h0;
            *hy = h1;
            *hz = h2;
        }
    }
}

template <bool MIXED>
__global__ void __launch_bounds__(kPairsBlock) k_pairs_eval(Particles P, NbrList L, Ctl *ctl, ForceConsts fc,
                                                            const PairConst *__restrict__ pp,
                                                            const PairConst *__restrict__ pw,
                                                            const WallGeom *__restrict__ walls) {
    grid_dep_wait();   // launched as a dependent (launch_k): the kernel before has completed
    grid_dep_release();
    const CtlSnap c = read_ctl(ctl, true);
    if (!c.go) return;
    const int np = ctl->npairs;
    const double4 *__restrict__ pc = P.pos[c.cur];
    const int vcur = ctl->vcur;
    const double *__restrict__ vc = P.vel[vcur];
    const double *__restrict__ wc = P.omg[vcur];
    for (int t = blockIdx.x * kPairsBlock + threadIdx.x; t < np; t += gridDim.x * kPairsBlock) {
        double cf[6];
        pairs_item<MIXED>(P, fc, pp, pw, walls, pc, vc, wc, L.pitem[t], cf);
        double2 *term = L.pterm + 3L * t;
        term[0] = make_double2(cf[0], cf[1]);
        term[1] = make_double2(cf[2], cf[3]);
        term[2] = make_double2(cf[4], cf[5]);
    }
}

// The mesh pass of k_pairs_sum, out of line, with the scene's wall constants looked up inside.
template <bool MIXED>
__device__ __noinline__ int mesh_contacts(const Particles &P, const ForceConsts &fc, const int i, const int scene_i,
                                          const D4 pi, const double ui0, const double ui1, const double ui2,
                                          const double wi0, const double wi1, const double wi2, const double m_i,
                                          const int mi, double *FT, int *status) {
    const SceneConst *scn = fc.scenes ? fc.scenes + scene_i : nullptr;
    const double K_n_pw = scn ? scn->K_n_pw : fc.K_n_pw, K_t_pw = scn ? scn->K_t_pw : fc.K_t_pw;
    const double mu_pw = scn ? scn->mu_pw : fc.mu_pw;
    return mesh_pass<MIXED>(P, fc, i, pi, ui0, ui1, ui2, wi0, wi1, wi2, m_i, mi, K_n_pw, K_t_pw, mu_pw, FT, status);
}

// The hooks after the pair forces and the velocity-Verlet update of particle i (stage3 of this
// step, stage1 + stage2 of the next, or F and tau stored after the run's last step); positions
// and velocities to the other buffers.
__device__ __forceinline__ void pairs_integrate(const Particles &P, const ForceConsts &fc, const CtlSnap &c,
                                                const int vcur, const int i, const D4 &pi, double ui0, double ui1,
                                                double ui2, double wi0, double wi1, double wi2, const double2 mIi,
                                                double F0, double F1, double F2, double T0, double T1, double T2,
                                                double &vmax2) {
    const int cap = P.cap, nxt = c.cur ^ 1;
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
    // stage3 of this step
    ui0 = dadd(ui0, dmul(dmul(h, F0), m_inverse));
    ui1 = dadd(ui1, dmul(dmul(h, F1), m_inverse));
    ui2 = dadd(ui2, dmul(dmul(h, F2), m_inverse));
    wi0 = dadd(wi0, dmul(dmul(h, T0), I_inverse));
    wi1 = dadd(wi1, dmul(dmul(h, T1), I_inverse));
    wi2 = dadd(wi2, dmul(dmul(h, T2), I_inverse));
    D4 pn = pi;
    if (c.last) {
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
        vmax2 = fmax(vmax2, dadd(dadd(dmul(ui0, ui0), dmul(ui1, ui1)), dmul(ui2, ui2)));
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

template <bool MIXED, bool MESH>
__global__ void __launch_bounds__(kPairsBlock) k_pairs_sum(Particles P, NbrList L, Ctl *ctl, ForceConsts fc) {
    grid_dep_wait();   // launched as a dependent (launch_k): the kernel before has completed
    grid_dep_release();
    const CtlSnap c = read_ctl(ctl, true);
    if (!c.go) return;
    const int cap = P.cap, vcur = ctl->vcur;
    const unsigned q = fc.quirks;
    const double4 *__restrict__ pc = P.pos[c.cur];
    const double *__restrict__ vc = P.vel[vcur];
    const double *__restrict__ wc = P.omg[vcur];
    double vmax2 = 0.0;
    int status = 0, active = 0;
    for (int i = blockIdx.x * kPairsBlock + threadIdx.x; i < P.n; i += gridDim.x * kPairsBlock) {
        const int4 rec = L.prec[i];
        const D4 pi = ld4(pc, i);
        double ui0 = vc[i], ui1 = vc[cap + i], ui2 = vc[2 * cap + i];
        double wi0 = wc[i], wi1 = wc[cap + i], wi2 = wc[2 * cap + i];
        const double2 mIi = load_mI(P, i);
        const int cs = P.cstate[i];   // the count and wall bits k_pairs_find left
        double F0 = 0., F1 = 0., F2 = 0., T0 = 0., T1 = 0., T2 = 0.;
        if (fc.has_ext) {
            F0 += P.ext[i];
            F1 += P.ext[cap + i];
            F2 += P.ext[2 * cap + i];
        }
        const int tp = rec.x + rec.y;
        for (int t = rec.x; t < tp; ++t) {   // pair terms in list order
            const double2 *term = L.pterm + 3L * t;
            const double2 a = term[0], b = term[1], d = term[2];
            F0 += a.x;
            F1 += a.y;
            F2 += b.x;
            if (!(q & DEM_Q3_NO_PP_TORQUE)) {
                T0 += b.y;
                T1 += d.x;
                T2 += d.y;
            }
        }
        for (int t = tp; t < tp + rec.w; ++t) {   // wall terms in wall order (Force.hpp:664-670)
            const double2 *term = L.pterm + 3L * t;
            const double2 a = term[0], b = term[1], d = term[2];
            F0 += a.x;
            F1 += a.y;
            F2 += b.x;
            T0 += b.y;
            T1 += d.x;
            T2 += d.y;
        }
        int mcnt = 0;
        if constexpr (MESH) {
            const int scene_i = P.scene ? P.scene[i] : 0;
            const int mi = fc.nmat > 1 ? (int)P.mat[i] : 0;
            double FT[6] = {F0, F1, F2, T0, T1, T2};
            mcnt = mesh_contacts<MIXED>(P, fc, i, scene_i, pi, ui0, ui1, ui2, wi0, wi1, wi2, mIi.x, mi, FT, &status);
            F0 = FT[0];
            F1 = FT[1];
            F2 = FT[2];
            T0 = FT[3];
            T1 = FT[4];
            T2 = FT[5];
        }
        active += ((rec.z | cs) != 0 || mcnt != 0) ? 1 : 0;
        pairs_integrate(P, fc, c, vcur, i, pi, ui0, ui1, ui2, wi0, wi1, wi2, mIi, F0, F1, F2, T0, T1, T2, vmax2);
    }
    finish_step_counted(ctl, P.vslots, vmax2, fc.dt, status, active, fc, !c.last);
}


}  // namespace
}  // namespace b200dem

namespace b200dem {
namespace {
// Launches the contact search of the pair-parallel step on a persistent grid.
template <bool MIXED>
inline void launch_pairs_find(const Particles &P, const NbrList &L, Ctl *ctl, const ForceConsts &fc,
                              const WallGeom *walls, int sms, cudaStream_t s) {
    int per = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pairs_find<MIXED>, kPairsBlock, 0);
    const long need = ((long)P.n + kPairsBlock - 1) / kPairsBlock;
    const long g = need < (long)sms * (per > 0 ? per : 1) ? need : (long)sms * (per > 0 ? per : 1);
    launch_k(k_pairs_find<MIXED>, (int)(g > 0 ? g : 1), kPairsBlock, 0, s, fc.pdl, P, L, ctl, fc, walls);
}
}  // namespace
}  // namespace b200dem
