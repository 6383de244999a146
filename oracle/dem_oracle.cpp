// dem_oracle.cpp -- CPU oracle for the CabanaDEM contact step (TEST INFRASTRUCTURE).
//
// Only tests/, the smoke check and bench.py's CPU-baseline leg use this library, as the
// checker.  Every function restates the reference file:line it cites, keeping the
// reference's expression order so that FP64 results can be compared bit for bit.
// Build flags keep that order: -O2 -ffp-contract=off -fno-fast-math (see Makefile).
#include "dem_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

inline double pow15(double x, int mode) { return mode == ORC_POW_SQRT ? x * std::sqrt(x) : std::pow(x, 1.5); }
inline double pow05(double x, int mode) { return mode == ORC_POW_SQRT ? std::sqrt(x) : std::pow(x, 0.5); }

// The contact law of src/CabanaDEM_Force.hpp:561-664 between particle i and a plane through
// its contact point: unit normal (nij_x, nij_y, nij_z) towards the particle, overlap > 0, the
// wall's material and velocity (vel_j; zero for the reference's static walls, :529), and the
// contact's tangential history (swx, swy, swz), read and written.  Adds to F and tau of i.
void plane_contact(orc_particles *p, int i, double nij_x, double nij_y, double nij_z, double overlap, double E_w,
                   double nu_w, double G_w, const double vel_j[3], double *swx, double *swy, double *swz,
                   const orc_force_params *fp, double dt) {
    const unsigned q = fp->quirks;
    const int pm = fp->pow_mode;
    const double cor_pw = fp->cor_pw, friction_pw = fp->mu_pw;
    const double *u = p->u, *omega = p->omega, *rad = p->rad, *m = p->m;
    double a_i = rad[i] - overlap / 2.;
    double vel_i[3];
    vel_i[0] = u[3 * i + 0] + (omega[3 * i + 1] * nij_z - omega[3 * i + 2] * nij_y) * a_i;
    vel_i[1] = u[3 * i + 1] + (omega[3 * i + 2] * nij_x - omega[3 * i + 0] * nij_z) * a_i;
    vel_i[2] = u[3 * i + 2] + (omega[3 * i + 0] * nij_y - omega[3 * i + 1] * nij_x) * a_i;
    double vel_ij[3] = {vel_i[0] - vel_j[0], vel_i[1] - vel_j[1], vel_i[2] - vel_j[2]};
    double vij_dot_nij = vel_ij[0] * nij_x + vel_ij[1] * nij_y + vel_ij[2] * nij_z;
    double vn_x = vij_dot_nij * nij_x;
    double vn_y = vij_dot_nij * nij_y;
    double vn_z = vij_dot_nij * nij_z;
    double vt_x = vel_ij[0] - vn_x;
    double vt_y = vel_ij[1] - vn_y;
    double vt_z = vel_ij[2] - vn_z;
    double tmp_1 = (1. - (p->nu[i] * p->nu[i])) / p->E[i];
    double tmp_2 = (1. - (nu_w * nu_w)) / E_w;
    double E_eff = 1. / (tmp_1 + tmp_2);
    double tmp_3 = 1. / rad[i];
    double tmp_4 = 0.;
    double R_eff = 1. / (tmp_3 + tmp_4);
    double kn = 4. / 3. * E_eff * std::sqrt(R_eff);
    tmp_1 = std::log(cor_pw);
    tmp_2 = tmp_1 * tmp_1 + M_PI * M_PI;
    double beta = tmp_1 / std::sqrt(tmp_2);
    double S_n = 2. * E_eff * std::sqrt(R_eff * overlap);
    tmp_1 = 1. / m[i];
    tmp_2 = 0.;
    double m_eff = 1. / (tmp_1 + tmp_2);
    double eta_n = -2. * std::sqrt(5. / 6.) * beta * std::sqrt(S_n * m_eff);
    double fn = kn * pow15(overlap, pm);
    double fn_x = fn * nij_x - eta_n * vn_x;
    double fn_y = fn * nij_y - eta_n * vn_y;
    double fn_z = fn * nij_z - eta_n * vn_z;
    double ft_x = 0., ft_y = 0., ft_z = 0.;
    double vij_magn = std::sqrt(vel_ij[0] * vel_ij[0] + vel_ij[1] * vel_ij[1] + vel_ij[2] * vel_ij[2]);
    if (vij_magn < 1e-12) {
        *swx = 0.;
        *swy = 0.;
        *swz = 0.;
    } else {
        *swx += vt_x * dt;
        *swy += vt_y * dt;
        *swz += vt_z * dt;
        tmp_1 = (2. - p->nu[i]) / p->G[i];
        tmp_2 = (2. - nu_w) / G_w;
        double G_eff = 1. / (tmp_1 + tmp_2);
        double kt = 8. * G_eff * std::sqrt(R_eff * overlap);
        double S_t = kt;
        double eta_t = (q & ORC_Q2_ETA_T_ZERO) ? -2 * std::sqrt((double)(5 / 6)) * beta * std::sqrt(S_t * m_eff)
                                               : -2. * std::sqrt(5. / 6.) * beta * std::sqrt(S_t * m_eff);
        double ft_x_star = -kt * *swx - eta_t * vt_x;
        double ft_y_star = -kt * *swy - eta_t * vt_y;
        double ft_z_star = -kt * *swz - eta_t * vt_z;
        double ft_magn = (q & ORC_Q5_WALL_FT_TYPO)
                             ? std::sqrt(ft_x_star * ft_x_star + ft_y_star * ft_y_star + ft_z_star * ft_y_star)
                             : std::sqrt(ft_x_star * ft_x_star + ft_y_star * ft_y_star + ft_z_star * ft_z_star);
        double ti_x = 0., ti_y = 0., ti_z = 0.;
        if (ft_magn > 1e-12) {
            ti_x = ft_x_star / ft_magn;
            ti_y = ft_y_star / ft_magn;
            ti_z = ft_z_star / ft_magn;
        }
        double fn_magn = std::sqrt(fn_x * fn_x + fn_y * fn_y + fn_z * fn_z);
        double ft_magn_star = std::min(friction_pw * fn_magn, ft_magn);
        ft_x = ft_magn_star * ti_x;
        ft_y = ft_magn_star * ti_y;
        ft_z = ft_magn_star * ti_z;
        ft_x += eta_t * vt_x;
        ft_y += eta_t * vt_y;
        ft_z += eta_t * vt_z;
        *swx = -ft_x / kt;
        *swy = -ft_y / kt;
        *swz = -ft_z / kt;
        if (!(q & ORC_Q2_ETA_T_ZERO)) {
            // with eta_t live (Q2 clear) the limited force is what acts; the damping is added
            // back (:640-643) only to reset the spring above.  The reference applies the sum,
            // which pushes a sliding contact along its sliding direction (eta_t = 0 there).
            ft_x = ft_magn_star * ti_x;
            ft_y = ft_magn_star * ti_y;
            ft_z = ft_magn_star * ti_z;
        }
    }
    p->force[3 * i + 0] += fn_x + ft_x;
    p->force[3 * i + 1] += fn_y + ft_y;
    p->force[3 * i + 2] += fn_z + ft_z;
    p->torque[3 * i + 0] += (nij_y * ft_z - nij_z * ft_y) * a_i;
    p->torque[3 * i + 1] += (nij_z * ft_x - nij_x * ft_z) * a_i;
    p->torque[3 * i + 2] += (nij_x * ft_y - nij_y * ft_x) * a_i;
}

}  // namespace

// ---------------------------------------------------------------------------------
// Neighbour list: the Cabana VerletList (FullNeighborTag) restated as every j != i
// with |x_i - x_j|^2 <= cutoff^2, listed in ascending j.  Call sites it replaces:
// src/CabanaDEM_Solver.hpp:61-63, :87-88; src/CabanaBondedDEM_Particles.hpp:155-157.
// ---------------------------------------------------------------------------------
struct orc_nlist {
    int n = 0;
    std::vector<int> offsets;
    std::vector<int> idx;
};

extern "C" orc_nlist *orc_nlist_create(void) { return new orc_nlist(); }
extern "C" void orc_nlist_destroy(orc_nlist *nl) { delete nl; }
extern "C" long orc_nlist_total(const orc_nlist *nl) { return (long)nl->idx.size(); }
extern "C" void orc_nlist_copy(const orc_nlist *nl, int *offsets, int *idx) {
    std::memcpy(offsets, nl->offsets.data(), sizeof(int) * (nl->n + 1));
    if (!nl->idx.empty()) std::memcpy(idx, nl->idx.data(), sizeof(int) * nl->idx.size());
}

extern "C" int orc_nlist_build(orc_nlist *nl, const orc_particles *p, double delta, double skin) {
    const int n = p->n;
    nl->n = n;
    nl->offsets.assign(n + 1, 0);
    nl->idx.clear();
    if (n == 0) return 0;
    double rmax = 0.0;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = 0; i < n; ++i) {
        rmax = std::max(rmax, p->rad[i]);
        for (int d = 0; d < 3; ++d) {
            lo[d] = std::min(lo[d], p->x[3 * i + d]);
            hi[d] = std::max(hi[d], p->x[3 * i + d]);
        }
    }
    const double cutmax = delta > 0.0 ? delta : 2.0 * rmax + skin;
    double cell = cutmax > 0.0 ? cutmax : 1.0;
    long dims[3];
    for (;;) {
        long tot = 1;
        for (int d = 0; d < 3; ++d) {
            dims[d] = (long)std::floor((hi[d] - lo[d]) / cell) + 1;
            tot *= dims[d];
        }
        if (tot <= std::max(64L, 8L * n)) break;
        cell *= 1.26;
    }
    const long ncell = dims[0] * dims[1] * dims[2];
    std::vector<int> cell_of(n);
    std::vector<int> cstart(ncell + 1, 0), order(n);
    for (int i = 0; i < n; ++i) {
        long c[3];
        for (int d = 0; d < 3; ++d) {
            c[d] = (long)std::floor((p->x[3 * i + d] - lo[d]) / cell);
            c[d] = std::min(std::max(c[d], 0L), dims[d] - 1);
        }
        cell_of[i] = (int)((c[2] * dims[1] + c[1]) * dims[0] + c[0]);
        cstart[cell_of[i] + 1]++;
    }
    for (long c = 0; c < ncell; ++c) cstart[c + 1] += cstart[c];
    {
        std::vector<int> fill(cstart.begin(), cstart.end() - 1);
        for (int i = 0; i < n; ++i) order[fill[cell_of[i]]++] = i;
    }
    auto visit = [&](int i, std::vector<int> &out) {
        out.clear();
        const int ci = cell_of[i];
        const long cx = ci % dims[0], cy = (ci / dims[0]) % dims[1], cz = ci / (dims[0] * dims[1]);
        for (long dz = -1; dz <= 1; ++dz)
            for (long dy = -1; dy <= 1; ++dy)
                for (long dx = -1; dx <= 1; ++dx) {
                    const long x = cx + dx, y = cy + dy, z = cz + dz;
                    if (x < 0 || y < 0 || z < 0 || x >= dims[0] || y >= dims[1] || z >= dims[2]) continue;
                    const long c = (z * dims[1] + y) * dims[0] + x;
                    for (int s = cstart[c]; s < cstart[c + 1]; ++s) {
                        const int j = order[s];
                        if (j == i) continue;
                        const double px = p->x[3 * i + 0] - p->x[3 * j + 0];
                        const double py = p->x[3 * i + 1] - p->x[3 * j + 1];
                        const double pz = p->x[3 * i + 2] - p->x[3 * j + 2];
                        const double r2 = px * px + py * py + pz * pz;
                        const double cut = delta > 0.0 ? delta : p->rad[i] + p->rad[j] + skin;
                        if (r2 <= cut * cut) out.push_back(j);
                    }
                }
        std::sort(out.begin(), out.end());
    };
    std::vector<int> counts(n);
#pragma omp parallel
    {
        std::vector<int> buf;
#pragma omp for schedule(static)
        for (int i = 0; i < n; ++i) {
            visit(i, buf);
            counts[i] = (int)buf.size();
        }
    }
    for (int i = 0; i < n; ++i) nl->offsets[i + 1] = nl->offsets[i] + counts[i];
    nl->idx.resize(nl->offsets[n]);
#pragma omp parallel
    {
        std::vector<int> buf;
#pragma omp for schedule(static)
        for (int i = 0; i < n; ++i) {
            visit(i, buf);
            std::copy(buf.begin(), buf.end(), nl->idx.begin() + nl->offsets[i]);
        }
    }
    return 0;
}

// ---------------------------------------------------------------------------------
// Integrator: src/CabanaDEM_Integrator.hpp:31-56 (stage1), :59-74 (stage2),
// :77-102 (stage3).  _half_dt = 0.5 * dt (:25).
// ---------------------------------------------------------------------------------
extern "C" void orc_stage1(orc_particles *p, double dt) {
    const double half_dt = 0.5 * dt;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < p->n; ++i) {
        double m_inverse = 1. / p->m[i];
        for (int d = 0; d < 3; ++d) p->u[3 * i + d] += half_dt * p->force[3 * i + d] * m_inverse;
        double I_inverse = 1. / p->I[i];
        for (int d = 0; d < 3; ++d) p->omega[3 * i + d] += half_dt * p->torque[3 * i + d] * I_inverse;
    }
}

extern "C" void orc_stage2(orc_particles *p, double dt) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < p->n; ++i)
        for (int d = 0; d < 3; ++d) p->x[3 * i + d] += dt * p->u[3 * i + d];
}

extern "C" void orc_stage2_walls(const orc_walls *w, double dt) {
    if (!w || !w->u) return;
    for (int j = 0; j < w->n; ++j)
        for (int d = 0; d < 3; ++d) w->x[3 * j + d] += dt * w->u[3 * j + d];
}

extern "C" void orc_stage3(orc_particles *p, double dt) { orc_stage1(p, dt); }

// src/CabanaDEM_Force.hpp:40-47
extern "C" void orc_zero_force(orc_particles *p) {
    std::memset(p->force, 0, sizeof(double) * 3 * p->n);
    std::memset(p->torque, 0, sizeof(double) * 3 * p->n);
}

// ---------------------------------------------------------------------------------
// src/CabanaDEM_Force.hpp:344-445: drop every tracked contact whose pair no longer
// overlaps, by swapping the last slot into its place.
// ---------------------------------------------------------------------------------
extern "C" void orc_update_tangential_contacts(orc_particles *p) {
    const int mc = p->max_cnts;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < p->n; ++i) {
        int *idx = p->tng_idx + (long)i * mc;
        double *hx = p->tng_ss_x + (long)i * mc, *hy = p->tng_ss_y + (long)i * mc, *hz = p->tng_ss_z + (long)i * mc;
        int count = 0;
        int k = 0;
        int idx_total_ctcs = p->tng_count[i];
        int last_idx_tmp = p->tng_count[i] - 1;
        int sidx = -1;
        while (count < idx_total_ctcs) {
            sidx = idx[k];
            if (sidx == -1) break;
            const double pos_ij[3] = {p->x[3 * i + 0] - p->x[3 * sidx + 0], p->x[3 * i + 1] - p->x[3 * sidx + 1],
                                      p->x[3 * i + 2] - p->x[3 * sidx + 2]};
            double r2ij = pos_ij[0] * pos_ij[0] + pos_ij[1] * pos_ij[1] + pos_ij[2] * pos_ij[2];
            double rij = std::sqrt(r2ij);
            double overlap = p->rad[i] + p->rad[sidx] - rij;
            if (overlap <= 0.) {
                if (k == last_idx_tmp) {
                    idx[k] = -1;
                    hx[k] = 0.;
                    hy[k] = 0.;
                    hz[k] = 0.;
                } else {
                    idx[k] = idx[last_idx_tmp];
                    idx[last_idx_tmp] = -1;
                    hx[k] = hx[last_idx_tmp];
                    hx[last_idx_tmp] = 0.;
                    hy[k] = hy[last_idx_tmp];
                    hy[last_idx_tmp] = 0.;
                    hz[k] = hz[last_idx_tmp];
                    hz[last_idx_tmp] = 0.;
                    last_idx_tmp -= 1;
                }
                p->tng_count[i] -= 1;
            } else {
                k = k + 1;
            }
            count += 1;
        }
    }
}

// ---------------------------------------------------------------------------------
// src/CabanaDEM_Force.hpp:50-341: Hertz normal + Mindlin tangential, full list,
// serial per particle i (neighbor_parallel_for with SerialOpTag, :334-339).
// ---------------------------------------------------------------------------------
extern "C" int orc_force_pp(orc_particles *p, const orc_nlist *nl, const orc_force_params *fp, double dt) {
    const int mc = p->max_cnts;
    const unsigned q = fp->quirks;
    const int pm = fp->pow_mode;
    const double cor_pp = fp->cor_pp, friction_pp = fp->mu_pp;
    int status = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(| : status)
    for (int i = 0; i < p->n; ++i) {
        const double *x = p->x, *u = p->u, *omega = p->omega, *rad = p->rad, *m = p->m;
        const double *E = p->E, *nu = p->nu, *G = p->G;
        int *tidx = p->tng_idx + (long)i * mc;
        double *hx = p->tng_ss_x + (long)i * mc, *hy = p->tng_ss_y + (long)i * mc, *hz = p->tng_ss_z + (long)i * mc;
        for (int s = nl->offsets[i]; s < nl->offsets[i + 1]; ++s) {
            const int j = nl->idx[s];
            double pos_ij[3] = {x[3 * i + 0] - x[3 * j + 0], x[3 * i + 1] - x[3 * j + 1], x[3 * i + 2] - x[3 * j + 2]};
            double r2ij = pos_ij[0] * pos_ij[0] + pos_ij[1] * pos_ij[1] + pos_ij[2] * pos_ij[2];
            double rij = std::sqrt(r2ij);
            double overlap = rad[i] + rad[j] - rij;
            double a_i = rad[i] - overlap / 2.;
            double a_j = rad[j] - overlap / 2.;
            double nij_x = pos_ij[0] / rij;
            double nij_y = pos_ij[1] / rij;
            double nij_z = pos_ij[2] / rij;
            double vel_i[3];
            vel_i[0] = u[3 * i + 0] + (omega[3 * i + 1] * nij_z - omega[3 * i + 2] * nij_y) * a_i;
            vel_i[1] = u[3 * i + 1] + (omega[3 * i + 2] * nij_x - omega[3 * i + 0] * nij_z) * a_i;
            vel_i[2] = u[3 * i + 2] + (omega[3 * i + 0] * nij_y - omega[3 * i + 1] * nij_x) * a_i;
            const double uj1 = (q & ORC_Q1_VELJ_USES_UI) ? u[3 * i + 1] : u[3 * j + 1];
            const double uj2 = (q & ORC_Q1_VELJ_USES_UI) ? u[3 * i + 2] : u[3 * j + 2];
            double vel_j[3];
            vel_j[0] = u[3 * j + 0] + (-omega[3 * j + 1] * nij_z + omega[3 * j + 2] * nij_y) * a_j;
            vel_j[1] = uj1 + (-omega[3 * j + 2] * nij_x + omega[3 * j + 0] * nij_z) * a_j;
            vel_j[2] = uj2 + (-omega[3 * j + 0] * nij_y + omega[3 * j + 1] * nij_x) * a_j;
            double vel_ij[3] = {vel_i[0] - vel_j[0], vel_i[1] - vel_j[1], vel_i[2] - vel_j[2]};
            double vij_dot_nij = vel_ij[0] * nij_x + vel_ij[1] * nij_y + vel_ij[2] * nij_z;
            double vn_x = vij_dot_nij * nij_x;
            double vn_y = vij_dot_nij * nij_y;
            double vn_z = vij_dot_nij * nij_z;
            double vt_x = vel_ij[0] - vn_x;
            double vt_y = vel_ij[1] - vn_y;
            double vt_z = vel_ij[2] - vn_z;
            if (!(overlap > 0.)) continue;
            // slot lookup / insert (:166-192); overflow is reported instead of written out of bounds
            int found = 0, found_at = -1;
            for (int k = 0; k < p->tng_count[i]; ++k)
                if (j == tidx[k]) {
                    found = 1;
                    found_at = k;
                }
            double hist[3] = {0., 0., 0.};
            if (found == 0) {
                if (p->tng_count[i] < mc) {
                    p->tng_count[i] += 1;
                    found_at = p->tng_count[i] - 1;
                    tidx[found_at] = j;
                    hx[found_at] = 0.;
                    hy[found_at] = 0.;
                    hz[found_at] = 0.;
                } else {
                    status |= ORC_ERR_CONTACT_OVERFLOW;
                    found_at = -1;
                }
            }
            if (found_at >= 0) {
                hist[0] = hx[found_at];
                hist[1] = hy[found_at];
                hist[2] = hz[found_at];
            }
            double tmp_1 = (1. - (nu[i] * nu[i])) / E[i];
            double tmp_2 = (1. - (nu[j] * nu[j])) / E[j];
            double E_eff = 1. / (tmp_1 + tmp_2);
            double tmp_3 = 1. / rad[i];
            double tmp_4 = 1. / rad[j];
            double R_eff = 1. / (tmp_3 + tmp_4);
            double kn = 4. / 3. * E_eff * std::sqrt(R_eff);
            tmp_1 = std::log(cor_pp);
            tmp_2 = tmp_1 * tmp_1 + M_PI * M_PI;
            double beta = tmp_1 / std::sqrt(tmp_2);
            double S_n = 2. * E_eff * std::sqrt(R_eff * overlap);
            tmp_1 = 1. / m[i];
            tmp_2 = 1. / m[j];
            double m_eff = 1. / (tmp_1 + tmp_2);
            double eta_n = -2. * std::sqrt(5. / 6.) * beta * std::sqrt(S_n * m_eff);
            tmp_1 = (2. - nu[i]) / G[i];
            tmp_2 = (2. - nu[j]) / G[j];
            double G_eff = 1. / (tmp_1 + tmp_2);
            double kt = 8. * G_eff * std::sqrt(R_eff * overlap);
            double S_t = kt;
            double eta_t = (q & ORC_Q2_ETA_T_ZERO) ? -2 * std::sqrt((double)(5 / 6)) * beta * std::sqrt(S_t * m_eff)
                                                   : -2. * std::sqrt(5. / 6.) * beta * std::sqrt(S_t * m_eff);
            double fn = kn * pow15(overlap, pm);
            double fn_x = fn * nij_x - eta_n * vn_x;
            double fn_y = fn * nij_y - eta_n * vn_y;
            double fn_z = fn * nij_z - eta_n * vn_z;
            double tf_x = 0., tf_y = 0., tf_z = 0.;
            double vij_magn = pow05(vel_ij[0] * vel_ij[0] + vel_ij[1] * vel_ij[1] + vel_ij[2] * vel_ij[2], pm);
            if (vij_magn < 1e-12) {
                hist[0] = 0.;
                hist[1] = 0.;
                hist[2] = 0.;
            } else {
                double tx_tmp = vel_ij[0] - nij_x * vij_dot_nij;
                double ty_tmp = vel_ij[1] - nij_y * vij_dot_nij;
                double tz_tmp = vel_ij[2] - nij_z * vij_dot_nij;
                double ti_magn = pow05(tx_tmp * tx_tmp + ty_tmp * ty_tmp + tz_tmp * tz_tmp, pm);
                double ti_x = 0., ti_y = 0., ti_z = 0.;
                if (ti_magn > 1e-12) {
                    ti_x = tx_tmp / ti_magn;
                    ti_y = ty_tmp / ti_magn;
                    ti_z = tz_tmp / ti_magn;
                }
                double dlx = hist[0] + vel_ij[0] * dt;
                double dly = hist[1] + vel_ij[1] * dt;
                double dlz = hist[2] + vel_ij[2] * dt;
                double dl_dot_ti = (dlx * ti_x + dly * ti_y + dlz * ti_z);
                hist[0] = dl_dot_ti * ti_x;
                hist[1] = dl_dot_ti * ti_y;
                hist[2] = dl_dot_ti * ti_z;
                double ftx = -kt * hist[0] - eta_t * vt_x;
                double fty = -kt * hist[1] - eta_t * vt_y;
                double ftz = -kt * hist[2] - eta_t * vt_z;
                double ft_magn = pow05(ftx * ftx + fty * fty + ftz * ftz, pm);
                double fn_magn = pow05(fn_x * fn_x + fn_y * fn_y + fn_z * fn_z, pm);
                double ft_magn_star = ft_magn;
                if (ft_magn_star > friction_pp * fn_magn) ft_magn_star = friction_pp * fn_magn;
                tf_x = -ft_magn_star * ti_x;
                tf_y = -ft_magn_star * ti_y;
                tf_z = -ft_magn_star * ti_z;
                double mdx = -tf_x / kt;
                double mdy = -tf_y / kt;
                double mdz = -tf_z / kt;
                if (q & ORC_Q4_UNIT_HISTORY) {
                    double lt_magn = pow05(mdx * mdx + mdy * mdy + mdz * mdz, pm);
                    if (lt_magn > 1e-12) {
                        hist[0] = mdx / lt_magn;
                        hist[1] = mdy / lt_magn;
                        hist[2] = mdz / lt_magn;
                    } else {
                        hist[0] = 0.;
                        hist[1] = 0.;
                        hist[2] = 0.;
                    }
                } else {
                    hist[0] = mdx;
                    hist[1] = mdy;
                    hist[2] = mdz;
                }
            }
            if (found_at >= 0) {
                hx[found_at] = hist[0];
                hy[found_at] = hist[1];
                hz[found_at] = hist[2];
            }
            p->force[3 * i + 0] += fn_x + tf_x;
            p->force[3 * i + 1] += fn_y + tf_y;
            p->force[3 * i + 2] += fn_z + tf_z;
            if (!(q & ORC_Q3_NO_PP_TORQUE)) {
                p->torque[3 * i + 0] += (nij_y * tf_z - nij_z * tf_y) * a_i;
                p->torque[3 * i + 1] += (nij_z * tf_x - nij_x * tf_z) * a_i;
                p->torque[3 * i + 2] += (nij_x * tf_y - nij_y * tf_x) * a_i;
            }
        }
    }
    return status;
}

// ---------------------------------------------------------------------------------
// src/CabanaDEM_Force.hpp:448-678: particle against each infinite plane, in wall order.
// Wall velocity is not used (:529, Q6); with Q6 clear vel_j is the wall's velocity.
// ---------------------------------------------------------------------------------
extern "C" void orc_force_wall(orc_particles *p, const orc_walls *w, const orc_force_params *fp, double dt) {
    const int mw = p->max_walls;
    const unsigned q = fp->quirks;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < p->n; ++i) {
        const double *x = p->x, *rad = p->rad;
        for (int j = 0; j < w->n; ++j) {
            double *swx = p->tng_sw_x + (long)i * mw + j, *swy = p->tng_sw_y + (long)i * mw + j,
                   *swz = p->tng_sw_z + (long)i * mw + j;
            double pos_ij[3] = {x[3 * i + 0] - w->x[3 * j + 0], x[3 * i + 1] - w->x[3 * j + 1],
                                x[3 * i + 2] - w->x[3 * j + 2]};
            double nij_x = w->normal[3 * j + 0];
            double nij_y = w->normal[3 * j + 1];
            double nij_z = w->normal[3 * j + 2];
            double tmp = pos_ij[0] * nij_x + pos_ij[1] * nij_y + pos_ij[2] * nij_z;
            double overlap = rad[i] - tmp;
            if (overlap > 0.) {
                double vel_j[3] = {0., 0., 0.};
                if (!(q & ORC_Q6_WALL_STATIC) && w->u)
                    for (int d = 0; d < 3; ++d) vel_j[d] = w->u[3 * j + d];
                plane_contact(p, i, nij_x, nij_y, nij_z, overlap, w->E[j], w->nu[j], w->G[j], vel_j, swx, swy, swz, fp,
                              dt);
            } else {
                *swx = 0.;
                *swy = 0.;
                *swz = 0.;
            }
        }
    }
}

// ---------------------------------------------------------------------------------
// Triangle-mesh wall (no reference counterpart).  Closest point of a triangle to a point:
// the Voronoi-region method of Ericson, Real-Time Collision Detection (2005), sec. 5.1.5.
// feature: 0 face interior, 1 edge, 2 vertex.
// ---------------------------------------------------------------------------------
static void tri_closest(const double p[3], const double a[3], const double b[3], const double c[3], double out[3],
                        int *feature) {
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
        *feature = 2;
        return;
    }
    double bp[3];
    for (int d = 0; d < 3; ++d) bp[d] = p[d] - b[d];
    const double d3 = ab[0] * bp[0] + ab[1] * bp[1] + ab[2] * bp[2];
    const double d4 = ac[0] * bp[0] + ac[1] * bp[1] + ac[2] * bp[2];
    if (d3 >= 0. && d4 <= d3) {
        for (int d = 0; d < 3; ++d) out[d] = b[d];
        *feature = 2;
        return;
    }
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0. && d1 >= 0. && d3 <= 0.) {
        const double v = d1 / (d1 - d3);
        for (int d = 0; d < 3; ++d) out[d] = a[d] + v * ab[d];
        *feature = 1;
        return;
    }
    double cp[3];
    for (int d = 0; d < 3; ++d) cp[d] = p[d] - c[d];
    const double d5 = ab[0] * cp[0] + ab[1] * cp[1] + ab[2] * cp[2];
    const double d6 = ac[0] * cp[0] + ac[1] * cp[1] + ac[2] * cp[2];
    if (d6 >= 0. && d5 <= d6) {
        for (int d = 0; d < 3; ++d) out[d] = c[d];
        *feature = 2;
        return;
    }
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0. && d2 >= 0. && d6 <= 0.) {
        const double w = d2 / (d2 - d6);
        for (int d = 0; d < 3; ++d) out[d] = a[d] + w * ac[d];
        *feature = 1;
        return;
    }
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0. && (d4 - d3) >= 0. && (d5 - d6) >= 0.) {
        const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        for (int d = 0; d < 3; ++d) out[d] = b[d] + w * (c[d] - b[d]);
        *feature = 1;
        return;
    }
    const double denom = 1. / (va + vb + vc);
    const double v = vb * denom, w = vc * denom;
    for (int d = 0; d < 3; ++d) out[d] = a[d] + ab[d] * v + ac[d] * w;
    *feature = 0;
}

static void mesh_vertices(const orc_mesh *m, int t, double a[3], double b[3], double c[3]) {
    for (int d = 0; d < 3; ++d) {
        a[d] = m->tri[9 * t + d] + m->D[d];
        b[d] = m->tri[9 * t + 3 + d] + m->D[d];
        c[d] = m->tri[9 * t + 6 + d] + m->D[d];
    }
}

// Contacts of particle i with the mesh, in triangle order:
//  1. every triangle whose closest point lies closer than r_i (0 < d) is a candidate contact;
//  2. face contacts are kept; an edge or vertex contact is dropped when its point lies on a
//     kept contact's point (a shared edge or vertex seen from two triangles) or on a triangle
//     that has a face contact (the particle rests on that face; the edge belongs to it);
//     tolerance 1e-9 r_i;
//  3. tracked slots: the slots whose triangle is still in contact keep their order and
//     history, then the new contacts in triangle order with zero history; slots past
//     max_contacts are not tracked (overflow status);
//  4. each kept contact acts as a plane through its point, normal (x - c)/d, overlap r - d,
//     the mesh's material and velocity (plane_contact), added in triangle order.
extern "C" int orc_force_mesh(orc_particles *p, orc_mesh *m, const orc_force_params *fp, double dt) {
    if (!m || m->nt <= 0) return 0;
    const int mc = m->max_contacts;
    const bool moving = !(fp->quirks & ORC_Q6_WALL_STATIC);
    int status = 0;
#pragma omp parallel for schedule(static) reduction(| : status)
    for (int i = 0; i < p->n; ++i) {
        const double r = p->rad[i];
        const double x[3] = {p->x[3 * i], p->x[3 * i + 1], p->x[3 * i + 2]};
        struct Hit {
            int t, feature;
            double c[3], d, overlap;
        };
        std::vector<Hit> hits;
        for (int t = 0; t < m->nt; ++t) {
            double a[3], b[3], c[3], q[3];
            int f;
            mesh_vertices(m, t, a, b, c);
            tri_closest(x, a, b, c, q, &f);
            const double dx = x[0] - q[0], dy = x[1] - q[1], dz = x[2] - q[2];
            const double d2 = dx * dx + dy * dy + dz * dz;
            if (!(d2 < r * r) || !(d2 > 0.)) continue;
            const double d = std::sqrt(d2);
            const double overlap = r - d;
            if (!(overlap > 0.)) continue;
            hits.push_back({t, f, {q[0], q[1], q[2]}, d, overlap});
        }
        const double eps = 1e-9 * r, eps2 = eps * eps;
        std::vector<char> keep(hits.size(), 0);
        for (size_t h = 0; h < hits.size(); ++h) keep[h] = hits[h].feature == 0;
        for (size_t h = 0; h < hits.size(); ++h) {
            if (hits[h].feature == 0) continue;
            bool drop = false;
            for (size_t k = 0; k < hits.size() && !drop; ++k) {
                if (k == h || !keep[k]) continue;
                const double ex = hits[h].c[0] - hits[k].c[0], ey = hits[h].c[1] - hits[k].c[1],
                             ez = hits[h].c[2] - hits[k].c[2];
                if (ex * ex + ey * ey + ez * ez <= eps2) drop = true;
                if (!drop && hits[k].feature == 0) {
                    double a[3], b[3], c[3], q[3];
                    int f;
                    mesh_vertices(m, hits[k].t, a, b, c);
                    tri_closest(hits[h].c, a, b, c, q, &f);
                    const double fx = hits[h].c[0] - q[0], fy = hits[h].c[1] - q[1], fz = hits[h].c[2] - q[2];
                    if (fx * fx + fy * fy + fz * fz <= eps2) drop = true;
                }
            }
            keep[h] = !drop;
        }
        // tracked slots
        int *tid = m->tid + (long)i * mc;
        double *thx = m->th_x + (long)i * mc, *thy = m->th_y + (long)i * mc, *thz = m->th_z + (long)i * mc;
        const int cnt0 = m->cnt[i];
        std::vector<int> ntid;
        std::vector<double> nhx, nhy, nhz;
        std::vector<char> had;
        for (int s2 = 0; s2 < cnt0; ++s2) {
            bool live = false;
            for (size_t h = 0; h < hits.size(); ++h)
                if (keep[h] && hits[h].t == tid[s2]) live = true;
            if (live) {
                ntid.push_back(tid[s2]);
                nhx.push_back(thx[s2]);
                nhy.push_back(thy[s2]);
                nhz.push_back(thz[s2]);
                had.push_back(1);
            }
        }
        for (size_t h = 0; h < hits.size(); ++h) {
            if (!keep[h]) continue;
            bool found = false;
            for (size_t s2 = 0; s2 < ntid.size(); ++s2)
                if (ntid[s2] == hits[h].t) found = true;
            if (found) continue;
            if ((int)ntid.size() < mc) {
                ntid.push_back(hits[h].t);
                nhx.push_back(0.);
                nhy.push_back(0.);
                nhz.push_back(0.);
                had.push_back(0);
            } else {
                status |= ORC_ERR_CONTACT_OVERFLOW;
            }
        }
        const int cnt1 = (int)ntid.size();
        for (int s2 = 0; s2 < mc; ++s2) {
            tid[s2] = s2 < cnt1 ? ntid[s2] : -1;
            thx[s2] = s2 < cnt1 ? nhx[s2] : 0.;
            thy[s2] = s2 < cnt1 ? nhy[s2] : 0.;
            thz[s2] = s2 < cnt1 ? nhz[s2] : 0.;
        }
        m->cnt[i] = cnt1;
        // forces, in triangle order
        const double vel_j[3] = {moving ? m->u[0] : 0., moving ? m->u[1] : 0., moving ? m->u[2] : 0.};
        for (size_t h = 0; h < hits.size(); ++h) {
            if (!keep[h]) continue;
            int slot = -1;
            for (int s2 = 0; s2 < cnt1; ++s2)
                if (tid[s2] == hits[h].t) slot = s2;
            double dummy[3] = {0., 0., 0.};
            double *sx = slot >= 0 ? thx + slot : dummy, *sy = slot >= 0 ? thy + slot : dummy + 1,
                   *sz = slot >= 0 ? thz + slot : dummy + 2;
            const double d = hits[h].d;
            const double nx = (x[0] - hits[h].c[0]) / d, ny = (x[1] - hits[h].c[1]) / d, nz = (x[2] - hits[h].c[2]) / d;
            plane_contact(p, i, nx, ny, nz, hits[h].overlap, m->E, m->nu, m->G, vel_j, sx, sy, sz, fp, dt);
        }
    }
    return status;
}

// Hook before the interaction forces: external force (tst_01_BDEM:70-117 adds it
// right after the force reset).
extern "C" void orc_apply_ext_force(orc_particles *p, const orc_hooks *h) {
    if (!h || !h->ext_force) return;
    for (int i = 0; i < p->n; ++i)
        for (int d = 0; d < 3; ++d) p->force[3 * i + d] += h->ext_force[3 * i + d];
}

// Hooks after the interaction forces: gravity (no reference counterpart) and the
// boundary-condition zeroing of tst_01_BDEM:19-67.
extern "C" void orc_apply_post_hooks(orc_particles *p, const orc_hooks *h) {
    if (!h) return;
    const bool grav = h->gravity[0] != 0.0 || h->gravity[1] != 0.0 || h->gravity[2] != 0.0;
    for (int i = 0; i < p->n; ++i) {
        if (grav)
            for (int d = 0; d < 3; ++d) p->force[3 * i + d] += p->m[i] * h->gravity[d];
        if (h->fix_flags) {
            if (h->fix_flags[i] & ORC_FIX_FORCE)
                for (int d = 0; d < 3; ++d) p->force[3 * i + d] = 0.;
            if (h->fix_flags[i] & ORC_FIX_TORQUE)
                for (int d = 0; d < 3; ++d) p->torque[3 * i + d] = 0.;
        }
    }
}

// src/CabanaDEM_Solver.hpp:81-94 + src/CabanaDEM_Force.hpp:700-710
extern "C" int orc_step(orc_particles *p, const orc_walls *w, const orc_force_params *fp, const orc_hooks *h,
                        orc_nlist *nl, double dt, double delta, double skin) {
    orc_stage1(p, dt);
    orc_stage2(p, dt);
    if (w && w->n > 0 && !(fp->quirks & ORC_Q6_WALL_STATIC)) orc_stage2_walls(w, dt);
    if (h && h->mesh && !(fp->quirks & ORC_Q6_WALL_STATIC))
        for (int d = 0; d < 3; ++d) h->mesh->D[d] += dt * h->mesh->u[d];
    orc_nlist_build(nl, p, delta, skin);
    orc_zero_force(p);
    orc_apply_ext_force(p, h);
    orc_update_tangential_contacts(p);
    int st = orc_force_pp(p, nl, fp, dt);
    if (w && w->n > 0) orc_force_wall(p, w, fp, dt);
    if (h && h->mesh) st |= orc_force_mesh(p, h->mesh, fp, dt);
    orc_apply_post_hooks(p, h);
    orc_stage3(p, dt);
    return st;
}

extern "C" int orc_run(orc_particles *p, const orc_walls *w, const orc_force_params *fp, const orc_hooks *h,
                       double dt, int nsteps, double delta, double skin) {
    orc_nlist nl;
    int st = 0;
    for (int s = 0; s < nsteps; ++s) st |= orc_step(p, w, fp, h, &nl, dt, delta, skin);
    return st;
}

extern "C" double orc_kinetic_energy(const orc_particles *p) {
    double e = 0.0;
    for (int i = 0; i < p->n; ++i) {
        const double *u = p->u + 3 * i, *w = p->omega + 3 * i;
        e += 0.5 * p->m[i] * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]) +
             0.5 * p->I[i] * (w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    }
    return e;
}

// Hertz elastic energy (no reference counterpart: the reference has no reductions).  The
// normal law fn = kn * overlap^1.5 with kn = 4/3 E_eff sqrt(R_eff) (Force.hpp:196-203 for a
// pair, :561-566 for a wall) is the derivative of kn * 2/5 * overlap^2.5, summed over every
// overlapping pair (each pair once, by brute force over all j > i, independent of any
// neighbour list) and over every particle-wall overlap.  out[0]: pairs, out[1]: walls.
extern "C" void orc_elastic_energy(const orc_particles *p, const orc_walls *w, double *out) {
    double epp = 0.0, epw = 0.0;
    for (int i = 0; i < p->n; ++i) {
        const double *xi = p->x + 3 * i;
        for (int j = i + 1; j < p->n; ++j) {
            const double *xj = p->x + 3 * j;
            const double dx = xi[0] - xj[0], dy = xi[1] - xj[1], dz = xi[2] - xj[2];
            const double overlap = p->rad[i] + p->rad[j] - std::sqrt(dx * dx + dy * dy + dz * dz);
            if (overlap <= 0.) continue;
            const double E_eff = 1. / ((1. - p->nu[i] * p->nu[i]) / p->E[i] + (1. - p->nu[j] * p->nu[j]) / p->E[j]);
            const double R_eff = 1. / (1. / p->rad[i] + 1. / p->rad[j]);
            const double kn = 4. / 3. * E_eff * std::sqrt(R_eff);
            epp += 0.4 * kn * overlap * overlap * std::sqrt(overlap);
        }
        if (!w) continue;
        for (int k = 0; k < w->n; ++k) {
            const double *wx = w->x + 3 * k, *wn = w->normal + 3 * k;
            const double d = (xi[0] - wx[0]) * wn[0] + (xi[1] - wx[1]) * wn[1] + (xi[2] - wx[2]) * wn[2];
            const double overlap = p->rad[i] - d;
            if (overlap <= 0.) continue;
            const double E_eff = 1. / ((1. - p->nu[i] * p->nu[i]) / p->E[i] + (1. - w->nu[k] * w->nu[k]) / w->E[k]);
            const double kn = 4. / 3. * E_eff * std::sqrt(p->rad[i]);
            epw += 0.4 * kn * overlap * overlap * std::sqrt(overlap);
        }
    }
    out[0] = epp;
    out[1] = epw;
}

// ---------------------------------------------------------------------------------
// Bonded DEM.
// ---------------------------------------------------------------------------------

// src/CabanaBondedDEM_Particles.hpp:118-137 (bond every neighbour with rij < factor *
// rad(i); the reference hard-codes factor 3 at :130 and searches within 4*rad(0)).
extern "C" int orc_setup_bonds(orc_bonds *b, const orc_particles *p, double factor, double search_cutoff) {
    double rmax = 0.0;
    for (int i = 0; i < p->n; ++i) rmax = std::max(rmax, p->rad[i]);
    if (search_cutoff <= 0.0) search_cutoff = factor * rmax;
    orc_nlist nl;
    orc_nlist_build(&nl, p, search_cutoff, 0.0);
    int status = 0;
    const int mb = b->max_bonds;
    for (int i = 0; i < p->n; ++i) {
        for (int s = nl.offsets[i]; s < nl.offsets[i + 1]; ++s) {
            const int j = nl.idx[s];
            double pos_ij[3] = {p->x[3 * i + 0] - p->x[3 * j + 0], p->x[3 * i + 1] - p->x[3 * j + 1],
                                p->x[3 * i + 2] - p->x[3 * j + 2]};
            double r2ij = pos_ij[0] * pos_ij[0] + pos_ij[1] * pos_ij[1] + pos_ij[2] * pos_ij[2];
            double rij = std::sqrt(r2ij);
            double bond_cond = factor * p->rad[i];
            if (rij < bond_cond) {
                if (b->count[i] >= mb) {
                    status |= ORC_ERR_BOND_OVERFLOW;
                    continue;
                }
                b->idx[(long)i * mb + b->count[i]] = j;
                b->init_len[(long)i * mb + b->count[i]] = rij;
                b->count[i] += 1;
            }
        }
    }
    return status;
}

// src/CabanaBondedDEM_Force.hpp:86-341
extern "C" int orc_bonded_force(orc_particles *p, orc_bonds *b, const orc_bond_params *bp, double dt) {
    const unsigned q = bp->quirks;
    const int mb = b->max_bonds;
    int status = 0;
#pragma omp parallel for schedule(static) reduction(| : status)
    for (int i = 0; i < p->n; ++i) {
        const double *x = p->x, *u = p->u, *omega = p->omega, *rad = p->rad;
        const int no_bonds_i = b->count[i];
        for (int k = 0; k < no_bonds_i; k++) {
            const long slot = (long)i * mb + k;
            const int j = b->idx[slot];
            if (j < 0 || b->broken[slot]) continue;
            long hs = slot;  // history slot
            if (q & ORC_BQ10_INDEX_BY_J) {
                if (j >= mb) {
                    status |= ORC_ERR_BOND_OVERFLOW;
                    continue;
                }
                hs = (long)i * mb + j;
            }
            double pos_ij[3] = {x[3 * i + 0] - x[3 * j + 0], x[3 * i + 1] - x[3 * j + 1], x[3 * i + 2] - x[3 * j + 2]};
            double r2ij = pos_ij[0] * pos_ij[0] + pos_ij[1] * pos_ij[1] + pos_ij[2] * pos_ij[2];
            double rij = std::sqrt(r2ij);
            const double L0 = b->init_len[hs];
            if (bp->break_strain > 0.0) {
                // bond breakage (no reference counterpart): FP64 strain against rest length
                double strain = (rij - L0) / L0;
                if (strain > bp->break_strain) {
                    b->broken[slot] = 1;
                    continue;
                }
            }
            double g_c = rij - rad[i] - rad[j];
            double a_i = rad[i] + g_c / 2.;
            double a_j = rad[j] + g_c / 2.;
            double normal[3] = {pos_ij[0] / rij, pos_ij[1] / rij, pos_ij[2] / rij};
            double vel_i[3], vel_j[3], vrel[3], vrel_n[3], vrel_t[3];
            vel_i[0] = u[3 * i + 0] + (omega[3 * i + 1] * normal[2] - omega[3 * i + 2] * normal[1]) * a_i;
            vel_i[1] = u[3 * i + 1] + (omega[3 * i + 2] * normal[0] - omega[3 * i + 0] * normal[2]) * a_i;
            vel_i[2] = u[3 * i + 2] + (omega[3 * i + 0] * normal[1] - omega[3 * i + 1] * normal[0]) * a_i;
            const double uj1 = (q & ORC_BQ1_VELJ_USES_UI) ? u[3 * i + 1] : u[3 * j + 1];
            const double uj2 = (q & ORC_BQ1_VELJ_USES_UI) ? u[3 * i + 2] : u[3 * j + 2];
            vel_j[0] = u[3 * j + 0] + (-omega[3 * j + 1] * normal[2] + omega[3 * j + 2] * normal[1]) * a_j;
            vel_j[1] = uj1 + (-omega[3 * j + 2] * normal[0] + omega[3 * j + 0] * normal[2]) * a_j;
            vel_j[2] = uj2 + (-omega[3 * j + 0] * normal[1] + omega[3 * j + 1] * normal[0]) * a_j;
            vrel[0] = vel_i[0] - vel_j[0];
            vrel[1] = vel_i[1] - vel_j[1];
            vrel[2] = vel_i[2] - vel_j[2];
            double vdp = vrel[0] * normal[0] + vrel[1] * normal[1] + vrel[2] * normal[2];
            vrel_n[0] = vdp * normal[0];
            vrel_n[1] = vdp * normal[1];
            vrel_n[2] = vdp * normal[2];
            vrel_t[0] = vrel[0] - vrel_n[0];
            vrel_t[1] = vrel[1] - vrel_n[1];
            vrel_t[2] = vrel[2] - vrel_n[2];
            double wr[3] = {omega[3 * i + 0] - omega[3 * j + 0], omega[3 * i + 1] - omega[3 * j + 1],
                            omega[3 * i + 2] - omega[3 * j + 2]};
            double wdp = wr[0] * normal[0] + wr[1] * normal[1] + wr[2] * normal[2];
            double wn[3] = {wdp * normal[0], wdp * normal[1], wdp * normal[2]};
            double wt[3] = {wr[0] - wn[0], wr[1] - wn[1], wr[2] - wn[2]};
            double rad_sum = rad[i] + rad[j];
            double beta_bond = bp->beta;
            double bond_radius_factor = bp->radius_factor;
            double bond_rad = std::min(rad[i], rad[j]) * bond_radius_factor;
            const double b2 = bp->pow_mode == ORC_POW_SQRT ? bond_rad * bond_rad : std::pow(bond_rad, 2.);
            const double b4 = bp->pow_mode == ORC_POW_SQRT ? (bond_rad * bond_rad) * (bond_rad * bond_rad)
                                                           : std::pow(bond_rad, 4.);
            double A_bond = M_PI * b2;
            double I_bond = M_PI * b4 / 4.0;
            double I_p_bond = I_bond * 2.0;
            double k_n_bond, k_t_bond, k_tor_bond, k_ben_bond;
            if (q & ORC_BQ11_HARDCODED_K) {
                k_n_bond = p->E[i] * A_bond / rad_sum;
                k_t_bond = p->G[i] * A_bond / rad_sum;
                k_tor_bond = p->G[i] * I_p_bond / rad_sum;
                k_ben_bond = p->E[i] * I_bond / rad_sum;
            } else {
                k_n_bond = bp->kn;
                k_t_bond = bp->kt;
                k_tor_bond = bp->kt * I_p_bond / A_bond;
                k_ben_bond = bp->kn * I_bond / A_bond;
            }
            double fn[3], fn_damped[3];
            double overlap_n = rij - L0;
            fn[0] = -k_n_bond * overlap_n * normal[0];
            fn[1] = -k_n_bond * overlap_n * normal[1];
            fn[2] = -k_n_bond * overlap_n * normal[2];
            double multiplierX = (vrel_n[0] >= 0.0) ? 1.0 : -1.0;
            double multiplierY = (vrel_n[1] >= 0.0) ? 1.0 : -1.0;
            double multiplierZ = (vrel_n[2] >= 0.0) ? 1.0 : -1.0;
            fn_damped[0] = fn[0] + beta_bond * std::fabs(fn[0]) * multiplierX;
            fn_damped[1] = fn[1] + beta_bond * std::fabs(fn[1]) * multiplierY;
            fn_damped[2] = fn[2] + beta_bond * std::fabs(fn[2]) * multiplierZ;
            double ft[3] = {b->ft_x[hs], b->ft_y[hs], b->ft_z[hs]};
            double ft_damped[3];
            double fdp = ft[0] * normal[0] + ft[1] * normal[1] + ft[2] * normal[2];
            double ft_norm[3] = {fdp * normal[0], fdp * normal[1], fdp * normal[2]};
            ft[0] -= ft_norm[0];
            ft[1] -= ft_norm[1];
            ft[2] -= ft_norm[2];
            double tmp = k_t_bond * dt;
            double dft[3] = {-vrel_t[0] * tmp, -vrel_t[1] * tmp, -vrel_t[2] * tmp};
            ft[0] += dft[0];
            ft[1] += dft[1];
            ft[2] += dft[2];
            multiplierX = (vrel_t[0] >= 0.0) ? 1.0 : -1.0;
            multiplierY = (vrel_t[1] >= 0.0) ? 1.0 : -1.0;
            multiplierZ = (vrel_t[2] >= 0.0) ? 1.0 : -1.0;
            ft_damped[0] = ft[0] - beta_bond * std::fabs(ft[0]) * multiplierX;
            ft_damped[1] = ft[1] - beta_bond * std::fabs(ft[1]) * multiplierY;
            ft_damped[2] = ft[2] - beta_bond * std::fabs(ft[2]) * multiplierZ;
            b->ft_x[hs] = ft_damped[0];
            b->ft_y[hs] = ft_damped[1];
            b->ft_z[hs] = ft_damped[2];
            double torq_norm[3] = {b->mn_x[hs], b->mn_y[hs], b->mn_z[hs]};
            double ntorq_damped[3];
            double tdp = torq_norm[0] * normal[0] + torq_norm[1] * normal[1] + torq_norm[2] * normal[2];
            torq_norm[0] = tdp * normal[0];
            torq_norm[1] = tdp * normal[1];
            torq_norm[2] = tdp * normal[2];
            tmp = k_tor_bond * dt;
            double dntorque[3] = {-wn[0] * tmp, -wn[1] * tmp, -wn[2] * tmp};
            torq_norm[0] += dntorque[0];
            torq_norm[1] += dntorque[1];
            torq_norm[2] += dntorque[2];
            multiplierX = (wn[0] >= 0.0) ? 1.0 : -1.0;
            multiplierY = (wn[1] >= 0.0) ? 1.0 : -1.0;
            multiplierZ = (wn[2] >= 0.0) ? 1.0 : -1.0;
            ntorq_damped[0] = torq_norm[0] - beta_bond * std::fabs(torq_norm[0]) * multiplierX;
            ntorq_damped[1] = torq_norm[1] - beta_bond * std::fabs(torq_norm[1]) * multiplierY;
            ntorq_damped[2] = torq_norm[2] - beta_bond * std::fabs(torq_norm[2]) * multiplierZ;
            b->mn_x[hs] = ntorq_damped[0];
            b->mn_y[hs] = ntorq_damped[1];
            b->mn_z[hs] = ntorq_damped[2];
            double torq_tang[3] = {b->mt_x[hs], b->mt_y[hs], b->mt_z[hs]};
            tdp = torq_tang[0] * normal[0] + torq_tang[1] * normal[1] + torq_tang[2] * normal[2];
            torq_tang[0] -= tdp * normal[0];
            torq_tang[1] -= tdp * normal[1];
            torq_tang[2] -= tdp * normal[2];
            tmp = k_ben_bond * dt;
            double dttorque[3] = {-wt[0] * tmp, -wt[1] * tmp, -wt[2] * tmp};
            torq_tang[0] += dttorque[0];
            torq_tang[1] += dttorque[1];
            torq_tang[2] += dttorque[2];
            double ttorq_damped[3];
            multiplierX = (wt[0] >= 0.0) ? 1.0 : -1.0;
            multiplierY = (wt[1] >= 0.0) ? 1.0 : -1.0;
            multiplierZ = (wt[2] >= 0.0) ? 1.0 : -1.0;
            ttorq_damped[0] = torq_tang[0] - beta_bond * std::fabs(torq_tang[0]) * multiplierX;
            ttorq_damped[1] = torq_tang[1] - beta_bond * std::fabs(torq_tang[1]) * multiplierY;
            ttorq_damped[2] = torq_tang[2] - beta_bond * std::fabs(torq_tang[2]) * multiplierZ;
            b->mt_x[hs] = ttorq_damped[0];
            b->mt_y[hs] = ttorq_damped[1];
            b->mt_z[hs] = ttorq_damped[2];
            double tor[3] = {0.0, 0.0, 0.0};
            double cri = rij * 1. / rad[i] * 1. / (rad[i] + rad[j]);
            p->force[3 * i + 0] += fn_damped[0] + ft_damped[0];
            p->force[3 * i + 1] += fn_damped[1] + ft_damped[1];
            p->force[3 * i + 2] += fn_damped[2] + ft_damped[2];
            p->torque[3 * i + 0] += ntorq_damped[0] + ttorq_damped[0] - cri * tor[0];
            p->torque[3 * i + 1] += ntorq_damped[1] + ttorq_damped[1] - cri * tor[1];
            p->torque[3 * i + 2] += ntorq_damped[2] + ttorq_damped[2] - cri * tor[2];
        }
    }
    return status;
}

// tst_01_BDEM_two_particles_tensile_3D.cpp:295-306
extern "C" int orc_bonded_step(orc_particles *p, orc_bonds *b, const orc_bond_params *bp, const orc_hooks *h,
                               double dt) {
    orc_stage1(p, dt);
    orc_stage2(p, dt);
    orc_zero_force(p);
    orc_apply_ext_force(p, h);
    int st = orc_bonded_force(p, b, bp, dt);
    orc_apply_post_hooks(p, h);
    orc_stage3(p, dt);
    return st;
}

extern "C" long orc_bonds_broken_total(const orc_bonds *b) {
    long c = 0;
    for (long s = 0; s < (long)b->n * b->max_bonds; ++s) c += b->broken[s] ? 1 : 0;
    return c;
}
