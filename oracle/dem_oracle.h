/*
 * dem_oracle.h -- CPU oracle for the CabanaDEM contact step (TEST INFRASTRUCTURE).
 *
 * This library is the checker, never the product: only tests/, the smoke check
 * and the CPU-baseline leg of bench.py load it.  It restates, line by line and in
 * FP64, the reference's own double-precision path:
 *
 *   src/CabanaDEM_Integrator.hpp:31-102   stage1 / stage2 / stage3
 *   src/CabanaDEM_Force.hpp:40-47         force/torque zeroing
 *   src/CabanaDEM_Force.hpp:344-445       update_tangential_contacts (swap-with-last)
 *   src/CabanaDEM_Force.hpp:50-341        Hertz + Mindlin particle-particle force
 *   src/CabanaDEM_Force.hpp:448-678       particle-infinite-wall force
 *   src/CabanaDEM_Force.hpp:700-710       phase order
 *   src/CabanaDEM_Solver.hpp:79-97        time loop
 *   src/CabanaBondedDEM_Particles.hpp:118-137   setupBonds
 *   src/CabanaBondedDEM_Force.hpp:86-341        computeBondedForce
 *
 * The neighbour list (Cabana VerletList, not vendored) is restated as "every j != i
 * within the cutoff, ascending j".  Each reference quirk is switchable (ORC_Q*).
 * Parallelism is `#pragma omp parallel for` over particles with serial per-particle
 * inner loops, the stand-in for the Kokkos OpenMP backend.
 */
#ifndef DEM_ORACLE_H
#define DEM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Reference behaviours that can be reproduced (bit set) or corrected (bit clear). */
#define ORC_Q1_VELJ_USES_UI   0x01u /* Force.hpp:133-137: vel_j y,z use u(i,.)          */
#define ORC_Q2_ETA_T_ZERO     0x02u /* Force.hpp:224,:618: sqrt(5/6) integer division    */
#define ORC_Q3_NO_PP_TORQUE   0x04u /* Force.hpp:324-326: pp contact adds no torque      */
#define ORC_Q4_UNIT_HISTORY   0x08u /* Force.hpp:310-319: history stored normalised      */
#define ORC_Q5_WALL_FT_TYPO   0x10u /* Force.hpp:624: ft_z*ft_y in |ft|                   */
#define ORC_Q6_WALL_STATIC    0x20u /* Force.hpp:529: vel_j = 0, walls never move          */
#define ORC_REF_COMPAT        0x3Fu

/* pow handling: 0 = libm pow() exactly as the reference; 1 = x*sqrt(x) and sqrt(x)
 * for pow(x,1.5) and pow(x,0.5) (the device kernels' arithmetic). */
#define ORC_POW_LIBM 0
#define ORC_POW_SQRT 1

/* status bits (sticky, OR-ed) */
#define ORC_ERR_CONTACT_OVERFLOW 0x1
#define ORC_ERR_BOND_OVERFLOW    0x2

/* per-particle fix flags (hook after the force pass, tst_01_BDEM:19-67) */
#define ORC_FIX_FORCE  0x1
#define ORC_FIX_TORQUE 0x2

typedef struct orc_particles {
    int n;
    int max_cnts;   /* tangential-history slots per particle (MaxCnts)   */
    int max_walls;  /* wall-history slots per particle (MaxNoWalls)      */
    double *x, *u, *omega, *force, *torque;     /* [n*3] row-major (i,d)  */
    double *m, *rad, *I, *E, *nu, *G;           /* [n]                    */
    int *tng_idx;                               /* [n*max_cnts]           */
    double *tng_ss_x, *tng_ss_y, *tng_ss_z;     /* [n*max_cnts]           */
    int *tng_count;                             /* [n]                    */
    double *tng_sw_x, *tng_sw_y, *tng_sw_z;     /* [n*max_walls]          */
} orc_particles;

typedef struct orc_walls {
    int n;
    double *x;        /* [n*3] point on the plane (advanced in place by moving walls) */
    double *normal;   /* [n*3] unit normal        */
    double *E, *nu, *G;
    double *u;        /* [n*3] velocity, or NULL: used only with ORC_Q6_WALL_STATIC clear */
} orc_walls;

typedef struct orc_force_params {
    double cor_pp, cor_pw, mu_pp, mu_pw;
    unsigned quirks;
    int pow_mode;
} orc_force_params;

/* Triangle-mesh wall (no reference counterpart; the reference has a Python intersection
 * prototype only).  Vertices [nt][3][3] at translation D (advanced by dt * u in stage2 when
 * ORC_Q6_WALL_STATIC is clear).  Per particle: up to max_contacts tracked triangle contacts. */
typedef struct orc_mesh {
    int nt;
    const double *tri;               /* [nt*9]: a, b, c                                  */
    double E, nu, G;
    double u[3];                     /* translation velocity                             */
    double D[3];                     /* accumulated translation (advanced in place)      */
    int max_contacts;
    int *tid;                        /* [n*max_contacts] triangle of each tracked slot   */
    double *th_x, *th_y, *th_z;      /* [n*max_contacts] tangential history              */
    int *cnt;                        /* [n] tracked triangle contacts                    */
} orc_mesh;

/* Hooks applied in the position of tst_01_BDEM's applyTensileForce /
 * applyBoundaryConditions: ext_force (may be NULL) is added before the interaction
 * forces, gravity * m after them, then fix flags zero F and/or tau. */
typedef struct orc_hooks {
    double gravity[3];
    const double *ext_force;          /* [n*3] or NULL */
    const unsigned char *fix_flags;   /* [n] or NULL   */
    orc_mesh *mesh;                   /* triangle-mesh wall or NULL (after the plane walls) */
} orc_hooks;

typedef struct orc_nlist orc_nlist;

orc_nlist *orc_nlist_create(void);
void orc_nlist_destroy(orc_nlist *nl);
/* cutoff(i,j) = delta if delta > 0, else rad_i + rad_j + skin.  Pair kept when
 * |x_i - x_j|^2 <= cutoff^2.  Lists are in ascending j. */
int orc_nlist_build(orc_nlist *nl, const orc_particles *p, double delta, double skin);
long orc_nlist_total(const orc_nlist *nl);
void orc_nlist_copy(const orc_nlist *nl, int *offsets /*n+1*/, int *idx /*total*/);

void orc_stage1(orc_particles *p, double dt);
void orc_stage2(orc_particles *p, double dt);
/* Kinematic walls (no reference counterpart): x_w += dt * u_w, with the particles' drift. */
void orc_stage2_walls(const orc_walls *w, double dt);
void orc_stage3(orc_particles *p, double dt);
void orc_zero_force(orc_particles *p);
void orc_update_tangential_contacts(orc_particles *p);
int  orc_force_pp(orc_particles *p, const orc_nlist *nl, const orc_force_params *fp, double dt);
void orc_force_wall(orc_particles *p, const orc_walls *w, const orc_force_params *fp, double dt);
void orc_apply_ext_force(orc_particles *p, const orc_hooks *h);
/* Contacts with the mesh, after the plane walls; returns ORC_ERR_CONTACT_OVERFLOW when a
 * particle has more than max_contacts triangle contacts (the rest are not tracked). */
int  orc_force_mesh(orc_particles *p, orc_mesh *m, const orc_force_params *fp, double dt);
void orc_apply_post_hooks(orc_particles *p, const orc_hooks *h);

/* One reference time step (Solver.hpp:81-94) with the neighbour list rebuilt from the
 * drifted positions.  Returns status bits. */
int orc_step(orc_particles *p, const orc_walls *w, const orc_force_params *fp,
             const orc_hooks *h, orc_nlist *nl, double dt, double delta, double skin);
/* nsteps calls of orc_step. */
int orc_run(orc_particles *p, const orc_walls *w, const orc_force_params *fp,
            const orc_hooks *h, double dt, int nsteps, double delta, double skin);

/* Kinetic (translational + rotational) energy, sequential sum over i. */
double orc_kinetic_energy(const orc_particles *p);
/* Hertz elastic energy 2/5 kn overlap^2.5 of every overlapping pair (each pair once, all
 * pairs by brute force) in out[0] and of every particle-wall overlap in out[1]. */
void orc_elastic_energy(const orc_particles *p, const orc_walls *w, double *out);

/* ---------------- bonded DEM (CabanaBondedDEM_*) ---------------- */
typedef struct orc_bonds {
    int n, max_bonds;
    int *idx;            /* [n*max_bonds] partner, -1 empty              */
    double *init_len;    /* [n*max_bonds]                                */
    int *count;          /* [n]                                          */
    double *fn_x, *fn_y, *fn_z, *ft_x, *ft_y, *ft_z;   /* [n*max_bonds]   */
    double *mn_x, *mn_y, *mn_z, *mt_x, *mt_y, *mt_z;   /* [n*max_bonds]   */
    unsigned char *broken;                              /* [n*max_bonds]   */
} orc_bonds;

#define ORC_BQ10_INDEX_BY_J    0x01u /* BondedDEM_Force.hpp:207,:231-322 history(i, j) */
#define ORC_BQ11_HARDCODED_K   0x02u /* BondedDEM_Force.hpp:186-198 k from E,G,A        */
#define ORC_BQ1_VELJ_USES_UI   0x04u /* BondedDEM_Force.hpp:142-146                     */
#define ORC_BOND_REF_COMPAT    0x07u

typedef struct orc_bond_params {
    unsigned quirks;
    double beta;            /* sign-damping factor (reference: 0.1)            */
    double radius_factor;   /* bond radius = min(r_i,r_j)*factor (ref: 1)       */
    double kn, kt;          /* explicit stiffnesses when BQ11 is clear          */
    double break_strain;    /* > 0: bond breaks when (rij-L0)/L0 > break_strain */
    int pow_mode;           /* ORC_POW_LIBM: pow(b,2.), pow(b,4.) as the reference; ORC_POW_SQRT: b*b */
} orc_bond_params;

/* setupBonds: bond every j != i with rij < factor * rad(i) among the neighbour
 * candidates within `search_cutoff`, in ascending j. */
int orc_setup_bonds(orc_bonds *b, const orc_particles *p, double factor, double search_cutoff);
/* computeBondedForce (accumulates into force/torque). Returns status bits. */
int orc_bonded_force(orc_particles *p, orc_bonds *b, const orc_bond_params *bp, double dt);
/* one bonded step in the order of tst_01_BDEM:295-306 */
int orc_bonded_step(orc_particles *p, orc_bonds *b, const orc_bond_params *bp,
                    const orc_hooks *h, double dt);
long orc_bonds_broken_total(const orc_bonds *b);

#ifdef __cplusplus
}
#endif
#endif
