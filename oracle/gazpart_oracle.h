/*
 * gazpart_oracle.h -- CPU restatement of GAZPART's frozen-flow ellipsoidal-particle
 * step (ADV_PARTICLE_ELLP followed by COLLISION), FP64, serial per particle.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the oracle for the CUDA path and the
 * timed CPU baseline; it is never linked into, called by, or shipped with the product.
 *
 * PARITY UNPINNED against the reference itself: the reference is Fortran (no Fortran
 * compiler exists on these machines) and ships no tests, golden vectors or fixtures.
 * The restatement is pinned instead by analytic known-answer tests (cubic
 * reproduction of the Lagrange stencil, exact rotations, sphere contact depth,
 * impulse energy conservation, half-stencil coverage, brute-force pair sets) and by a
 * cross-check of the Levenberg-Marquardt solve against scipy's MINPACK lmder.
 *
 * Every routine follows the reference file and lines given in its comment
 * (paths relative to the reference's source/ directory).  Arithmetic follows the
 * reference's evaluation order; build with -ffp-contract=off -fno-fast-math (the
 * reference is built by gfortran -O3 without -march, so without FMA contraction).
 *
 * Generalisation: the reference keeps shape and density per class/sub-class
 * (EMAJ_PART(IG,IDP), APR_PART(IG), RHOP(IG,IDP), IPXX..(IG,IDP)); here every
 * particle carries its own copy of those values, with identical per-particle
 * arithmetic.  A one-class run is the reference's case exactly.
 */
#ifndef GAZPART_ORACLE_H
#define GAZPART_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Mesh and physics inputs that the reference reads from its modules
 * (mod_param_phys.f90:14-113, mod_dns_dim.f90:57,136, init_run.f90:123-135,
 * meshing.f90:43-45).  One record per ensemble. */
typedef struct {
    int32_t nx, ny, nz;          /* NX, NY, NZ */
    double lx, ly, lz;           /* LXMAX, LYMAX, LZMAX */
    double dx, dy, dz;           /* DX = LXMAX/real(NX-1)  (meshing.f90:43-45) */
    double visc, rhof, ppi;      /* VISC, RHOF, PPI = 4*atan(1) */
    double dtime;                /* DTIME */
    double gravity;              /* GRAVITY(IG), added to the z force */
    double ecp, mup;             /* ECP(IG), MUP(IG): particle-particle */
    double ecw, muw;             /* ECW, MUW: particle-wall */
    int32_t periodicity;         /* PERIODICITY (x wrap of positions/boxes) */
    int32_t wall_boundary;       /* WALL_BOUNDARY (x wrap of the stencil) */
    int32_t frozen_flow;         /* FROZEN_FLOW (3: channel, y and z wrap only) */
} orc_setup;

/* Per-particle shape/density (reference: per class; see header comment). */
typedef struct {
    const double *emaj;   /* EMAJ_PART: semi-axis along the symmetry axis */
    const double *apr;    /* APR_PART: aspect ratio; other semi-axes = emaj/apr */
    const double *rhop;   /* RHOP */
    const double *ipxx, *ipyy, *ipzz;  /* IPXX..IPZZ per unit mass */
} orc_props;

/* Particle state, structure of arrays (PARTTYPE hot fields,
 * mod_particle_parallel.f90:17-87). */
typedef struct {
    int64_t n;
    double *x, *y, *z;
    double *u, *v, *w;
    double *qa, *qb, *qc, *qd;
    double *ox, *oy, *oz;
    double *ufap, *vfap, *wfap;     /* fluid velocity at particle (output) */
    double *vortx, *vorty, *vortz;  /* fluid vorticity at particle (output) */
} orc_state;

/* Collision box grid (collision_initiation.f90:44-103, mod_collision.f90:19-38). */
typedef struct {
    int32_t nxbox, nybox, nzbox, nbox;
    double dxbox, dybox, dzbox;
    double xminbox, yminbox, zminbox;
    double xmaxbox, ymaxbox, zmaxbox;
    double delta_coll;
} orc_boxgrid;

/* Status codes shared with the CUDA library's error enum. */
enum {
    ORC_OK = 0,
    ORC_ENAN_FORCE = 1,
    ORC_ENAN_TORQUE = 2,
    ORC_EENERGY = 3,
    ORC_ESINGULAR = 4,
    ORC_EOUT_OF_GRID = 6,
    ORC_EBADARG = 9
};

/* ---- small-kernel restatements (exported for unit tests) ---- */
void orc_transform_vec(double v[3], const double q[4]);            /* transform_basis.f90:44-77 */
void orc_transform_tensor(double a[9], const double q[4]);         /* transform_basis.f90:44-82 (a column-major 3x3) */
void orc_mult_quat(const double x[4], const double y[4], double r[4]); /* mod_quaternion.f90:136-145 */
int  orc_invert3(const double m[9], double inv[9]);                 /* invert_ndim3_matrix.f90:1-39 */
void orc_quaternion_integration(double q[4], double ox, double oy, double oz, double dt); /* adv_quaternion.f90:1-117 */
void orc_euler_integration(double ipxx, double ipyy, double ipzz, double dt,
                           double *ox, double *oy, double *oz);     /* adv_angular_velocity.f90:113-149 */

int orc_fluid_force(const orc_setup *s, double emaj, double apr, double rhop,
                    double up, double vp, double wp, double uf, double vf, double wf,
                    const double q[4], double fdrag[3], double flift[3]);   /* fluid_force_ellipsoid.f90 */
int orc_fluid_torque(const orc_setup *s, double emaj, double apr, double rhop,
                     double up_n, double vp_n, double wp_n,     /* PART(I)%UP..  (Q3) */
                     double uf, double vf, double wf,           /* PART(I)%UFAP.. */
                     double vortx, double vorty, double vortz,  /* PART(I)%VORTXAP.. */
                     double ox, double oy, double oz, const double q[4],
                     double tpitch[3], double trot[3]);          /* fluid_torque_ellipsoid.f90 */

void orc_interp_lag3(const orc_setup *s, const double *uain, int64_t nint,
                     const double *xint, const double *yint, const double *zint,
                     double *uint);                               /* interp_lag3.f90:11-298 */
void orc_frozen_interp_lag3(const double *xain, const double *yain, const double *zain,
                            int32_t nx, int32_t ny, int32_t nz, const double *uain,
                            int64_t nint, const double *xint, const double *yint,
                            const double *zint, double *uint);  /* frozen_interp_lag3.f90:11-274 */

int orc_wall_boundary_condition(const orc_setup *s, double emaj, double apr,
                                double xp, double yp, double zp, const double q[4],
                                double wall_normal[3], double impact_arm[3],
                                double *delta_x, int32_t *is_intersect); /* ellipsoid_wall_boundary_new.f90 */
int orc_wall_rebound(const orc_setup *s, double ipxx, double ipyy, double ipzz,
                     double *u, double *v, double *w, double *ox, double *oy, double *oz,
                     const double q[4], const double r_impact[3], const double norm_w[3]); /* wall_ellipsoid_rebound.f90 */

/* One ADV_PARTICLE_ELLP step (interpolation of the six fields, the RK2 predictor/
 * corrector with wall handling, and BOUNDARY_PARTICLE's periodic wrap).
 * fields: six arrays u,v,w,vortx,vorty,vortz each (NX, NY+4, NZ+4), x fastest.
 * Returns ORC_OK or the first error code; *err_id receives the particle index. */
int orc_adv_particle_ellp(const orc_setup *s, const orc_props *p,
                          const double *const fields[6], orc_state *st,
                          int32_t nthreads, int64_t *err_id);

/* ---- collisions ---- */
void orc_collision_initiation(const orc_setup *s, double max_emaj, orc_boxgrid *g); /* collision_initiation.f90:44-103 */
/* con: nbox*27 int32 (1-based box ids, as COLBOX%CON), ncon: nbox int32 */
void orc_box_connectivity(const orc_boxgrid *g, int32_t periodicity,
                          int32_t *ncon, int32_t *con);             /* collision_box_connectivity.f90:42-322 */
/* Box id (1-based IJK) of each particle; returns ORC_EOUT_OF_GRID (first index in
 * *err_id) if a particle falls outside the grid (collision_detection_connectivity.f90:74-89). */
int orc_box_index(const orc_boxgrid *g, int64_t n, const double *x, const double *y,
                  const double *z, int32_t *ijk, int64_t *err_id);
/* HOME/NEAR candidate list in the reference's order (collision_detection_connectivity.f90:56-210).
 * Indices are 0-based.  Call with home==NULL to count only.  Returns the count, or -1. */
int64_t orc_detect_pairs(const orc_boxgrid *g, const int32_t *ncon, const int32_t *con,
                         int64_t n, const double *x, const double *y, const double *z,
                         int64_t cap, int32_t *home, int32_t *near);

/* Contact test of two ellipsoids (ellipsoid_contact_detection.f90:1-187).
 * x_out (optional) receives the final LM angles, info_out the LM info code. */
int32_t orc_contact_detection(double emaj1, double apr1, double emaj2, double apr2,
                              const double b1[3], const double q1[4],
                              const double b2[3], const double q2[4],
                              double ept1[3], double ept2[3], double cnormal[3],
                              double x_out[2], int32_t *info_out, int32_t *nfev_out);
/* Margin function (mod_particle_parallel.f90:145-201) */
double orc_fmargin(double emaj, double apr, const double point[3], const double center[3],
                   const double q[4]);

/* Impulse response (collision_response.f90:1-437).  Inertia of particle 1 for both
 * bodies (reference behaviour).  u1/o1 etc are in/out; returns ORC_EENERGY on the
 * reference's energy-balance failure. */
int orc_collision_response(const orc_setup *s, double ipxx, double ipyy, double ipzz,
                           double u1[3], double o1[3], const double q1[4],
                           double u2[3], double o2[3], const double q2[4],
                           const double r1[3], const double r2[3], const double n[3]);

/* COLLISION for one ensemble (collision.f90:53-174 with NPROC=1, then
 * collision_interaction.f90:190-419).  prefilter!=0 skips candidate pairs whose
 * bounding spheres (radius max(emaj, emaj/apr)) are more than (1+1e-9) apart, which
 * cannot change the result (a contact needs each contact point inside the other body).
 * Outputs (optional, may be NULL): the ordered list of pairs that collided
 * (coll_home/coll_near, 0-based, in acceptance order) and their count.
 * nthreads>1 evaluates candidate contacts in parallel; acceptance stays serial. */
int orc_collision(const orc_setup *s, const orc_props *p, const orc_boxgrid *g,
                  const int32_t *ncon, const int32_t *con, orc_state *st,
                  int32_t prefilter, int32_t nthreads,
                  int64_t coll_cap, int32_t *coll_home, int32_t *coll_near,
                  int64_t *n_coll, int64_t *n_candidates, int64_t *n_contacts,
                  int64_t *err_id);

/* COLLISION with the statistics of COLLISION_INTERACTION (collision_interaction.f90:
 * 171,330-345,397-398,429-430), serial walk: colstat (ngroups*ngroups*8, by (IDP of
 * HOME, IDP of NEAR)) receives for the pairs found in contact while both particles are
 * uncoloured [0] their number, [1] the collisions, [2] 2[1]/DTIME, [3] sum of the overlap
 * depth |EPT1-EPT2|, [4] [3]/[0], [5] sum of NVREL, [6] sum of |v_rel|, [7] sum of the
 * collision angle.  group: IDP per particle (1..ngroups) or NULL. */
int orc_collision_stats(const orc_setup *s, const orc_props *p, const orc_boxgrid *g,
                        const int32_t *ncon, const int32_t *con, orc_state *st, int32_t prefilter,
                        const int32_t *group, int32_t ngroups, double *colstat, int64_t *n_coll,
                        int64_t *err_id);

/* STAT_PARTFLUID (stat_partfluid.f90:122-299): the 35 per-particle quantities and the
 * count, and their sums per polydisperse index (st->ufap.. are the fluid values the
 * last step interpolated at each particle). */
void orc_stat_partfluid_particle(const orc_setup *s, double emaj, double apr, double rhop, const double u[3],
                                 const double om[3], const double q[4], const double uf[3], const double wv[3],
                                 double v[36]);
void orc_stat_partfluid(const orc_setup *s, const orc_props *p, const orc_state *st, const int32_t *group,
                        int32_t ngroups, double *out);

/* Evaluate one candidate pair exactly as collision_interaction.f90:216-348 does
 * (minimum image, contact, contact-point velocities, NVREL).  Returns 1 if the
 * pair would collide (flag && NVREL<ZERO), 0 otherwise. */
int32_t orc_pair_eval(const orc_setup *s, const orc_props *p, const orc_state *st,
                      int64_t i1, int64_t i2, double ept1[3], double ept2[3],
                      double cn[3], double rx1[3], double rx2[3], int32_t *flag_out);

/* ---- MINPACK-style helpers, exported for the scipy cross-check ---- */
double orc_enorm(int32_t n, const double *x);   /* minpack_reduc.f90:180-232 */
/* residual (fcn iflag=1), Jacobian (fcn iflag=2, column-major 3x2) and the bare LM
 * solve of the contact problem (ellipsoid_contact_detection.f90:92,193-334) */
void orc_contact_residual(double emaj1, double apr1, double emaj2, double apr2,
                          const double b1[3], const double q1[4], const double b2[3],
                          const double q2[4], const double x[2], double fvec[3]);
void orc_contact_jacobian(double emaj1, double apr1, double emaj2, double apr2,
                          const double b1[3], const double q1[4], const double b2[3],
                          const double q2[4], const double x[2], double fjac[6]);
int32_t orc_contact_lm(double emaj1, double apr1, double emaj2, double apr2,
                       const double b1[3], const double q1[4], const double b2[3],
                       const double q2[4], double x[2], double tol, int32_t *nfev);

#ifdef __cplusplus
}
#endif
#endif
