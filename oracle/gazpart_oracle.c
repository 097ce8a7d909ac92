/*
 * gazpart_oracle.c -- CPU restatement of GAZPART's frozen-flow ellipsoidal-particle
 * step.  TEST INFRASTRUCTURE ONLY (oracle and timed CPU baseline); see the header.
 *
 * PARITY UNPINNED against the reference binary (no Fortran compiler, no reference
 * tests or fixtures); pinned by analytic known-answer tests and a scipy MINPACK
 * cross-check of the Levenberg-Marquardt solve.
 *
 * File:line citations are relative to the reference's source/ directory.
 * Matrices are 3x3 column-major (Fortran layout): a[i + 3*j] = A(i+1, j+1).
 */
#include "gazpart_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ZERO_REF 1.0e-33   /* ZERO (mod_dns_dim.f90:136) */
#define M3(a, i, j) ((a)[(i) + 3 * (j)])

/* ------------------------------------------------------------------------- */
/* Rotation helpers                                                          */
/* ------------------------------------------------------------------------- */

/* R(q) exactly as transform_basis.f90:44-54 (and calculate_ellipsoid_matrix.f90:54-64,
 * mod_particle_parallel.f90:176-186, which use the same expressions). */
static void rotmat(const double q[4], double r[9]) {
    const double q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3];
    M3(r, 0, 0) = 1.0 - 2.0 * (q2 * q2 + q3 * q3);
    M3(r, 0, 1) = 2.0 * (q1 * q2 - q0 * q3);
    M3(r, 0, 2) = 2.0 * (q1 * q3 + q0 * q2);
    M3(r, 1, 0) = 2.0 * (q1 * q2 + q0 * q3);
    M3(r, 1, 1) = 1.0 - 2.0 * (q1 * q1 + q3 * q3);
    M3(r, 1, 2) = 2.0 * (q2 * q3 - q0 * q1);
    M3(r, 2, 0) = 2.0 * (q1 * q3 - q0 * q2);
    M3(r, 2, 1) = 2.0 * (q2 * q3 + q0 * q1);
    M3(r, 2, 2) = 1.0 - 2.0 * (q1 * q1 + q2 * q2);
}

/* C = A*B for 3x3 (gfortran's inlined matmul: k summed in order 1..3). */
static void matmul33(const double a[9], const double b[9], double c[9]) {
    double t[9];
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i)
            t[i + 3 * j] = M3(a, i, 0) * M3(b, 0, j) + M3(a, i, 1) * M3(b, 1, j) +
                           M3(a, i, 2) * M3(b, 2, j);
    memcpy(c, t, sizeof t);
}

static void matvec3(const double a[9], const double v[3], double out[3]) {
    double t[3];
    for (int i = 0; i < 3; ++i)
        t[i] = M3(a, i, 0) * v[0] + M3(a, i, 1) * v[1] + M3(a, i, 2) * v[2];
    out[0] = t[0]; out[1] = t[1]; out[2] = t[2];
}

static void transpose33(const double a[9], double t[9]) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) M3(t, i, j) = M3(a, j, i);
}

static inline double dot3(const double a[3], const double b[3]) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

static inline void conjq(const double q[4], double c[4]) {
    c[0] = q[0]; c[1] = -q[1]; c[2] = -q[2]; c[3] = -q[3];   /* mod_quaternion.f90:98-107 */
}

/* transform_basis.f90:77 -- vector case A_Tr = R*A_b */
void orc_transform_vec(double v[3], const double q[4]) {
    double r[9];
    rotmat(q, r);
    matvec3(r, v, v);
}

/* transform_basis.f90:82 -- tensor case A_Tr = R*(A_b*R^T) */
void orc_transform_tensor(double a[9], const double q[4]) {
    double r[9], rt[9], t[9];
    rotmat(q, r);
    transpose33(r, rt);
    matmul33(a, rt, t);
    matmul33(r, t, a);
}

/* mod_quaternion.f90:136-145 */
void orc_mult_quat(const double x[4], const double y[4], double r[4]) {
    double a = x[0] * y[0] - x[1] * y[1] - x[2] * y[2] - x[3] * y[3];
    double b = x[0] * y[1] + x[1] * y[0] + x[2] * y[3] - x[3] * y[2];
    double c = x[0] * y[2] - x[1] * y[3] + x[2] * y[0] + x[3] * y[1];
    double d = x[0] * y[3] + x[1] * y[2] - x[2] * y[1] + x[3] * y[0];
    r[0] = a; r[1] = b; r[2] = c; r[3] = d;
}

/* invert_ndim3_matrix.f90:1-39.  Returns ORC_ESINGULAR where the reference stops. */
int orc_invert3(const double m[9], double inv[9]) {
#define M(i, j) M3(m, (i)-1, (j)-1)
    double detinv = 1.0 / (M(1, 1) * M(2, 2) * M(3, 3) - M(1, 1) * M(2, 3) * M(3, 2) -
                           M(1, 2) * M(2, 1) * M(3, 3) + M(1, 2) * M(2, 3) * M(3, 1) +
                           M(1, 3) * M(2, 1) * M(3, 2) - M(1, 3) * M(2, 2) * M(3, 1));
    if (detinv == 0.0) return ORC_ESINGULAR;
    M3(inv, 0, 0) = +detinv * (M(2, 2) * M(3, 3) - M(2, 3) * M(3, 2));
    M3(inv, 1, 0) = -detinv * (M(2, 1) * M(3, 3) - M(2, 3) * M(3, 1));
    M3(inv, 2, 0) = +detinv * (M(2, 1) * M(3, 2) - M(2, 2) * M(3, 1));
    M3(inv, 0, 1) = -detinv * (M(1, 2) * M(3, 3) - M(1, 3) * M(3, 2));
    M3(inv, 1, 1) = +detinv * (M(1, 1) * M(3, 3) - M(1, 3) * M(3, 1));
    M3(inv, 2, 1) = -detinv * (M(1, 1) * M(3, 2) - M(1, 2) * M(3, 1));
    M3(inv, 0, 2) = +detinv * (M(1, 2) * M(2, 3) - M(1, 3) * M(2, 2));
    M3(inv, 1, 2) = -detinv * (M(1, 1) * M(2, 3) - M(1, 3) * M(2, 1));
    M3(inv, 2, 2) = +detinv * (M(1, 1) * M(2, 2) - M(1, 2) * M(2, 1));
#undef M
    return ORC_OK;
}

/* adv_quaternion.f90:39-84 (METHOD=1, direct multiplication; no renormalisation). */
void orc_quaternion_integration(double q[4], double ox, double oy, double oz, double dt) {
    double omg[3] = {ox, oy, oz};
    orc_transform_vec(omg, q);
    double norm_omg = sqrt(omg[0] * omg[0] + omg[1] * omg[1] + omg[2] * omg[2]);
    double map[4];
    if (norm_omg != 0.0) {
        map[0] = cos((norm_omg * dt) / 2.0);
        map[1] = sin((norm_omg * dt) / 2.0) * (omg[0] / norm_omg);
        map[2] = sin((norm_omg * dt) / 2.0) * (omg[1] / norm_omg);
        map[3] = sin((norm_omg * dt) / 2.0) * (omg[2] / norm_omg);
    } else {
        map[0] = 1.0; map[1] = 0.0; map[2] = 0.0; map[3] = 0.0;
    }
    double nq[4];
    orc_mult_quat(map, q, nq);
    q[0] = nq[0]; q[1] = nq[1]; q[2] = nq[2]; q[3] = nq[3];
}

/* adv_angular_velocity.f90:113-149 (METHOD=2, RK4 torque-free Euler equations). */
void orc_euler_integration(double ipxx, double ipyy, double ipzz, double dt,
                           double *ox, double *oy, double *oz) {
    const double w0x = *ox, w0y = *oy, w0z = *oz;
    const double cx = (ipyy - ipzz) / ipxx, cy = (ipzz - ipxx) / ipyy, cz = (ipxx - ipyy) / ipzz;
    double k1x = dt * (w0y * w0z * cx);
    double k1y = dt * (w0z * w0x * cy);
    double k1z = dt * (w0x * w0y * cz);
    double k2x = dt * ((w0y + 0.5 * k1y) * (w0z + 0.5 * k1z) * cx);
    double k2y = dt * ((w0z + 0.5 * k1z) * (w0x + 0.5 * k1x) * cy);
    double k2z = dt * ((w0x + 0.5 * k1x) * (w0y + 0.5 * k1y) * cz);
    double k3x = dt * ((w0y + 0.5 * k2y) * (w0z + 0.5 * k2z) * cx);
    double k3y = dt * ((w0z + 0.5 * k2z) * (w0x + 0.5 * k2x) * cy);
    double k3z = dt * ((w0x + 0.5 * k2x) * (w0y + 0.5 * k2y) * cz);
    double k4x = dt * ((w0y + k3y) * (w0z + k3z) * cx);
    double k4y = dt * ((w0z + k3z) * (w0x + k3x) * cy);
    double k4z = dt * ((w0x + k3x) * (w0y + k3y) * cz);
    *ox = w0x + (k1x + 2.0 * k2x + 2.0 * k3x + k4x) / 6.0;
    *oy = w0y + (k1y + 2.0 * k2y + 2.0 * k3y + k4y) / 6.0;
    *oz = w0z + (k1z + 2.0 * k2z + 2.0 * k3z + k4z) / 6.0;
}

/* ------------------------------------------------------------------------- */
/* Fluid force and torque                                                    */
/* ------------------------------------------------------------------------- */

/* PMASS (fluid_force_ellipsoid.f90:59, fluid_torque_ellipsoid.f90:85) */
static inline double pmass_of(const orc_setup *s, double emaj, double apr, double rhop) {
    return rhop * (4.0 / 3.0) * s->ppi * pow(emaj, 3.0) / (apr * apr);
}

/* fluid_force_ellipsoid.f90:1-161.  Zastawny et al. (2012) drag and lift, per unit
 * mass, computed in the body frame and rotated back to the lab frame.
 * Guard (the reference stops or yields NaN there): a relative velocity of exactly
 * zero gives zero force, and a zero transverse component gives zero transverse lift;
 * both are the limits of the correlations as the speed goes to zero. */
int orc_fluid_force(const orc_setup *s, double emaj, double apr, double rhop,
                    double up, double vp, double wp, double uf, double vf, double wf,
                    const double q[4], double fdrag[3], double flift[3]) {
    const double a0 = 1.95, a1 = 18.12, a2 = 1.023, a3 = 4.26, a4 = 0.384;
    const double a5 = 21.52, a6 = 0.990, a7 = 2.86, a8 = 0.260;
    const double b1 = 0.083, b2 = -0.21, b3 = 1.582, b4 = 0.851, b5 = 1.842;
    const double b6 = -0.802, b7 = -0.006, b8 = 0.874, b9 = 0.009, b10 = 0.570;
    const double pmass = pmass_of(s, emaj, apr, rhop);
    double urel[3] = {uf - up, vf - vp, wf - wp};
    double urel_mag = sqrt(urel[0] * urel[0] + urel[1] * urel[1] + urel[2] * urel[2]);
    double dequiv = (2.0 * emaj) / pow(apr, 2.0 / 3.0);
    double rep = (urel_mag * dequiv) / s->visc;
    fdrag[0] = fdrag[1] = fdrag[2] = 0.0;
    flift[0] = flift[1] = flift[2] = 0.0;
    if (urel_mag == 0.0) return ORC_OK;    /* guard, see above */
    double pf[3] = {urel[0], urel[1], urel[2]};
    double cq[4];
    conjq(q, cq);
    orc_transform_vec(pf, cq);
    double syz = sqrt(pf[1] * pf[1] + pf[2] * pf[2]);
    double phi = fabs(atan(syz / pf[0]));
    double uflu_mag = sqrt(pf[0] * pf[0] + pf[1] * pf[1] + pf[2] * pf[2]);
    double cd0 = (a1 / pow(rep, a2)) + (a3 / pow(rep, a4));
    double cd90 = (a5 / pow(rep, a6)) + (a7 / pow(rep, a8));
    double cdrag = cd0 + (cd90 - cd0) * pow(sin(phi), a0);
    double clift = ((b1 / pow(rep, b2)) + (b3 / pow(rep, b4))) * pow(sin(phi), b5 + b6 * pow(rep, b7)) *
                   pow(cos(phi), b8 + b9 * pow(rep, b10));
    double c = (1.0 / 2.0) * (s->rhof / pmass) * (1.0 / 4.0) * (s->ppi * (dequiv * dequiv));
    fdrag[0] = c * cdrag * uflu_mag * pf[0];
    fdrag[1] = c * cdrag * uflu_mag * pf[1];
    fdrag[2] = c * cdrag * uflu_mag * pf[2];
    flift[0] = c * clift * (uflu_mag * uflu_mag) * sin(phi) * copysign(1.0, -pf[0]);
    if (syz != 0.0) {   /* guard, see above */
        flift[1] = c * clift * (uflu_mag * uflu_mag) * cos(phi) * (pf[1] / syz);
        flift[2] = c * clift * (uflu_mag * uflu_mag) * cos(phi) * (pf[2] / syz);
    }
    orc_transform_vec(fdrag, q);
    orc_transform_vec(flift, q);
    if (cdrag != cdrag) return ORC_ENAN_FORCE;   /* fluid_force_ellipsoid.f90:150-159 */
    return ORC_OK;
}

/* stat_partfluid.f90:122-293 for one particle: the 35 quantities the reference sums,
 * in its order, then 1.0 (the count).  No guards: the reference divides as written. */
void orc_stat_partfluid_particle(const orc_setup *s, double emaj, double apr, double rhop, const double u[3],
                                 const double om[3], const double q[4], const double uf[3], const double wv[3],
                                 double v[36]) {
    const double a0 = 1.95, a1 = 18.12, a2 = 1.023, a3 = 4.26, a4 = 0.384;
    const double a5 = 21.52, a6 = 0.990, a7 = 2.86, a8 = 0.260;
    const double b1 = 0.083, b2 = -0.21, b3 = 1.582, b4 = 0.851, b5 = 1.842;
    const double b6 = -0.802, b7 = -0.006, b8 = 0.874, b9 = 0.009, b10 = 0.570;
    const double c1 = 0.935, c2 = 0.146, c3 = -0.469, c4 = 0.145, c5 = 0.116;
    const double c6 = 0.748, c7 = 0.041, c8 = 0.221, c9 = 0.657, c10 = 0.044;
    const double r1 = 0.573, r2 = -0.154, r3 = 116.61, r4 = 1.0;
    const double r1_ = 1.244, r2_ = 0.239, r3_ = 378.12, r4_ = 0.789;
    const double ppi = s->ppi, rhof = s->rhof, visc = s->visc;
    double pa[3] = {1.0, 0.0, 0.0};                                          /* :127-129 */
    double pmass = pmass_of(s, emaj, apr, rhop);                            /* :131 */
    double urel[3] = {uf[0] - u[0], uf[1] - u[1], uf[2] - u[2]};            /* :134-136 */
    double urel_mag = sqrt(urel[0] * urel[0] + urel[1] * urel[1] + urel[2] * urel[2]);
    double dequiv = 2.0 * emaj / pow(apr, 2.0 / 3.0);                       /* :140 */
    double rep = (urel_mag * dequiv) / visc;
    double pf[3] = {uf[0] - u[0], uf[1] - u[1], uf[2] - u[2]};
    double cq[4];
    conjq(q, cq);
    orc_transform_vec(pf, cq);                                               /* :150 */
    double phi = fabs(atan((sqrt(pf[1] * pf[1] + pf[2] * pf[2])) / (pf[0])));
    double umag = sqrt(pf[0] * pf[0] + pf[1] * pf[1] + pf[2] * pf[2]);
    double cd0 = a1 / pow(rep, a2) + a3 / pow(rep, a4);                     /* :160-166 */
    double cd90 = a5 / pow(rep, a6) + a7 / pow(rep, a8);
    double cdrag = cd0 + (cd90 - cd0) * pow(sin(phi), a0);
    double clift = (b1 / pow(rep, b2) + b3 / pow(rep, b4)) * pow(sin(phi), b5 + b6 * pow(rep, b7)) *
                   pow(cos(phi), b8 + b9 * pow(rep, b10));
    double fd[3], fl[3];
    double syz = sqrt(pf[1] * pf[1] + pf[2] * pf[2]);
    for (int k = 0; k < 3; ++k)                                              /* :170-178 */
        fd[k] = (1.0 / 2.0) * (rhof / pmass) * (1.0 / 4.0) * (ppi * (dequiv * dequiv)) * cdrag * umag * pf[k];
    fl[0] = (1.0 / 2.0) * (rhof / pmass) * (1.0 / 4.0) * (ppi * (dequiv * dequiv)) * clift * (umag * umag) *
            sin(phi) * copysign(1.0, -pf[0]);
    fl[1] = (1.0 / 2.0) * (rhof / pmass) * (1.0 / 4.0) * (ppi * (dequiv * dequiv)) * clift * (umag * umag) *
            cos(phi) * (pf[1] / syz);
    fl[2] = (1.0 / 2.0) * (rhof / pmass) * (1.0 / 4.0) * (ppi * (dequiv * dequiv)) * clift * (umag * umag) *
            cos(phi) * (pf[2] / syz);
    orc_transform_vec(fd, q);
    orc_transform_vec(fl, q);
    v[0] = rep; v[1] = cdrag; v[2] = clift;                                  /* :183-195 */
    v[3] = fd[0]; v[4] = fd[1]; v[5] = fd[2];
    v[6] = fl[0]; v[7] = fl[1]; v[8] = fl[2];
    v[9] = sqrt(fd[0] * fd[0] + fd[1] * fd[1] + fd[2] * fd[2]);
    v[10] = sqrt(fl[0] * fl[0] + fl[1] * fl[1] + fl[2] * fl[2]);
    double curl[3] = {wv[0], wv[1], wv[2]};                                  /* :199-203 */
    orc_transform_vec(curl, cq);
    double o0 = 0.5 * curl[0] - om[0], o1 = 0.5 * curl[1] - om[1], o2 = 0.5 * curl[2] - om[2];
    double omag = sqrt(o0 * o0 + o1 * o1 + o2 * o2);
    double oyz = sqrt(o2 * o2 + o1 * o1);
    double re_r = (omag * (dequiv * dequiv)) / visc;                         /* :214 */
    double ctp = (c1 / pow(rep, c2) + c3 / pow(rep, c4)) * pow(sin(phi), c5 + c6 * pow(rep, c7)) *
                 pow(cos(phi), c8 + c9 * pow(rep, c10));
    double ctr = r1 * pow(re_r, r2) + r3 / pow(re_r, r4);
    double ctr2 = r1_ * pow(re_r, r2_) + r3_ / pow(re_r, r4_);
    double tp[3], tr[3];                                                     /* :224-243 */
    tp[0] = 0.0;
    tp[1] = (1.0 / 4.0) * (rhof / pmass) * (1.0 / 4.0) * ppi * ((dequiv * dequiv) * dequiv) * ctp * (umag * umag) *
            (fabs(pf[2]) / sqrt(pf[1] * pf[1] + pf[2] * pf[2])) * copysign(1.0, pf[0] * pf[2]);
    tp[2] = (1.0 / 4.0) * (rhof / pmass) * (1.0 / 4.0) * ppi * ((dequiv * dequiv) * dequiv) * ctp * (umag * umag) *
            (fabs(pf[1]) / sqrt(pf[1] * pf[1] + pf[2] * pf[2])) * copysign(1.0, pf[0] * pf[1]);
    double h = dequiv / 2.0, h2 = h * h, h5 = h2 * h2 * h;
    tr[0] = ctr * (rhof / pmass) / 2.0 * h5 * fabs(o0) * o0;
    tr[1] = ctr2 * (rhof / pmass) / 2.0 * h5 * oyz * o1;
    tr[2] = ctr2 * (rhof / pmass) / 2.0 * h5 * oyz * o2;
    orc_transform_vec(pa, q);                                                /* :245 */
    v[11] = re_r; v[12] = ctp; v[13] = ctr;                                  /* :247-263 */
    v[14] = tp[0]; v[15] = tp[1]; v[16] = tp[2];
    v[17] = tr[0]; v[18] = tr[1]; v[19] = tr[2];
    v[20] = sqrt(tp[0] * tp[0] + tp[1] * tp[1] + tp[2] * tp[2]);
    v[21] = sqrt(tr[0] * tr[0] + tr[1] * tr[1] + tr[2] * tr[2]);
    double minax = emaj / apr;                                               /* :265-276 */
    double fbeta;
    if (apr == 1.0) fbeta = 1.0;
    else fbeta = (apr * log(apr + sqrt(apr * apr - 1.0))) / (sqrt(apr * apr - 1.0));
    double taupf = (2.0 / 9.0) * (rhop * (minax * minax)) / (rhof * visc);
    taupf = taupf * fbeta;
    v[22] = taupf;
    v[23] = s->gravity;
    v[24] = phi;
    v[25] = pa[0]; v[26] = pa[1]; v[27] = pa[2];
    v[28] = (0.5 * rhof * cdrag * (ppi / 4.0) * (dequiv * dequiv) * umag) / pmass;   /* :285 */
    v[29] = u[0]; v[30] = u[1]; v[31] = u[2];
    v[32] = om[0]; v[33] = om[1]; v[34] = om[2];
    v[35] = 1.0;
}

/* stat_partfluid.f90:115-299: the sums over the particles, in their order, per index
 * (group[i] in 1..ngroups, or all 1 when group is NULL); out: ngroups*36. */
void orc_stat_partfluid(const orc_setup *s, const orc_props *p, const orc_state *st, const int32_t *group,
                        int32_t ngroups, double *out) {
    for (int64_t k = 0; k < (int64_t)ngroups * 36; ++k) out[k] = 0.0;
    for (int64_t i = 0; i < st->n; ++i) {
        double v[36];
        const double u[3] = {st->u[i], st->v[i], st->w[i]};
        const double om[3] = {st->ox[i], st->oy[i], st->oz[i]};
        const double q[4] = {st->qa[i], st->qb[i], st->qc[i], st->qd[i]};
        const double uf[3] = {st->ufap[i], st->vfap[i], st->wfap[i]};
        const double wv[3] = {st->vortx[i], st->vorty[i], st->vortz[i]};
        orc_stat_partfluid_particle(s, p->emaj[i], p->apr[i], p->rhop[i], u, om, q, uf, wv, v);
        double *o = out + (int64_t)(group ? group[i] - 1 : 0) * 36;
        for (int k = 0; k < 36; ++k) o[k] = o[k] + v[k];
    }
}

/* fluid_torque_ellipsoid.f90:1-190.  Pitching and rotation torque per unit mass in the
 * body frame.  The relative velocity uses the particle's stored velocity u_n
 * (fluid_torque_ellipsoid.f90:88-105), not the stage velocity.
 * Guards as in orc_fluid_force: zero relative speed -> zero pitching torque, zero
 * transverse component -> zero pitching torque, zero rotational Reynolds number ->
 * zero rotation torque. */
int orc_fluid_torque(const orc_setup *s, double emaj, double apr, double rhop,
                     double up_n, double vp_n, double wp_n,
                     double uf, double vf, double wf,
                     double vortx, double vorty, double vortz,
                     double ox, double oy, double oz, const double q[4],
                     double tpitch[3], double trot[3]) {
    const double c1 = 0.935, c2 = 0.146, c3 = -0.469, c4 = 0.145, c5 = 0.116;
    const double c6 = 0.748, c7 = 0.041, c8 = 0.221, c9 = 0.657, c10 = 0.044;
    const double r1 = 0.573, r2 = -0.154, r3 = 116.61, r4 = 1.0;
    const double r1_ = 1.244, r2_ = 0.239, r3_ = 378.12, r4_ = 0.789;
    const double pmass = pmass_of(s, emaj, apr, rhop);
    double urel[3] = {uf - up_n, vf - vp_n, wf - wp_n};
    double urel_mag = sqrt(urel[0] * urel[0] + urel[1] * urel[1] + urel[2] * urel[2]);
    double dequiv = 2.0 * emaj / pow(apr, 2.0 / 3.0);
    double rep = (urel_mag * dequiv) / s->visc;
    double cq[4];
    conjq(q, cq);
    double pf[3] = {urel[0], urel[1], urel[2]};
    orc_transform_vec(pf, cq);
    double syz = sqrt(pf[1] * pf[1] + pf[2] * pf[2]);
    double phi = fabs(atan(syz / pf[0]));
    double uflu_mag = sqrt(pf[0] * pf[0] + pf[1] * pf[1] + pf[2] * pf[2]);
    double curl[3] = {vortx, vorty, vortz};
    orc_transform_vec(curl, cq);
    double orel[3] = {0.5 * curl[0] - ox, 0.5 * curl[1] - oy, 0.5 * curl[2] - oz};
    double orel_mag = sqrt(orel[0] * orel[0] + orel[1] * orel[1] + orel[2] * orel[2]);
    double orel_yz = sqrt(orel[2] * orel[2] + orel[1] * orel[1]);
    double re_r = (orel_mag * (dequiv * dequiv)) / s->visc;
    tpitch[0] = 0.0; tpitch[1] = 0.0; tpitch[2] = 0.0;
    trot[0] = 0.0; trot[1] = 0.0; trot[2] = 0.0;
    if (urel_mag != 0.0 && syz != 0.0) {   /* guard */
        double ctpitch = (c1 / pow(rep, c2) + c3 / pow(rep, c4)) * (pow(sin(phi), c5 + c6 * pow(rep, c7))) *
                         (pow(cos(phi), c8 + c9 * pow(rep, c10)));
        double d3 = dequiv * dequiv * dequiv;
        double cp = (1.0 / 4.0) * (s->rhof / pmass) * (1.0 / 4.0) * s->ppi * d3 * ctpitch * (uflu_mag * uflu_mag);
        tpitch[1] = cp * (fabs(pf[2]) / syz) * copysign(1.0, pf[0] * pf[2]);
        tpitch[2] = cp * (fabs(pf[1]) / syz) * copysign(1.0, pf[0] * pf[1]);
    }
    if (re_r != 0.0) {   /* guard */
        double ctrot = r1 * pow(re_r, r2) + r3 / pow(re_r, r4);
        double ctrot2 = r1_ * pow(re_r, r2_) + r3_ / pow(re_r, r4_);
        double h = dequiv / 2.0, h2 = h * h, h5 = h2 * h2 * h;
        double k = 0.5 * s->rhof / pmass;
        trot[0] = ctrot * k * h5 * fabs(orel[0]) * orel[0];
        trot[1] = ctrot2 * k * h5 * orel_yz * orel[1];
        trot[2] = ctrot2 * k * h5 * orel_yz * orel[2];
    }
    if (ox != ox) return ORC_ENAN_TORQUE;   /* fluid_torque_ellipsoid.f90:178-188 */
    return ORC_OK;
}

/* ------------------------------------------------------------------------- */
/* Interpolation                                                             */
/* ------------------------------------------------------------------------- */

/* Cubic Lagrange weights, interp_lag3.f90:196-211 */
static inline void lag3_weights(double a, double f[4]) {
    f[0] = -1. / 6. * (a - 2.) * (a - 1.) * a;
    f[1] = 1. / 2. * (a - 2.) * (a - 1.) * (a + 1.);
    f[2] = -1. / 2. * (a - 2.) * a * (a + 1.);
    f[3] = 1. / 6. * (a - 1.) * a * (a + 1.);
}

/* 64-point sum with the reference's nesting z(y(x)), interp_lag3.f90:220-288.
 * idx(i,j,k) returns the linear index of the field point. */
#define LAG3_SUM(FIELD, IX, JY, KZ, FX, FY, FZ, OUT)                                      \
    do {                                                                                   \
        double zs = 0.0;                                                                   \
        for (int kk = 0; kk < 4; ++kk) {                                                   \
            double ys = 0.0;                                                               \
            for (int jj = 0; jj < 4; ++jj) {                                               \
                double xs = FX[0] * FIELD[IDX(IX[0], JY[jj], KZ[kk])] +                    \
                            FX[1] * FIELD[IDX(IX[1], JY[jj], KZ[kk])] +                    \
                            FX[2] * FIELD[IDX(IX[2], JY[jj], KZ[kk])] +                    \
                            FX[3] * FIELD[IDX(IX[3], JY[jj], KZ[kk])];                     \
                ys = (jj == 0) ? FY[0] * xs : ys + FY[jj] * xs;                            \
            }                                                                              \
            zs = (kk == 0) ? FZ[0] * ys : zs + FZ[kk] * ys;                                \
        }                                                                                  \
        OUT = zs;                                                                          \
    } while (0)

/* interp_lag3.f90:11-298 with ISTART=1, IEND=N, NGHTCELL=2.
 * uain: (NX, NY+4, NZ+4) with y/z ghost planes, x fastest. */
void orc_interp_lag3(const orc_setup *s, const double *uain, int64_t nint,
                     const double *xint, const double *yint, const double *zint,
                     double *uint) {
    const int64_t NX = s->nx, NY = s->ny;
    const double dxa = 1.0 * s->dx - 0.0 * s->dx;  /* XAIN(2)-XAIN(1), meshing.f90:55 */
    const double dya = s->dy * 1.0 - s->dy * 0.0;
    const double dza = s->dz * 1.0 - s->dz * 0.0;
#define IDX(i, j, k) (((int64_t)(i) - 1) + NX * (((int64_t)(j) + 1) + (NY + 4) * ((int64_t)(k) + 1)))
    for (int64_t np = 0; np < nint; ++np) {
        int i0 = (int)(xint[np] / dxa) + 1;
        int j0 = (int)(yint[np] / dya) + 1;
        int k0 = (int)(zint[np] / dza) + 1;
        int ip1, ip2, im1;
        const int iend = s->nx, istart = 1;
        if (i0 == iend && s->wall_boundary) ip1 = iend - 1;
        else if (i0 == iend) ip1 = 1;
        else ip1 = i0 + 1;
        if (ip1 == iend && s->wall_boundary) ip2 = iend - 1;
        else if (ip1 == iend) ip2 = 1;
        else ip2 = ip1 + 1;
        if (i0 == istart && s->wall_boundary) im1 = istart + 1;
        else if (i0 == istart) im1 = iend;
        else im1 = i0 - 1;
        int ix[4] = {im1, i0, ip1, ip2};
        int jy[4] = {j0 - 1, j0, j0 + 1, j0 + 2};
        int kz[4] = {k0 - 1, k0, k0 + 1, k0 + 2};
        double alfa = (xint[np] - (double)(i0 - 1) * s->dx) / dxa;   /* XMESH(I)=(I-1)*DX */
        double beta = (yint[np] - s->dy * (double)(j0 - 1)) / dya;   /* YMESH(J)=DY*(J-1) */
        double gama = (zint[np] - s->dz * (double)(k0 - 1)) / dza;
        double fx[4], fy[4], fz[4];
        lag3_weights(alfa, fx);
        lag3_weights(beta, fy);
        lag3_weights(gama, fz);
        double out;
        LAG3_SUM(uain, ix, jy, kz, fx, fy, fz, out);
        uint[np] = out;
    }
#undef IDX
}

/* frozen_interp_lag3.f90:11-274: same stencil on a plain (NX,NY,NZ) array with
 * mirror boundaries (including the reference's JP2 test against NZ at :148).
 * Out-of-range stencil indices (the reference would read out of bounds) give NaN. */
void orc_frozen_interp_lag3(const double *xain, const double *yain, const double *zain,
                            int32_t nx, int32_t ny, int32_t nz, const double *uain,
                            int64_t nint, const double *xint, const double *yint,
                            const double *zint, double *uint) {
    const int64_t NX = nx, NY = ny;
    const double dxa = xain[1] - xain[0], dya = yain[1] - yain[0], dza = zain[1] - zain[0];
#define IDX(i, j, k) (((int64_t)(i) - 1) + NX * (((int64_t)(j) - 1) + NY * ((int64_t)(k) - 1)))
    for (int64_t np = 0; np < nint; ++np) {
        int i0 = (int)(xint[np] / dxa) + 1;
        int j0 = (int)(yint[np] / dya) + 1;
        int k0 = (int)(zint[np] / dza) + 1;
        int ip1 = i0 + 1; if (i0 == nx) ip1 = nx - 1;
        int ip2 = ip1 + 1; if (ip1 == nx) ip2 = nx - 1;
        int im1 = i0 - 1; if (i0 == 1) im1 = 2;
        int jm1 = j0 - 1; if (j0 == 1) jm1 = 2;
        int jp1 = j0 + 1; if (j0 == ny) jp1 = ny - 1;
        int jp2 = jp1 + 1; if (jp1 == nz) jp2 = ny - 1;
        int km1 = k0 - 1; if (k0 == 1) km1 = 2;
        int kp1 = k0 + 1; if (k0 == nz) kp1 = nz - 1;
        int kp2 = kp1 + 1; if (kp1 == nz) kp2 = nz - 1;
        int ix[4] = {im1, i0, ip1, ip2};
        int jy[4] = {jm1, j0, jp1, jp2};
        int kz[4] = {km1, k0, kp1, kp2};
        int bad = 0;
        for (int t = 0; t < 4; ++t) {
            if (ix[t] < 1 || ix[t] > nx || jy[t] < 1 || jy[t] > ny || kz[t] < 1 || kz[t] > nz) bad = 1;
        }
        if (i0 < 1 || i0 > nx || j0 < 1 || j0 > ny || k0 < 1 || k0 > nz) bad = 1;
        if (bad) { uint[np] = NAN; continue; }
        double alfa = (xint[np] - xain[i0 - 1]) / dxa;
        double beta = (yint[np] - yain[j0 - 1]) / dya;
        double gama = (zint[np] - zain[k0 - 1]) / dza;
        double fx[4], fy[4], fz[4];
        lag3_weights(alfa, fx);
        lag3_weights(beta, fy);
        lag3_weights(gama, fz);
        double out;
        LAG3_SUM(uain, ix, jy, kz, fx, fy, fz, out);
        uint[np] = out;
    }
#undef IDX
}

/* ------------------------------------------------------------------------- */
/* Walls                                                                     */
/* ------------------------------------------------------------------------- */

static void inv_ellipsoid_matrix(double emaj, double apr, const double q[4], double ell[9]) {
    double a = emaj, b = a / apr, c = b;
    memset(ell, 0, 9 * sizeof(double));
    M3(ell, 0, 0) = 1.0 / (a * a);
    M3(ell, 1, 1) = 1.0 / (b * b);
    M3(ell, 2, 2) = 1.0 / (c * c);
    orc_transform_tensor(ell, q);
}

/* closest_point_plane.f90:1-120 */
static int closest_point_plane(double emaj, double apr, double xp, double yp, double zp,
                               const double q[4], const double wpos[3], const double wn[3],
                               double plane_vec[3], double *margin) {
    double ellc[3] = {xp, yp, zp};
    double ell[9], inv[9];
    inv_ellipsoid_matrix(emaj, apr, q, ell);
    if (orc_invert3(ell, inv)) return ORC_ESINGULAR;
    double ivn[3];
    matvec3(inv, wn, ivn);
    double tn = wn[0] * ivn[0] + wn[1] * ivn[1] + wn[2] * ivn[2];
    double d[3] = {wpos[0] - ellc[0], wpos[1] - ellc[1], wpos[2] - ellc[2]};
    double tw = wn[0] * d[0] + wn[1] * d[1] + wn[2] * d[2];
    double lagrange = tw / tn;
    for (int i = 0; i < 3; ++i) plane_vec[i] = ellc[i] + lagrange * ivn[i];
    double vec[3] = {plane_vec[0] - ellc[0], plane_vec[1] - ellc[1], plane_vec[2] - ellc[2]};
    double e_[3];
    matvec3(ell, vec, e_);
    *margin = vec[0] * e_[0] + vec[1] * e_[1] + vec[2] * e_[2];
    return ORC_OK;
}

/* max_encroachment_ellipsoid.f90:1-106 */
static int max_encroachment(double emaj, double apr, double xp, double yp, double zp,
                            const double q[4], const double n[3], double point[3]) {
    double ellc[3] = {xp, yp, zp};
    double ell[9], inv[9];
    inv_ellipsoid_matrix(emaj, apr, q, ell);
    if (orc_invert3(ell, inv)) return ORC_ESINGULAR;
    double ivn[3];
    matvec3(inv, n, ivn);
    double tn = n[0] * ivn[0] + n[1] * ivn[1] + n[2] * ivn[2];
    double s = sqrt(tn);
    for (int i = 0; i < 3; ++i) point[i] = ellc[i] - ivn[i] / s;
    return ORC_OK;
}

/* ellipsoid_wall_boundary_new.f90:1-113.  delta_x is written only when intersecting
 * (the reference leaves it untouched otherwise). */
int orc_wall_boundary_condition(const orc_setup *s, double emaj, double apr,
                                double xp, double yp, double zp, const double q[4],
                                double wall_normal[3], double impact_arm[3],
                                double *delta_x, int32_t *is_intersect) {
    double wpos[3];
    impact_arm[0] = impact_arm[1] = impact_arm[2] = 0.0;
    *is_intersect = 0;
    if (xp < s->lx / 2.0) {
        wpos[0] = 0.0; wpos[1] = yp; wpos[2] = zp;
        wall_normal[0] = 1.0; wall_normal[1] = 0.0; wall_normal[2] = 0.0;
    } else {
        wpos[0] = s->lx; wpos[1] = yp; wpos[2] = zp;
        wall_normal[0] = -1.0; wall_normal[1] = 0.0; wall_normal[2] = 0.0;
    }
    double plane_pt[3], margin;
    int rc = closest_point_plane(emaj, apr, xp, yp, zp, q, wpos, wall_normal, plane_pt, &margin);
    if (rc) return rc;
    if (margin < 1.0) {
        *is_intersect = 1;
        double ellip_pt[3];
        rc = max_encroachment(emaj, apr, xp, yp, zp, q, wall_normal, ellip_pt);
        if (rc) return rc;
        impact_arm[0] = (xp - ellip_pt[0]);
        impact_arm[1] = (yp - ellip_pt[1]);
        impact_arm[2] = (zp - ellip_pt[2]);
        *delta_x = wpos[0] - ellip_pt[0];
    }
    return ORC_OK;
}

static void skew(const double r[3], double rx[9]) {
    M3(rx, 0, 0) = 0.0;   M3(rx, 0, 1) = -r[2]; M3(rx, 0, 2) = r[1];
    M3(rx, 1, 0) = r[2];  M3(rx, 1, 1) = 0.0;   M3(rx, 1, 2) = -r[0];
    M3(rx, 2, 0) = -r[1]; M3(rx, 2, 1) = r[0];  M3(rx, 2, 2) = 0.0;
}

/* wall_ellipsoid_rebound.f90:1-387 */
int orc_wall_rebound(const orc_setup *s, double ipxx, double ipyy, double ipzz,
                     double *u, double *v, double *w, double *ox, double *oy, double *oz,
                     const double q[4], const double ri[3], const double nw[3]) {
    double up[3] = {*u, *v, *w};
    double omg[3] = {*ox, *oy, *oz};
    orc_transform_vec(omg, q);
    double vpc[3];
    vpc[0] = up[0] + (omg[1] * ri[2] - omg[2] * ri[1]);
    vpc[1] = up[1] + (omg[2] * ri[0] - omg[0] * ri[2]);
    vpc[2] = up[2] + (omg[0] * ri[1] - omg[1] * ri[0]);
    double vrn = vpc[0] * nw[0] + vpc[1] * nw[1] + vpc[2] * nw[2];
    double delv[3];
    for (int i = 0; i < 3; ++i) delv[i] = vpc[i] + s->ecw * vrn * nw[i];
    double ip[9] = {0}, inv_ip[9] = {0};
    M3(ip, 0, 0) = ipxx; M3(ip, 1, 1) = ipyy; M3(ip, 2, 2) = ipzz;
    orc_transform_tensor(ip, q);
    if (orc_invert3(ip, inv_ip)) return ORC_ESINGULAR;
    double rx[9], rxt[9], t[9], k[9], k1[9];
    skew(ri, rx);
    transpose33(rx, rxt);
    matmul33(inv_ip, rx, t);
    matmul33(rxt, t, t);
    for (int i = 0; i < 9; ++i) k[i] = ((i % 4) == 0 ? 1.0 : 0.0) + t[i];
    if (orc_invert3(k, k1)) return ORC_ESINGULAR;
    double pc[3];
    matvec3(k1, delv, pc);
    pc[0] = -pc[0]; pc[1] = -pc[1]; pc[2] = -pc[2];
    double pcn = pc[0] * nw[0] + pc[1] * nw[1] + pc[2] * nw[2];
    double pct_x = pc[0] - pcn * nw[0], pct_y = pc[1] - pcn * nw[1], pct_z = pc[2] - pcn * nw[2];
    double pct = sqrt(pct_x * pct_x + pct_y * pct_y + pct_z * pct_z);
    if (pct > s->muw * pcn) {
        double tw[3] = {vpc[0] - vrn * nw[0], vpc[1] - vrn * nw[1], vpc[2] - vrn * nw[2]};
        double nrm_tw = sqrt(tw[0] * tw[0] + tw[1] * tw[1] + tw[2] * tw[2]);
        if (nrm_tw != 0.0) {
            tw[0] = -tw[0] / nrm_tw; tw[1] = -tw[1] / nrm_tw; tw[2] = -tw[2] / nrm_tw;
        }
        double vimp[3] = {nw[0] + s->muw * tw[0], nw[1] + s->muw * tw[1], nw[2] + s->muw * tw[2]};
        double kn[3];
        matvec3(k, vimp, kn);
        double kn_dot_n = kn[0] * nw[0] + kn[1] * nw[1] + kn[2] * nw[2];
        pcn = -1.0 * (delv[0] * nw[0] + delv[1] * nw[1] + delv[2] * nw[2]);
        for (int i = 0; i < 3; ++i) pc[i] = (pcn / kn_dot_n) * vimp[i];
    }
    double e_it = 0.5 * (*u * *u + *v * *v + *w * *w);
    double am[3];
    matvec3(ip, omg, am);
    double e_ir = 0.5 * (omg[0] * am[0] + omg[1] * am[1] + omg[2] * am[2]);
    double e_i = e_it + e_ir;
    *u = *u + pc[0]; *v = *v + pc[1]; *w = *w + pc[2];
    double tmp[3], dom[3];
    matvec3(rx, pc, tmp);
    matvec3(inv_ip, tmp, dom);
    for (int i = 0; i < 3; ++i) omg[i] = omg[i] + dom[i];
    double e_ft = 0.5 * (*u * *u + *v * *v + *w * *w);
    matvec3(ip, omg, am);
    double e_fr = 0.5 * (omg[0] * am[0] + omg[1] * am[1] + omg[2] * am[2]);
    double e_f = e_ft + e_fr;
    double cq[4];
    conjq(q, cq);
    orc_transform_vec(omg, cq);
    *ox = omg[0]; *oy = omg[1]; *oz = omg[2];
    if (fabs((e_i - e_f) / e_i) * 100.0 > 1.0e-9) return ORC_EENERGY;  /* :372-385 */
    return ORC_OK;
}

/* ------------------------------------------------------------------------- */
/* ADV_PARTICLE_ELLP                                                         */
/* ------------------------------------------------------------------------- */

typedef struct { double x, y, z, u, v, w, ox, oy, oz, q[4]; } pstate;

static inline void k_omega(const double t[3], double ox, double oy, double oz,
                           double ipxx, double ipyy, double ipzz, double k[3]) {
    /* adv_particle_new.f90:305-307 */
    k[0] = (t[0] + oy * oz * (ipyy - ipzz)) / ipxx;
    k[1] = (t[1] + oz * ox * (ipzz - ipxx)) / ipyy;
    k[2] = (t[2] + ox * oy * (ipxx - ipyy)) / ipzz;
}

/* One particle of adv_particle_new.f90:268-637 (PARTDEF=2, FROZEN_FLOW>0). */
static int advance_one(const orc_setup *s, double emaj, double apr, double rhop,
                       double ipxx, double ipyy, double ipzz,
                       const double uf[3], const double vort[3], pstate *P) {
    int rc;
    const double dt = s->dtime;
    double k1x[3] = {P->u, P->v, P->w};
    double fd[3], fl[3], tp[3], tr[3];
    rc = orc_fluid_force(s, emaj, apr, rhop, P->u, P->v, P->w, uf[0], uf[1], uf[2], P->q, fd, fl);
    if (rc) return rc;
    double ff[3] = {fd[0] + fl[0], fd[1] + fl[1], fd[2] + fl[2]};
    rc = orc_fluid_torque(s, emaj, apr, rhop, P->u, P->v, P->w, uf[0], uf[1], uf[2],
                          vort[0], vort[1], vort[2], P->ox, P->oy, P->oz, P->q, tp, tr);
    if (rc) return rc;
    double ft[3] = {tp[0] + tr[0], tp[1] + tr[1], tp[2] + tr[2]};
    double k1u[3] = {ff[0], ff[1], ff[2] + s->gravity};
    double k1o[3];
    k_omega(ft, P->ox, P->oy, P->oz, ipxx, ipyy, ipzz, k1o);

    double xp1 = P->x + dt * k1x[0], yp1 = P->y + dt * k1x[1], zp1 = P->z + dt * k1x[2];
    double up1 = P->u + dt * k1u[0], vp1 = P->v + dt * k1u[1], wp1 = P->w + dt * k1u[2];
    double ox1 = P->ox + dt * k1o[0], oy1 = P->oy + dt * k1o[1], oz1 = P->oz + dt * k1o[2];
    double quat1[4] = {P->q[0], P->q[1], P->q[2], P->q[3]};
    orc_quaternion_integration(quat1, ox1, oy1, oz1, dt);

    double wall_normal[3], impact_arm[3], delta_x = 0.0;
    int32_t isect;
    rc = orc_wall_boundary_condition(s, emaj, apr, xp1, yp1, zp1, quat1, wall_normal, impact_arm, &delta_x, &isect);
    if (rc) return rc;
    double omg_lab[3] = {ox1, oy1, oz1};
    orc_transform_vec(omg_lab, quat1);
    double vpc[3];
    vpc[0] = up1 + (omg_lab[1] * impact_arm[2] - omg_lab[2] * impact_arm[1]);
    vpc[1] = vp1 + (omg_lab[2] * impact_arm[0] - omg_lab[0] * impact_arm[2]);
    vpc[2] = wp1 + (omg_lab[0] * impact_arm[1] - omg_lab[1] * impact_arm[0]);

    if (isect && up1 * wall_normal[0] < 0.0) {
        /* adv_particle_new.f90:358-511: rebound branch */
        double x_wall = xp1 + delta_x;
        xp1 = x_wall;
        double delt = fabs(delta_x) / sqrt(vpc[0] * vpc[0] + vpc[1] * vpc[1] + vpc[2] * vpc[2]);
        yp1 = P->y + (dt - delt) * k1x[1];
        zp1 = P->z + (dt - delt) * k1x[2];
        up1 = P->u + (dt - delt) * k1u[0];
        vp1 = P->v + (dt - delt) * k1u[1];
        wp1 = P->w + (dt - delt) * k1u[2];
        ox1 = P->ox + (dt - delt) * k1o[0];
        oy1 = P->oy + (dt - delt) * k1o[1];
        oz1 = P->oz + (dt - delt) * k1o[2];
        quat1[0] = P->q[0]; quat1[1] = P->q[1]; quat1[2] = P->q[2]; quat1[3] = P->q[3];
        orc_quaternion_integration(quat1, ox1, oy1, oz1, dt - delt);
        rc = orc_wall_rebound(s, ipxx, ipyy, ipzz, &up1, &vp1, &wp1, &ox1, &oy1, &oz1, quat1, impact_arm, wall_normal);
        if (rc) return rc;
        double k2x[3] = {up1, vp1, wp1};
        rc = orc_fluid_force(s, emaj, apr, rhop, up1, vp1, wp1, uf[0], uf[1], uf[2], quat1, fd, fl);
        if (rc) return rc;
        ff[0] = fd[0] + fl[0]; ff[1] = fd[1] + fl[1]; ff[2] = fd[2] + fl[2];
        rc = orc_fluid_torque(s, emaj, apr, rhop, P->u, P->v, P->w, uf[0], uf[1], uf[2],
                              vort[0], vort[1], vort[2], ox1, oy1, oz1, quat1, tp, tr);
        if (rc) return rc;
        ft[0] = tp[0] + tr[0]; ft[1] = tp[1] + tr[1]; ft[2] = tp[2] + tr[2];
        double k2u[3] = {ff[0], ff[1], ff[2] + s->gravity};
        double k2o[3];
        k_omega(ft, ox1, oy1, oz1, ipxx, ipyy, ipzz, k2o);
        P->x = xp1 + (delt) * k2x[0];
        P->y = yp1 + (delt) * k2x[1];
        P->z = zp1 + (delt) * k2x[2];
        P->u = up1 + (delt) * k2u[0];
        P->v = vp1 + (delt) * k2u[1];
        P->w = wp1 + (delt) * k2u[2];
        P->ox = ox1 + (delt) * k2o[0];
        P->oy = oy1 + (delt) * k2o[1];
        P->oz = oz1 + (delt) * k2o[2];
        P->q[0] = quat1[0]; P->q[1] = quat1[1]; P->q[2] = quat1[2]; P->q[3] = quat1[3];
        orc_quaternion_integration(P->q, P->ox, P->oy, P->oz, delt);
        return ORC_OK;
    }
    /* adv_particle_new.f90:513-637: unbounced second stage */
    double k2x[3] = {up1, vp1, wp1};
    rc = orc_fluid_force(s, emaj, apr, rhop, up1, vp1, wp1, uf[0], uf[1], uf[2], quat1, fd, fl);
    if (rc) return rc;
    ff[0] = fd[0] + fl[0]; ff[1] = fd[1] + fl[1]; ff[2] = fd[2] + fl[2];
    rc = orc_fluid_torque(s, emaj, apr, rhop, P->u, P->v, P->w, uf[0], uf[1], uf[2],
                          vort[0], vort[1], vort[2], ox1, oy1, oz1, quat1, tp, tr);
    if (rc) return rc;
    ft[0] = tp[0] + tr[0]; ft[1] = tp[1] + tr[1]; ft[2] = tp[2] + tr[2];
    double k2u[3] = {ff[0], ff[1], ff[2] + s->gravity};
    double k2o[3];
    k_omega(ft, ox1, oy1, oz1, ipxx, ipyy, ipzz, k2o);
    double xp2 = P->x + 0.5 * dt * (k1x[0] + k2x[0]);
    double yp2 = P->y + 0.5 * dt * (k1x[1] + k2x[1]);
    double zp2 = P->z + 0.5 * dt * (k1x[2] + k2x[2]);
    rc = orc_wall_boundary_condition(s, emaj, apr, xp2, yp2, zp2, quat1, wall_normal, impact_arm, &delta_x, &isect);
    if (rc) return rc;
    if (isect) {
        P->x = P->x + dt * k1x[0];
        P->y = P->y + dt * k1x[1];
        P->z = P->z + dt * k1x[2];
        P->u = P->u + dt * k1u[0];
        P->v = P->v + dt * k1u[1];
        P->w = P->w + dt * k1u[2];
        P->ox = P->ox + dt * k1o[0];
        P->oy = P->oy + dt * k1o[1];
        P->oz = P->oz + dt * k1o[2];
    } else {
        P->x = P->x + 0.5 * dt * (k1x[0] + k2x[0]);
        P->y = P->y + 0.5 * dt * (k1x[1] + k2x[1]);
        P->z = P->z + 0.5 * dt * (k1x[2] + k2x[2]);
        P->u = P->u + 0.5 * dt * (k1u[0] + k2u[0]);
        P->v = P->v + 0.5 * dt * (k1u[1] + k2u[1]);
        P->w = P->w + 0.5 * dt * (k1u[2] + k2u[2]);
        P->ox = P->ox + 0.5 * dt * (k1o[0] + k2o[0]);
        P->oy = P->oy + 0.5 * dt * (k1o[1] + k2o[1]);
        P->oz = P->oz + 0.5 * dt * (k1o[2] + k2o[2]);
    }
    P->q[0] = quat1[0]; P->q[1] = quat1[1]; P->q[2] = quat1[2]; P->q[3] = quat1[3];
    orc_quaternion_integration(P->q, P->ox, P->oy, P->oz, dt);
    return ORC_OK;
}

int orc_adv_particle_ellp(const orc_setup *s, const orc_props *p,
                          const double *const fields[6], orc_state *st,
                          int32_t nthreads, int64_t *err_id) {
    const int64_t n = st->n;
    int64_t first_bad = n;
    int first_rc = ORC_OK;
    /* 1. interpolation of u,v,w and the vorticity at x_n (adv_particle_new.f90:139-206) */
    double *outs[6] = {st->ufap, st->vfap, st->wfap, st->vortx, st->vorty, st->vortz};
#ifdef _OPENMP
    int nt = nthreads > 0 ? nthreads : 1;
#pragma omp parallel for schedule(static) num_threads(nt)
#endif
    for (int64_t blk = 0; blk < (n + 4095) / 4096; ++blk) {
        int64_t b0 = blk * 4096, cnt = (n - b0) < 4096 ? (n - b0) : 4096;
        for (int c = 0; c < 6; ++c)
            orc_interp_lag3(s, fields[c], cnt, st->x + b0, st->y + b0, st->z + b0, outs[c] + b0);
    }
    /* 2. particle loop (adv_particle_new.f90:268-644) */
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(nt)
#endif
    for (int64_t i = 0; i < n; ++i) {
        pstate P = {st->x[i], st->y[i], st->z[i], st->u[i], st->v[i], st->w[i],
                    st->ox[i], st->oy[i], st->oz[i], {st->qa[i], st->qb[i], st->qc[i], st->qd[i]}};
        double uf[3] = {st->ufap[i], st->vfap[i], st->wfap[i]};
        double vo[3] = {st->vortx[i], st->vorty[i], st->vortz[i]};
        int rc = advance_one(s, p->emaj[i], p->apr[i], p->rhop[i], p->ipxx[i], p->ipyy[i], p->ipzz[i], uf, vo, &P);
        if (rc) {
#ifdef _OPENMP
#pragma omp critical
#endif
            {
                if (i < first_bad) { first_bad = i; first_rc = rc; }
            }
        }
        st->x[i] = P.x; st->y[i] = P.y; st->z[i] = P.z;
        st->u[i] = P.u; st->v[i] = P.v; st->w[i] = P.w;
        st->ox[i] = P.ox; st->oy[i] = P.oy; st->oz[i] = P.oz;
        st->qa[i] = P.q[0]; st->qb[i] = P.q[1]; st->qc[i] = P.q[2]; st->qd[i] = P.q[3];
    }
    /* 3. particle boundary conditions (adv_particle_new.f90:685-686): the channel
     * (FROZEN_FLOW = 3) wraps y and z only, BOUNDARY_PARTICLE_Y_Z
     * (boundary_particle_yz.f90:44-70); below it, a periodic box wraps every direction,
     * BOUNDARY_PARTICLE (boundary_particle.f90:45-62) */
    if (s->frozen_flow == 3) {
        for (int64_t i = 0; i < n; ++i) {
            if (st->y[i] > s->ly) st->y[i] = st->y[i] - s->ly;
            else if (st->y[i] < 0.) st->y[i] = st->y[i] + s->ly;
            if (st->z[i] > s->lz) st->z[i] = st->z[i] - s->lz;
            else if (st->z[i] < 0.) st->z[i] = st->z[i] + s->lz;
        }
    } else if (s->periodicity) {
        for (int64_t i = 0; i < n; ++i) {
            if (st->x[i] > s->lx) st->x[i] = st->x[i] - s->lx;
            if (st->x[i] < 0.) st->x[i] = st->x[i] + s->lx;
            if (st->y[i] > s->ly) st->y[i] = st->y[i] - s->ly;
            if (st->y[i] < 0.) st->y[i] = st->y[i] + s->ly;
            if (st->z[i] > s->lz) st->z[i] = st->z[i] - s->lz;
            if (st->z[i] < 0.) st->z[i] = st->z[i] + s->lz;
        }
    }
    if (err_id) *err_id = first_rc ? first_bad : -1;
    return first_rc;
}

/* ------------------------------------------------------------------------- */
/* Collision grid                                                            */
/* ------------------------------------------------------------------------- */

/* collision_initiation.f90:44-103 with INIT_GRID=2 and NPROC=1 (DELTA_COLL=ZERO). */
void orc_collision_initiation(const orc_setup *s, double max_emaj, orc_boxgrid *g) {
    double dpmax = 2.0 * max_emaj;
    double dxbox = 2.0 * dpmax;
    g->nxbox = (int32_t)(s->lx / dxbox);
    g->dxbox = s->lx / (double)g->nxbox;
    g->delta_coll = ZERO_REF;
    g->xminbox = (double)(1 - 1) * s->dx;
    g->xmaxbox = (double)(s->nx - 1) * s->dx + s->dx;
    g->yminbox = s->dy * (double)(1 - 1) - g->delta_coll;
    g->ymaxbox = s->dy * (double)(s->ny - 1) + s->dy + g->delta_coll;
    g->zminbox = s->dz * (double)(1 - 1) - g->delta_coll;
    g->zmaxbox = s->dz * (double)(s->nz - 1) + s->dz + g->delta_coll;
    g->nybox = (int32_t)((g->ymaxbox - g->yminbox) / g->dxbox);
    g->nzbox = (int32_t)((g->zmaxbox - g->zminbox) / g->dxbox);
    g->dybox = (g->ymaxbox - g->yminbox) / (double)g->nybox;
    g->dzbox = (g->zmaxbox - g->zminbox) / (double)g->nzbox;
    g->nbox = g->nxbox * g->nybox * g->nzbox;
}

/* collision_box_connectivity.f90:42-322 (NPROC=1: y and z always wrap). */
void orc_box_connectivity(const orc_boxgrid *g, int32_t periodicity, int32_t *ncon, int32_t *con) {
    const int NXB = g->nxbox, NYB = g->nybox, NZB = g->nzbox;
#define BOX(i, j, k) ((i) + ((j)-1) * NXB + ((k)-1) * NXB * NYB)
    for (int i0 = 1; i0 <= NXB; ++i0)
        for (int j0 = 1; j0 <= NYB; ++j0)
            for (int k0 = 1; k0 <= NZB; ++k0) {
                int ijk = BOX(i0, j0, k0);
                int im1 = i0 - 1, ip1 = i0 + 1, jm1 = j0 - 1, jp1 = j0 + 1, km1 = k0 - 1, kp1 = k0 + 1;
                if (im1 < 1 && periodicity) im1 = NXB;
                if (ip1 > NXB && periodicity) ip1 = 1;
                if (jm1 < 1) jm1 = NYB;
                if (jp1 > NYB) jp1 = 1;
                if (km1 < 1) km1 = NZB;
                if (kp1 > NZB) kp1 = 1;
                int nn = 0;
                int32_t *c = con + (int64_t)(ijk - 1) * 27;
                if (km1 >= 1) {
                    if (jp1 <= NYB) {
                        if (ip1 <= NXB) c[nn++] = BOX(ip1, jp1, km1);          /* box 9 */
                    }
                }
                if (jm1 >= 1) {
                    if (ip1 <= NXB) c[nn++] = BOX(ip1, jm1, k0);               /* box 12 */
                }
                if (ip1 <= NXB) c[nn++] = BOX(ip1, j0, k0);                    /* box 15 */
                if (jp1 <= NYB) {
                    c[nn++] = BOX(i0, jp1, k0);                                 /* box 17 */
                    if (ip1 <= NXB) c[nn++] = BOX(ip1, jp1, k0);               /* box 18 */
                }
                if (kp1 <= NZB) {
                    if (jm1 >= 1) {
                        c[nn++] = BOX(i0, jm1, kp1);                            /* box 20 */
                        if (ip1 <= NXB) c[nn++] = BOX(ip1, jm1, kp1);          /* box 21 */
                    }
                    if (im1 >= 1) c[nn++] = BOX(im1, j0, kp1);                 /* box 22 */
                    c[nn++] = BOX(i0, j0, kp1);                                 /* box 23 */
                    if (ip1 <= NXB) c[nn++] = BOX(ip1, j0, kp1);               /* box 24 */
                    if (jp1 <= NYB) {
                        if (im1 >= 1) c[nn++] = BOX(im1, jp1, kp1);            /* box 25 */
                        c[nn++] = BOX(i0, jp1, kp1);                            /* box 26 */
                        if (ip1 <= NXB) c[nn++] = BOX(ip1, jp1, kp1);          /* box 27 */
                    }
                }
                for (int t = nn; t < 27; ++t) c[t] = 0;
                ncon[ijk - 1] = nn;
            }
#undef BOX
}

/* collision_detection_connectivity.f90:74-89 */
int orc_box_index(const orc_boxgrid *g, int64_t n, const double *x, const double *y,
                  const double *z, int32_t *ijk, int64_t *err_id) {
    int rc = ORC_OK;
    if (err_id) *err_id = -1;
    for (int64_t np = 0; np < n; ++np) {
        int i0 = (int)((x[np] - g->xminbox) / g->dxbox) + 1;
        int j0 = (int)((y[np] - g->yminbox) / g->dybox) + 1;
        int k0 = (int)((z[np] - g->zminbox) / g->dzbox) + 1;
        if (i0 < 1 || i0 > g->nxbox || j0 < 1 || j0 > g->nybox || k0 < 1 || k0 > g->nzbox) {
            if (rc == ORC_OK && err_id) *err_id = np;
            rc = ORC_EOUT_OF_GRID;
            ijk[np] = 0;
            continue;
        }
        ijk[np] = i0 + (j0 - 1) * g->nxbox + (k0 - 1) * g->nxbox * g->nybox;
    }
    return rc;
}

/* Box membership lists in ascending particle index (PARTBOX,
 * collision_detection_connectivity.f90:101-118). start has nbox+1 entries. */
static int build_box_lists(const orc_boxgrid *g, int64_t n, const int32_t *ijk,
                           int64_t **start_out, int32_t **list_out) {
    int64_t *start = (int64_t *)calloc((size_t)g->nbox + 1, sizeof(int64_t));
    int32_t *list = (int32_t *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int32_t));
    if (!start || !list) { free(start); free(list); return -1; }
    for (int64_t i = 0; i < n; ++i) start[ijk[i]]++;          /* ijk is 1-based */
    for (int64_t b = 1; b <= g->nbox; ++b) start[b] += start[b - 1];
    int64_t *fill = (int64_t *)malloc((size_t)g->nbox * sizeof(int64_t));
    if (!fill) { free(start); free(list); return -1; }
    memcpy(fill, start, (size_t)g->nbox * sizeof(int64_t));
    for (int64_t i = 0; i < n; ++i) list[fill[ijk[i] - 1]++] = (int32_t)i;
    free(fill);
    *start_out = start;
    *list_out = list;
    return 0;
}

/* collision_detection_connectivity.f90:145-210 */
int64_t orc_detect_pairs(const orc_boxgrid *g, const int32_t *ncon, const int32_t *con,
                         int64_t n, const double *x, const double *y, const double *z,
                         int64_t cap, int32_t *home, int32_t *near) {
    int32_t *ijk = (int32_t *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int32_t));
    if (!ijk) return -1;
    int64_t eid;
    if (orc_box_index(g, n, x, y, z, ijk, &eid)) { free(ijk); return -1; }
    int64_t *start; int32_t *list;
    if (build_box_lists(g, n, ijk, &start, &list)) { free(ijk); return -1; }
    int64_t np0 = 0;
    for (int64_t b = 0; b < g->nbox; ++b) {
        int64_t s0 = start[b], s1 = start[b + 1];
        if (s1 == s0) continue;
        for (int64_t a = s0; a < s1; ++a) {
            for (int64_t c = a + 1; c < s1; ++c) {
                if (home && np0 < cap) { home[np0] = list[a]; near[np0] = list[c]; }
                np0++;
            }
            for (int nv = 0; nv < ncon[b]; ++nv) {
                int64_t nb = con[b * 27 + nv] - 1;
                for (int64_t c = start[nb]; c < start[nb + 1]; ++c) {
                    if (home && np0 < cap) { home[np0] = list[a]; near[np0] = list[c]; }
                    np0++;
                }
            }
        }
    }
    free(ijk); free(start); free(list);
    return np0;
}

/* ------------------------------------------------------------------------- */
/* Levenberg-Marquardt (MINPACK lmder, Moré 1978; MINPACK-1 user guide ANL-80-74), */
/* restated for the fixed problem size n=2 variables, m=3 residuals used by       */
/* ellipsoid_contact_detection.f90:92 through lmder1 (minpack_reduc.f90:652-757):  */
/* ftol=xtol=tol, gtol=0, maxfev=100*(n+1), mode=1, factor=100.                    */
/* ------------------------------------------------------------------------- */

#define LM_N 2
#define LM_M 3

double orc_enorm(int32_t n, const double *x) {
    /* Euclidean norm with the three-accumulator scaling of MINPACK's enorm
     * (minpack_reduc.f90:180-232): rdwarf=3.834e-20, rgiant=1.304e19. */
    const double rdwarf = 3.834e-20, rgiant = 1.304e19;
    double s1 = 0.0, s2 = 0.0, s3 = 0.0, x1max = 0.0, x3max = 0.0;
    double agiant = rgiant / (double)n;
    for (int i = 0; i < n; ++i) {
        double xabs = fabs(x[i]);
        if (xabs > rdwarf && xabs < agiant) {
            s2 = s2 + xabs * xabs;
        } else if (xabs <= rdwarf) {
            if (xabs <= x3max) {
                if (xabs != 0.0) { double r = xabs / x3max; s3 = s3 + r * r; }
            } else {
                double r = x3max / xabs;
                s3 = 1.0 + s3 * (r * r);
                x3max = xabs;
            }
        } else if (xabs <= x1max) {
            double r = xabs / x1max;
            s1 = s1 + r * r;
        } else {
            double r = x1max / xabs;
            s1 = 1.0 + s1 * (r * r);
            x1max = xabs;
        }
    }
    if (s1 != 0.0) return x1max * sqrt(s1 + (s2 / x1max) / x1max);
    if (s2 == 0.0) return x3max * sqrt(s3);
    if (s2 >= x3max) return sqrt(s2 * (1.0 + (x3max / s2) * (x3max * s3)));
    return sqrt(x3max * ((s2 / x3max) + (x3max * s3)));
}

/* ------------------------------------------------------------------------- */
/* Trigonometric functions of the contact solve.  The reference calls libm's     */
/* sin/cos/asin/acos there; this oracle and the CUDA kernels both use the       */
/* functions below (same constants, same operation order, no contraction), so    */
/* the Levenberg-Marquardt iterates of the two agree bit for bit.  The contact   */
/* solve only resolves its angles to xtol = sqrt(eps), far above the one-ulp     */
/* differences between these functions and any libm.                             */
/* ------------------------------------------------------------------------- */
#define CT_QUAL static inline
CT_QUAL double ct_poly_sin(double z) {
  double p = 1.9572941063391263e-20;
  p = p * z + -8.22063524662433e-18;
  p = p * z + 2.8114572543455206e-15;
  p = p * z + -7.647163731819816e-13;
  p = p * z + 1.6059043836821613e-10;
  p = p * z + -2.505210838544172e-08;
  p = p * z + 2.7557319223985893e-06;
  p = p * z + -0.0001984126984126984;
  p = p * z + 0.008333333333333333;
  p = p * z + -0.16666666666666666;
  return p;
}

CT_QUAL double ct_poly_cos(double z) {
  double p = 4.110317623312165e-19;
  p = p * z + -1.5619206968586225e-16;
  p = p * z + 4.779477332387385e-14;
  p = p * z + -1.1470745597729725e-11;
  p = p * z + 2.08767569878681e-09;
  p = p * z + -2.755731922398589e-07;
  p = p * z + 2.48015873015873e-05;
  p = p * z + -0.001388888888888889;
  p = p * z + 0.041666666666666664;
  return p;
}

/* sin and cos of x: Cody-Waite reduction by pi/2 = P1 + P2 + P3 (33 + 33 + 53 bits, so
 * k*P1 and k*P2 are exact for |k| < 2^20; the three parts are fdlibm's published
 * pio2_1, pio2_2 and pio2_2t, e_rem_pio2.c), Taylor polynomials (coefficients 1/n!) on
 * [-pi/4, pi/4]. */
CT_QUAL void ct_sincos(double x, double *s, double *c) {
  if (!(fabs(x) < 1.0e9)) {
    *s = x - x + (0.0 / 0.0 + x * 0.0);
    *c = *s;
    return;
  }
  const double k = rint(x * 0.6366197723675814);
  const double r = ((x - k * 1.5707963267341256) - k * 6.077100506303966e-11) - k * 2.0222662487959506e-21;
  const double z = r * r;
  const double sn = r + r * z * ct_poly_sin(z);
  const double cs = 1.0 + z * (-0.5 + z * ct_poly_cos(z));
  switch ((long long)k & 3) {
    case 0: *s = sn; *c = cs; break;
    case 1: *s = cs; *c = -sn; break;
    case 2: *s = -sn; *c = -cs; break;
    default: *s = -cs; *c = sn; break;
  }
}

CT_QUAL double ct_cos(double x) {
  double s, c;
  ct_sincos(x, &s, &c);
  return c;
}

/* asin on |x| <= 1/2 by its Taylor series x + sum_k C(2k,k)/(4^k (2k+1)) x^(2k+1) */
CT_QUAL double ct_asin_small(double x) {
  const double z = x * x;
  double p = 0.0020776610325181676;
  p = p * z + 0.0022014739737101384;
  p = p * z + 0.002338091892111975;
  p = p * z + 0.0024894486782468836;
  p = p * z + 0.00265787063820729;
  p = p * z + 0.002846178401108942;
  p = p * z + 0.0030578216492580306;
  p = p * z + 0.003297059503473485;
  p = p * z + 0.0035692053938259347;
  p = p * z + 0.003880964558837669;
  p = p * z + 0.004240907093679363;
  p = p * z + 0.004660143486915096;
  p = p * z + 0.005153309682319905;
  p = p * z + 0.005740037670841924;
  p = p * z + 0.006447210311889649;
  p = p * z + 0.0073125258735988454;
  p = p * z + 0.008390335809616815;
  p = p * z + 0.009761609529194078;
  p = p * z + 0.011551800896139705;
  p = p * z + 0.01396484375;
  p = p * z + 0.017352764423076924;
  p = p * z + 0.022372159090909092;
  p = p * z + 0.030381944444444444;
  p = p * z + 0.044642857142857144;
  p = p * z + 0.075;
  p = p * z + 0.16666666666666666;
  return x + x * z * p;
}

/* asin(x) = pi/2 - 2 asin(sqrt((1-|x|)/2)) for |x| > 1/2; NaN outside [-1, 1] */
CT_QUAL double ct_asin(double x) {
  const double ax = fabs(x);
  if (!(ax <= 1.0)) return (x - x) / (x - x) + x;
  double r;
  if (ax <= 0.5) {
    r = ct_asin_small(ax);
  } else {
    const double t = sqrt((1.0 - ax) * 0.5);
    r = (1.5707963267948966 - 2.0 * ct_asin_small(t)) + 6.123233995736766e-17;
  }
  return copysign(r, x);
}

CT_QUAL double ct_acos(double x) { return (1.5707963267948966 - ct_asin(x)) + 6.123233995736766e-17; }

#ifdef ORC_LIBM_TRIG
/* The reference's own trigonometry in the contact solve (libm sin, cos, asin, acos;
 * ellipsoid_contact_detection.f90:77-87,193-334).  Built as a second library, it measures
 * how often the shared functions above change a contact decision. */
#define ct_sincos(x, s, c) (*(s) = sin(x), *(c) = cos(x))
#define ct_cos cos
#define ct_asin asin
#define ct_acos acos
#endif

typedef struct {
    double e1[9], e2[9];     /* rotated ellipsoid matrices (calculate_ellipsoid_matrix.f90) */
    double b1[3], b2[3];
} contact_prob;

static void ellipsoid_matrix(double emaj, double apr, const double q[4], double e[9]) {
    /* calculate_ellipsoid_matrix.f90:33-72: R*diag(a^2,b^2,c^2)*R^T */
    double a = emaj, b = a / apr, c = b;
    memset(e, 0, 9 * sizeof(double));
    M3(e, 0, 0) = a * a;
    M3(e, 1, 1) = b * b;
    M3(e, 2, 2) = c * c;
    orc_transform_tensor(e, q);
}

/* pair_depth / fcn geometry: ellipsoid_pair_depth.f90:117-142, ellipsoid_contact_detection.f90:249-287 */
static void contact_points(const contact_prob *P, const double x[2], double c1[3],
                           double tmp1[3], double tmp2[3], double *lam1, double *lam2,
                           double pt1[3], double pt2[3]) {
    double s0, k0, s1, k1;
    ct_sincos(x[0], &s0, &k0);
    ct_sincos(x[1], &s1, &k1);
    c1[0] = k0 * k1;
    c1[1] = s0 * k1;
    c1[2] = s1;
    double c2[3] = {-c1[0], -c1[1], -c1[2]};
    matvec3(P->e1, c1, tmp1);
    matvec3(P->e2, c2, tmp2);
    double l1 = 0.25 * (c1[0] * tmp1[0] + c1[1] * tmp1[1] + c1[2] * tmp1[2]);
    l1 = sqrt(l1);
    double l2 = 0.25 * (c2[0] * tmp2[0] + c2[1] * tmp2[1] + c2[2] * tmp2[2]);
    l2 = sqrt(l2);
    for (int i = 0; i < 3; ++i) pt1[i] = (1.0 / (2.0 * l1)) * tmp1[i] + P->b1[i];
    for (int i = 0; i < 3; ++i) pt2[i] = (1.0 / (2.0 * l2)) * tmp2[i] + P->b2[i];
    *lam1 = l1; *lam2 = l2;
}

/* fcn with iflag=1: fvec = depth.*depth (ellipsoid_contact_detection.f90:290-295) */
static void fcn_f(const contact_prob *P, const double x[2], double fvec[3]) {
    double c1[3], t1[3], t2[3], l1, l2, pt1[3], pt2[3];
    contact_points(P, x, c1, t1, t2, &l1, &l2, pt1, pt2);
    for (int i = 0; i < 3; ++i) { double d = pt1[i] - pt2[i]; fvec[i] = d * d; }
}

/* grad of contact point: (1/(2l))E - (1/(8 l^3)) E c c^T E  (ellipsoid_contact_detection.f90:309-318) */
static void grad_coeff(const double e[9], const double c[3], double l, double coeff[9]) {
    double row[3];   /* c^T E */
    for (int j = 0; j < 3; ++j) row[j] = c[0] * M3(e, 0, j) + c[1] * M3(e, 1, j) + c[2] * M3(e, 2, j);
    double outer[9];
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) M3(outer, i, j) = c[i] * row[j];
    double eo[9];
    matmul33(e, outer, eo);
    double s = 1.0 / (2.0 * l), t = 1.0 / (8.0 * (l * l * l));   /* lambda**3.0 */
    for (int k = 0; k < 9; ++k) coeff[k] = s * e[k] - t * eo[k];
}

/* fcn with iflag=2: analytic Jacobian (ellipsoid_contact_detection.f90:296-332).
 * fjac column-major 3x2. */
static void fcn_j(const contact_prob *P, const double x[2], double fjac[6]) {
    double c1[3], t1[3], t2[3], l1, l2, pt1[3], pt2[3];
    contact_points(P, x, c1, t1, t2, &l1, &l2, pt1, pt2);
    double depth[3] = {pt1[0] - pt2[0], pt1[1] - pt2[1], pt1[2] - pt2[2]};
    double g[6];   /* Grad_cvec 3x2 */
    double s0, k0, s1, k1;
    ct_sincos(x[0], &s0, &k0);
    ct_sincos(x[1], &s1, &k1);
    g[0] = -s0 * k1;
    g[1] = k0 * k1;
    g[2] = 0.0;
    g[3] = -k0 * s1;
    g[4] = -s0 * s1;
    g[5] = k1;
    double c2[3] = {-c1[0], -c1[1], -c1[2]};
    double co1[9], co2[9];
    grad_coeff(P->e1, c1, l1, co1);
    grad_coeff(P->e2, c2, l2, co2);
    for (int j = 0; j < 2; ++j) {
        const double *gj = g + 3 * j;
        double ng[3] = {-gj[0], -gj[1], -gj[2]};
        double gp1[3], gp2[3];
        matvec3(co1, gj, gp1);
        matvec3(co2, ng, gp2);
        for (int i = 0; i < 3; ++i) {
            double gd = gp1[i] - gp2[i];
            fjac[i + 3 * j] = 2.0 * (depth[i] * gd);
        }
    }
}

/* QR with column pivoting by Householder reflections (MINPACK qrfac). a is 3x2
 * column-major and is overwritten with the reflection vectors / R off-diagonal. */
static void lm_qrfac(double a[6], int ipvt[2], double rdiag[2], double acnorm[2]) {
    const double epsmch = DBL_EPSILON;
    double wa[2];
    for (int j = 0; j < LM_N; ++j) {
        acnorm[j] = orc_enorm(LM_M, a + 3 * j);
        rdiag[j] = acnorm[j];
        wa[j] = rdiag[j];
        ipvt[j] = j;
    }
    for (int j = 0; j < LM_N; ++j) {   /* min(m,n) = 2 */
        int kmax = j;
        for (int k = j; k < LM_N; ++k)
            if (rdiag[k] > rdiag[kmax]) kmax = k;
        if (kmax != j) {
            for (int i = 0; i < LM_M; ++i) { double t = a[i + 3 * j]; a[i + 3 * j] = a[i + 3 * kmax]; a[i + 3 * kmax] = t; }
            rdiag[kmax] = rdiag[j];
            wa[kmax] = wa[j];
            int k = ipvt[j]; ipvt[j] = ipvt[kmax]; ipvt[kmax] = k;
        }
        double ajnorm = orc_enorm(LM_M - j, a + j + 3 * j);
        if (ajnorm != 0.0) {
            if (a[j + 3 * j] < 0.0) ajnorm = -ajnorm;
            for (int i = j; i < LM_M; ++i) a[i + 3 * j] = a[i + 3 * j] / ajnorm;
            a[j + 3 * j] = a[j + 3 * j] + 1.0;
            for (int k = j + 1; k < LM_N; ++k) {
                double sum = 0.0;
                for (int i = j; i < LM_M; ++i) sum = sum + a[i + 3 * j] * a[i + 3 * k];
                double temp = sum / a[j + 3 * j];
                for (int i = j; i < LM_M; ++i) a[i + 3 * k] = a[i + 3 * k] - temp * a[i + 3 * j];
                if (rdiag[k] != 0.0) {
                    temp = a[j + 3 * k] / rdiag[k];
                    double f = 1.0 - temp * temp;
                    rdiag[k] = rdiag[k] * sqrt(f > 0.0 ? f : 0.0);
                    double r = rdiag[k] / wa[k];
                    if (0.05 * (r * r) <= epsmch) {
                        rdiag[k] = orc_enorm(LM_M - j - 1, a + (j + 1) + 3 * k);
                        wa[k] = rdiag[k];
                    }
                }
            }
        }
        rdiag[j] = -ajnorm;
    }
}

/* Least-squares solve of [R; sqrt(par) D] x ~ [qtb; 0] by Givens rotations
 * (MINPACK qrsolv).  r is 2x2 column-major with leading dimension 3 (the fjac array). */
static void lm_qrsolv(double r[6], const int ipvt[2], const double diag[2], const double qtb[2],
                      double x[2], double sdiag[2]) {
    double wa[2];
    for (int j = 0; j < LM_N; ++j) {
        for (int i = j; i < LM_N; ++i) r[i + 3 * j] = r[j + 3 * i];
        x[j] = r[j + 3 * j];
        wa[j] = qtb[j];
    }
    for (int j = 0; j < LM_N; ++j) {
        int l = ipvt[j];
        if (diag[l] != 0.0) {
            for (int k = j; k < LM_N; ++k) sdiag[k] = 0.0;
            sdiag[j] = diag[l];
            double qtbpj = 0.0;
            for (int k = j; k < LM_N; ++k) {
                if (sdiag[k] == 0.0) continue;
                double cs, sn;
                if (fabs(r[k + 3 * k]) >= fabs(sdiag[k])) {
                    double tn = sdiag[k] / r[k + 3 * k];
                    cs = 0.5 / sqrt(0.25 + 0.25 * (tn * tn));
                    sn = cs * tn;
                } else {
                    double ct = r[k + 3 * k] / sdiag[k];
                    sn = 0.5 / sqrt(0.25 + 0.25 * (ct * ct));
                    cs = sn * ct;
                }
                r[k + 3 * k] = cs * r[k + 3 * k] + sn * sdiag[k];
                double temp = cs * wa[k] + sn * qtbpj;
                qtbpj = -sn * wa[k] + cs * qtbpj;
                wa[k] = temp;
                for (int i = k + 1; i < LM_N; ++i) {
                    temp = cs * r[i + 3 * k] + sn * sdiag[i];
                    sdiag[i] = -sn * r[i + 3 * k] + cs * sdiag[i];
                    r[i + 3 * k] = temp;
                }
            }
        }
        sdiag[j] = r[j + 3 * j];
        r[j + 3 * j] = x[j];
    }
    int nsing = LM_N;
    for (int j = 0; j < LM_N; ++j) {
        if (sdiag[j] == 0.0 && nsing == LM_N) nsing = j;
        if (nsing < LM_N) wa[j] = 0.0;
    }
    for (int k = 0; k < nsing; ++k) {
        int j = nsing - k - 1;
        double sum = 0.0;
        for (int i = j + 1; i < nsing; ++i) sum = sum + r[i + 3 * j] * wa[i];
        wa[j] = (wa[j] - sum) / sdiag[j];
    }
    for (int j = 0; j < LM_N; ++j) x[ipvt[j]] = wa[j];
}

/* Levenberg-Marquardt parameter (MINPACK lmpar): at most 10 iterations. */
static void lm_lmpar(double r[6], const int ipvt[2], const double diag[2], const double qtb[2],
                     double delta, double *par, double x[2], double sdiag[2]) {
    const double dwarf = DBL_MIN;
    double wa1[2], wa2[2];
    int nsing = LM_N;
    for (int j = 0; j < LM_N; ++j) {
        wa1[j] = qtb[j];
        if (r[j + 3 * j] == 0.0 && nsing == LM_N) nsing = j;
        if (nsing < LM_N) wa1[j] = 0.0;
    }
    for (int k = 0; k < nsing; ++k) {
        int j = nsing - k - 1;
        wa1[j] = wa1[j] / r[j + 3 * j];
        double temp = wa1[j];
        for (int i = 0; i < j; ++i) wa1[i] = wa1[i] - r[i + 3 * j] * temp;
    }
    for (int j = 0; j < LM_N; ++j) x[ipvt[j]] = wa1[j];
    int iter = 0;
    for (int j = 0; j < LM_N; ++j) wa2[j] = diag[j] * x[j];
    double dxnorm = orc_enorm(LM_N, wa2);
    double fp = dxnorm - delta;
    if (fp <= 0.1 * delta) {
        *par = 0.0;   /* iter == 0 */
        return;
    }
    double parl = 0.0;
    if (nsing >= LM_N) {
        for (int j = 0; j < LM_N; ++j) { int l = ipvt[j]; wa1[j] = diag[l] * (wa2[l] / dxnorm); }
        for (int j = 0; j < LM_N; ++j) {
            double sum = 0.0;
            for (int i = 0; i < j; ++i) sum = sum + r[i + 3 * j] * wa1[i];
            wa1[j] = (wa1[j] - sum) / r[j + 3 * j];
        }
        double temp = orc_enorm(LM_N, wa1);
        parl = ((fp / delta) / temp) / temp;
    }
    for (int j = 0; j < LM_N; ++j) {
        double sum = 0.0;
        for (int i = 0; i <= j; ++i) sum = sum + r[i + 3 * j] * qtb[i];
        wa1[j] = sum / diag[ipvt[j]];
    }
    double gnorm = orc_enorm(LM_N, wa1);
    double paru = gnorm / delta;
    if (paru == 0.0) paru = dwarf / (delta < 0.1 ? delta : 0.1);
    double p = *par;
    p = (p > parl) ? p : parl;
    p = (p < paru) ? p : paru;
    if (p == 0.0) p = gnorm / dxnorm;
    for (;;) {
        iter = iter + 1;
        if (p == 0.0) { double t = 0.001 * paru; p = (dwarf > t) ? dwarf : t; }
        double temp = sqrt(p);
        for (int j = 0; j < LM_N; ++j) wa1[j] = temp * diag[j];
        lm_qrsolv(r, ipvt, wa1, qtb, x, sdiag);
        for (int j = 0; j < LM_N; ++j) wa2[j] = diag[j] * x[j];
        dxnorm = orc_enorm(LM_N, wa2);
        temp = fp;
        fp = dxnorm - delta;
        if (fabs(fp) <= 0.1 * delta || (parl == 0.0 && fp <= temp && temp < 0.0) || iter == 10) break;
        for (int j = 0; j < LM_N; ++j) { int l = ipvt[j]; wa1[j] = diag[l] * (wa2[l] / dxnorm); }
        for (int j = 0; j < LM_N; ++j) {
            wa1[j] = wa1[j] / sdiag[j];
            temp = wa1[j];
            for (int i = j + 1; i < LM_N; ++i) wa1[i] = wa1[i] - r[i + 3 * j] * temp;
        }
        temp = orc_enorm(LM_N, wa1);
        double parc = ((fp / delta) / temp) / temp;
        if (fp > 0.0) parl = (parl > p) ? parl : p;
        if (fp < 0.0) paru = (paru < p) ? paru : p;
        double t2 = p + parc;
        p = (parl > t2) ? parl : t2;
    }
    *par = p;
}

/* lmder control loop (minpack_reduc.f90:243-640 control flow). Returns info (1..8, with
 * lmder1's mapping of 8 to 4). */
static int lm_lmder(const contact_prob *P, double x[2], double tol, int *nfev_out) {
    const double epsmch = DBL_EPSILON;
    const double ftol = tol, xtol = tol, gtol = 0.0, factor = 100.0;
    const int maxfev = 100 * (LM_N + 1);
    double fvec[3], fjac[6], diag[2], qtf[2], wa1[2], wa2[2], wa3[2], wa4[3];
    int ipvt[2];
    int info = 0, nfev, iter;
    double fnorm, par, xnorm = 0.0, delta = 0.0, temp = 0.0;
    fcn_f(P, x, fvec);
    nfev = 1;
    fnorm = orc_enorm(LM_M, fvec);
    par = 0.0;
    iter = 1;
    for (;;) {   /* outer */
        fcn_j(P, x, fjac);
        lm_qrfac(fjac, ipvt, wa1, wa2);   /* wa1 = rdiag, wa2 = acnorm */
        if (iter == 1) {
            for (int j = 0; j < LM_N; ++j) { diag[j] = wa2[j]; if (wa2[j] == 0.0) diag[j] = 1.0; }
            for (int j = 0; j < LM_N; ++j) wa3[j] = diag[j] * x[j];
            xnorm = orc_enorm(LM_N, wa3);
            delta = factor * xnorm;
            if (delta == 0.0) delta = factor;
        }
        for (int i = 0; i < LM_M; ++i) wa4[i] = fvec[i];
        for (int j = 0; j < LM_N; ++j) {
            if (fjac[j + 3 * j] != 0.0) {
                double sum = 0.0;
                for (int i = j; i < LM_M; ++i) sum = sum + fjac[i + 3 * j] * wa4[i];
                double t = -sum / fjac[j + 3 * j];
                for (int i = j; i < LM_M; ++i) wa4[i] = wa4[i] + fjac[i + 3 * j] * t;
            }
            fjac[j + 3 * j] = wa1[j];
            qtf[j] = wa4[j];
        }
        double gnorm = 0.0;
        if (fnorm != 0.0) {
            for (int j = 0; j < LM_N; ++j) {
                int l = ipvt[j];
                if (wa2[l] != 0.0) {
                    double sum = 0.0;
                    for (int i = 0; i <= j; ++i) sum = sum + fjac[i + 3 * j] * (qtf[i] / fnorm);
                    double g = fabs(sum / wa2[l]);
                    gnorm = (gnorm > g) ? gnorm : g;   /* max(gnorm, g) */
                }
            }
        }
        if (gnorm <= gtol) info = 4;
        if (info != 0) break;
        for (int j = 0; j < LM_N; ++j) diag[j] = (diag[j] > wa2[j]) ? diag[j] : wa2[j];
        for (;;) {   /* inner */
            lm_lmpar(fjac, ipvt, diag, qtf, delta, &par, wa1, wa2);
            for (int j = 0; j < LM_N; ++j) {
                wa1[j] = -wa1[j];
                wa2[j] = x[j] + wa1[j];
                wa3[j] = diag[j] * wa1[j];
            }
            double pnorm = orc_enorm(LM_N, wa3);
            if (iter == 1) delta = (delta < pnorm) ? delta : pnorm;
            fcn_f(P, wa2, wa4);
            nfev = nfev + 1;
            double fnorm1 = orc_enorm(LM_M, wa4);
            double actred = -1.0;
            if (0.1 * fnorm1 < fnorm) { double r = fnorm1 / fnorm; actred = 1.0 - r * r; }
            for (int j = 0; j < LM_N; ++j) {
                wa3[j] = 0.0;
                double t = wa1[ipvt[j]];
                for (int i = 0; i <= j; ++i) wa3[i] = wa3[i] + fjac[i + 3 * j] * t;
            }
            double temp1 = orc_enorm(LM_N, wa3) / fnorm;
            double temp2 = (sqrt(par) * pnorm) / fnorm;
            double prered = temp1 * temp1 + (temp2 * temp2) / 0.5;
            double dirder = -(temp1 * temp1 + temp2 * temp2);
            double ratio = 0.0;
            if (prered != 0.0) ratio = actred / prered;
            if (ratio <= 0.25) {
                if (actred >= 0.0) temp = 0.5;
                if (actred < 0.0) temp = 0.5 * dirder / (dirder + 0.5 * actred);
                if (0.1 * fnorm1 >= fnorm || temp < 0.1) temp = 0.1;
                double m = (delta < pnorm / 0.1) ? delta : pnorm / 0.1;
                delta = temp * m;
                par = par / temp;
            } else if (par == 0.0 || ratio >= 0.75) {
                delta = pnorm / 0.5;
                par = 0.5 * par;
            }
            if (ratio >= 1.0e-4) {
                for (int j = 0; j < LM_N; ++j) { x[j] = wa2[j]; wa2[j] = diag[j] * x[j]; }
                for (int i = 0; i < LM_M; ++i) fvec[i] = wa4[i];
                xnorm = orc_enorm(LM_N, wa2);
                fnorm = fnorm1;
                iter = iter + 1;
            }
            if (fabs(actred) <= ftol && prered <= ftol && 0.5 * ratio <= 1.0) info = 1;
            if (delta <= xtol * xnorm) info = 2;
            if (fabs(actred) <= ftol && prered <= ftol && 0.5 * ratio <= 1.0 && info == 2) info = 3;
            if (info != 0) goto done;
            if (nfev >= maxfev) info = 5;
            if (fabs(actred) <= epsmch && prered <= epsmch && 0.5 * ratio <= 1.0) info = 6;
            if (delta <= epsmch * xnorm) info = 7;
            if (gnorm <= epsmch) info = 8;
            if (info != 0) goto done;
            if (ratio >= 1.0e-4) break;
        }
    }
done:
    if (nfev_out) *nfev_out = nfev;
    if (info == 8) info = 4;   /* lmder1 (minpack_reduc.f90:754) */
    return info;
}

/* mod_particle_parallel.f90:145-201 */
double orc_fmargin(double emaj, double apr, const double point[3], const double center[3],
                   const double q[4]) {
    double ell[9];
    inv_ellipsoid_matrix(emaj, apr, q, ell);
    double vec[3] = {point[0] - center[0], point[1] - center[1], point[2] - center[2]};
    double e_[3];
    matvec3(ell, vec, e_);
    return vec[0] * e_[0] + vec[1] * e_[1] + vec[2] * e_[2];
}

/* ellipsoid_contact_detection.f90:1-187.  When the initial angle guess is NaN
 * (acos of a ratio just above 1, :86-87) every LM iterate stays NaN and the
 * reference reports no contact after exhausting maxfev; that result is returned
 * directly. */
int32_t orc_contact_detection(double emaj1, double apr1, double emaj2, double apr2,
                              const double b1[3], const double q1[4],
                              const double b2[3], const double q2[4],
                              double ept1[3], double ept2[3], double cnormal[3],
                              double x_out[2], int32_t *info_out, int32_t *nfev_out) {
    const double tol = sqrt(DBL_EPSILON);
    double cn[3] = {b1[0] - b2[0], b1[1] - b2[1], b1[2] - b2[2]};
    double c_norm = sqrt(cn[0] * cn[0] + cn[1] * cn[1] + cn[2] * cn[2]);
    if (c_norm != 0.0) { cn[0] = cn[0] / c_norm; cn[1] = cn[1] / c_norm; cn[2] = cn[2] / c_norm; }
    double x[2];
    x[1] = ct_asin(cn[2]);
    x[0] = ct_acos(cn[0] / ct_cos(x[1]));
    contact_prob P;
    ellipsoid_matrix(emaj1, apr1, q1, P.e1);
    ellipsoid_matrix(emaj2, apr2, q2, P.e2);
    for (int i = 0; i < 3; ++i) { P.b1[i] = b1[i]; P.b2[i] = b2[i]; }
    int info = 0, nfev = 0;
    if (x[0] != x[0] || x[1] != x[1]) {
        for (int i = 0; i < 3; ++i) { ept1[i] = NAN; ept2[i] = NAN; cnormal[i] = NAN; }
        if (x_out) { x_out[0] = NAN; x_out[1] = NAN; }
        if (info_out) *info_out = 5;
        if (nfev_out) *nfev_out = 100 * (LM_N + 1);
        return 0;
    }
    info = lm_lmder(&P, x, tol, &nfev);
    double c1[3], t1[3], t2[3], l1, l2, pt1[3], pt2[3];
    contact_points(&P, x, c1, t1, t2, &l1, &l2, pt1, pt2);   /* pair_depth */
    double depth[3] = {pt1[0] - pt2[0], pt1[1] - pt2[1], pt1[2] - pt2[2]};
    double contact = depth[0] * c1[0] + depth[1] * c1[1] + depth[2] * c1[2];
    int32_t flag = 0;
    if ((contact > 0) && (orc_fmargin(emaj1, apr1, pt2, b1, q1) < 1.0) &&
        (orc_fmargin(emaj2, apr2, pt1, b2, q2) < 1.0))
        flag = 1;
    for (int i = 0; i < 3; ++i) { ept1[i] = pt1[i]; ept2[i] = pt2[i]; cnormal[i] = c1[i]; }
    if (x_out) { x_out[0] = x[0]; x_out[1] = x[1]; }
    if (info_out) *info_out = info;
    if (nfev_out) *nfev_out = nfev;
    return flag;
}

/* collision_response.f90:1-437 (inertia of particle 1 used for both bodies, :140-145) */
int orc_collision_response(const orc_setup *s, double ipxx, double ipyy, double ipzz,
                           double u1[3], double o1[3], const double q1[4],
                           double u2[3], double o2[3], const double q2[4],
                           const double r1[3], const double r2[3], const double n[3]) {
    double up1[3] = {u1[0], u1[1], u1[2]}, up2[3] = {u2[0], u2[1], u2[2]};
    double om1[3] = {o1[0], o1[1], o1[2]}, om2[3] = {o2[0], o2[1], o2[2]};
    orc_transform_vec(om1, q1);
    orc_transform_vec(om2, q2);
    double upc1[3], upc2[3];
    upc1[0] = u1[0] + (om1[1] * r1[2] - om1[2] * r1[1]);
    upc1[1] = u1[1] + (om1[2] * r1[0] - om1[0] * r1[2]);
    upc1[2] = u1[2] + (om1[0] * r1[1] - om1[1] * r1[0]);
    upc2[0] = u2[0] + (om2[1] * r2[2] - om2[2] * r2[1]);
    upc2[1] = u2[1] + (om2[2] * r2[0] - om2[0] * r2[2]);
    upc2[2] = u2[2] + (om2[0] * r2[1] - om2[1] * r2[0]);
    double urel[3] = {upc2[0] - upc1[0], upc2[1] - upc1[1], upc2[2] - upc1[2]};
    double urn = urel[0] * n[0] + urel[1] * n[1] + urel[2] * n[2];
    double delu[3];
    for (int i = 0; i < 3; ++i) delu[i] = urel[i] + s->ecp * urn * n[i];
    double ip1[9] = {0}, ip2[9], inv1[9] = {0}, inv2[9] = {0};
    M3(ip1, 0, 0) = ipxx; M3(ip1, 1, 1) = ipyy; M3(ip1, 2, 2) = ipzz;
    memcpy(ip2, ip1, sizeof ip1);
    orc_transform_tensor(ip1, q1);
    orc_transform_tensor(ip2, q2);
    if (orc_invert3(ip1, inv1)) return ORC_ESINGULAR;
    if (orc_invert3(ip2, inv2)) return ORC_ESINGULAR;
    double rx1[9], rxt1[9], rx2[9], rxt2[9], t[9], k1[9], k2[9], k[9], invk[9];
    skew(r1, rx1); transpose33(rx1, rxt1);
    matmul33(inv1, rx1, t); matmul33(rxt1, t, t);
    for (int i = 0; i < 9; ++i) k1[i] = ((i % 4) == 0 ? 1.0 : 0.0) + t[i];
    skew(r2, rx2); transpose33(rx2, rxt2);
    matmul33(inv2, rx2, t); matmul33(rxt2, t, t);
    for (int i = 0; i < 9; ++i) k2[i] = ((i % 4) == 0 ? 1.0 : 0.0) + t[i];
    for (int i = 0; i < 9; ++i) k[i] = k1[i] + k2[i];
    if (orc_invert3(k, invk)) return ORC_ESINGULAR;
    double pc[3];
    matvec3(invk, delu, pc);
    pc[0] = -pc[0]; pc[1] = -pc[1]; pc[2] = -pc[2];
    double pcn = pc[0] * n[0] + pc[1] * n[1] + pc[2] * n[2];
    double px = pc[0] - pcn * n[0], py = pc[1] - pcn * n[1], pz = pc[2] - pcn * n[2];
    double pct = sqrt(px * px + py * py + pz * pz);
    if (pct > s->mup * pcn) {
        double tw[3] = {urel[0] - urn * n[0], urel[1] - urn * n[1], urel[2] - urn * n[2]};
        double nrm = sqrt(tw[0] * tw[0] + tw[1] * tw[1] + tw[2] * tw[2]);
        if (nrm != 0.0) { tw[0] = -tw[0] / nrm; tw[1] = -tw[1] / nrm; tw[2] = -tw[2] / nrm; }
        double vimp[3] = {n[0] + s->mup * tw[0], n[1] + s->mup * tw[1], n[2] + s->mup * tw[2]};
        double kn[3];
        matvec3(k, vimp, kn);
        double kn_dot_n = kn[0] * n[0] + kn[1] * n[1] + kn[2] * n[2];
        pcn = -1.0 * (delu[0] * n[0] + delu[1] * n[1] + delu[2] * n[2]);
        for (int i = 0; i < 3; ++i) pc[i] = (pcn / kn_dot_n) * vimp[i];
    }
    double am[3];
    double eit1 = 0.5 * (up1[0] * up1[0] + up1[1] * up1[1] + up1[2] * up1[2]);
    matvec3(ip1, om1, am);
    double eir1 = 0.5 * (om1[0] * am[0] + om1[1] * am[1] + om1[2] * am[2]);
    double ei1 = eit1 + eir1;
    double eit2 = 0.5 * (up2[0] * up2[0] + up2[1] * up2[1] + up2[2] * up2[2]);
    matvec3(ip2, om2, am);
    double eir2 = 0.5 * (om2[0] * am[0] + om2[1] * am[1] + om2[2] * am[2]);
    double ei2 = eit2 + eir2;
    double e_i = ei1 + ei2;
    u1[0] = u1[0] - pc[0]; u1[1] = u1[1] - pc[1]; u1[2] = u1[2] - pc[2];
    double mpc[3] = {-pc[0], -pc[1], -pc[2]}, tmp[3], dom[3];
    matvec3(rx1, mpc, tmp); matvec3(inv1, tmp, dom);
    for (int i = 0; i < 3; ++i) om1[i] = om1[i] + dom[i];
    u2[0] = u2[0] + pc[0]; u2[1] = u2[1] + pc[1]; u2[2] = u2[2] + pc[2];
    matvec3(rx2, pc, tmp); matvec3(inv2, tmp, dom);
    for (int i = 0; i < 3; ++i) om2[i] = om2[i] + dom[i];
    double eft1 = 0.5 * (u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]);
    matvec3(ip1, om1, am);
    double efr1 = 0.5 * (om1[0] * am[0] + om1[1] * am[1] + om1[2] * am[2]);
    double ef1 = eft1 + efr1;
    double eft2 = 0.5 * (u2[0] * u2[0] + u2[1] * u2[1] + u2[2] * u2[2]);
    matvec3(ip2, om2, am);
    double efr2 = 0.5 * (om2[0] * am[0] + om2[1] * am[1] + om2[2] * am[2]);
    double ef2 = eft2 + efr2;
    double e_f = ef1 + ef2;
    double cq[4];
    conjq(q1, cq); orc_transform_vec(om1, cq);
    conjq(q2, cq); orc_transform_vec(om2, cq);
    o1[0] = om1[0]; o1[1] = om1[1]; o1[2] = om1[2];
    o2[0] = om2[0]; o2[1] = om2[1]; o2[2] = om2[2];
    if (fabs((e_i - e_f) / e_i) > 1.0e-9) return ORC_EENERGY;   /* :408-436 */
    return ORC_OK;
}

/* ------------------------------------------------------------------------- */
/* COLLISION_INTERACTION                                                     */
/* ------------------------------------------------------------------------- */

static inline double bound_radius(double emaj, double apr) {
    double b = emaj / apr;
    return emaj > b ? emaj : b;
}

/* collision_interaction.f90:216-348 for one pair (HOME i1, NEAR i2). */
/* collision_interaction.f90:216-328; also returns NVREL and |v_rel| (NRM_VREL) of a
 * pair in contact, for the collision statistics (:330-345). */
static int32_t pair_eval_full(const orc_setup *s, const orc_props *p, const orc_state *st,
                              int64_t i1, int64_t i2, double ept1[3], double ept2[3],
                              double cn[3], double rx1[3], double rx2[3], int32_t *flag_out,
                              double *nvrel_out, double *nrm_out) {
    double xn = st->x[i1], yn = st->y[i1], zn = st->z[i1];
    double vkx = st->x[i2] - xn, vky = st->y[i2] - yn, vkz = st->z[i2] - zn;
    if ((fabs(vkx) > s->lx / 2) && s->periodicity) vkx = vkx - copysign(s->lx, vkx);
    if (fabs(vky) > s->ly / 2.) vky = vky - copysign(s->ly, vky);   /* NPROC==1 */
    if (fabs(vkz) > s->lz / 2.) vkz = vkz - copysign(s->lz, vkz);
    double b1[3] = {st->x[i1], st->y[i1], st->z[i1]};
    double b2[3] = {st->x[i1] + vkx, st->y[i1] + vky, st->z[i1] + vkz};
    double q1[4] = {st->qa[i1], st->qb[i1], st->qc[i1], st->qd[i1]};
    double q2[4] = {st->qa[i2], st->qb[i2], st->qc[i2], st->qd[i2]};
    int32_t flag = orc_contact_detection(p->emaj[i1], p->apr[i1], p->emaj[i2], p->apr[i2],
                                         b1, q1, b2, q2, ept1, ept2, cn, NULL, NULL, NULL);
    if (flag_out) *flag_out = flag;
    if (!flag) return 0;
    rx1[0] = (ept1[0] - st->x[i1]); rx1[1] = (ept1[1] - st->y[i1]); rx1[2] = (ept1[2] - st->z[i1]);
    double om1[3] = {st->ox[i1], st->oy[i1], st->oz[i1]};
    orc_transform_vec(om1, q1);
    double up1 = st->u[i1] + (om1[1] * rx1[2] - om1[2] * rx1[1]);
    double vp1 = st->v[i1] + (om1[2] * rx1[0] - om1[0] * rx1[2]);
    double wp1 = st->w[i1] + (om1[0] * rx1[1] - om1[1] * rx1[0]);
    rx2[0] = (ept2[0] - (st->x[i1] + vkx));
    rx2[1] = (ept2[1] - (st->y[i1] + vky));
    rx2[2] = (ept2[2] - (st->z[i1] + vkz));
    double om2[3] = {st->ox[i2], st->oy[i2], st->oz[i2]};
    orc_transform_vec(om2, q2);
    double up2 = st->u[i2] + (om2[1] * rx2[2] - om2[2] * rx2[1]);
    double vp2 = st->v[i2] + (om2[2] * rx2[0] - om2[0] * rx2[2]);
    double wp2 = st->w[i2] + (om2[0] * rx2[1] - om2[1] * rx2[0]);
    double vrelx = up2 - up1, vrely = vp2 - vp1, vrelz = wp2 - wp1;
    double nvrel = vrelx * cn[0] + vrely * cn[1] + vrelz * cn[2];
    if (nvrel_out) *nvrel_out = nvrel;
    if (nrm_out) *nrm_out = sqrt(vrelx * vrelx + vrely * vrely + vrelz * vrelz);
    return (nvrel < ZERO_REF) ? 1 : 0;
}

int32_t orc_pair_eval(const orc_setup *s, const orc_props *p, const orc_state *st,
                      int64_t i1, int64_t i2, double ept1[3], double ept2[3],
                      double cn[3], double rx1[3], double rx2[3], int32_t *flag_out) {
    return pair_eval_full(s, p, st, i1, i2, ept1, ept2, cn, rx1, rx2, flag_out, NULL, NULL);
}

static int prefilter_pass(const orc_setup *s, const orc_props *p, const orc_state *st,
                          int64_t i1, int64_t i2) {
    double vkx = st->x[i2] - st->x[i1], vky = st->y[i2] - st->y[i1], vkz = st->z[i2] - st->z[i1];
    if ((fabs(vkx) > s->lx / 2) && s->periodicity) vkx = vkx - copysign(s->lx, vkx);
    if (fabs(vky) > s->ly / 2.) vky = vky - copysign(s->ly, vky);
    if (fabs(vkz) > s->lz / 2.) vkz = vkz - copysign(s->lz, vkz);
    double rr = (bound_radius(p->emaj[i1], p->apr[i1]) + bound_radius(p->emaj[i2], p->apr[i2])) * (1.0 + 1e-9);
    return (vkx * vkx + vky * vky + vkz * vkz) <= rr * rr;
}

typedef struct {
    int64_t box;    /* IJK-1 */
    int32_t a_rank; /* position of HOME in its box list */
    int32_t slot;   /* 0 same box, 1+NV for neighbour boxes */
    int32_t c_rank; /* position of NEAR in its box list */
    int32_t home, near;
    double ept1[3], ept2[3], cn[3], rx1[3], rx2[3];
} coll_rec;

static int rec_cmp(const void *pa, const void *pb) {
    const coll_rec *a = (const coll_rec *)pa, *b = (const coll_rec *)pb;
    if (a->box != b->box) return a->box < b->box ? -1 : 1;
    if (a->a_rank != b->a_rank) return a->a_rank < b->a_rank ? -1 : 1;
    if (a->slot != b->slot) return a->slot < b->slot ? -1 : 1;
    if (a->c_rank != b->c_rank) return a->c_rank < b->c_rank ? -1 : 1;
    return 0;
}

static int apply_response(const orc_setup *s, const orc_props *p, orc_state *st, const coll_rec *r) {
    int64_t i1 = r->home, i2 = r->near;
    double u1[3] = {st->u[i1], st->v[i1], st->w[i1]}, o1[3] = {st->ox[i1], st->oy[i1], st->oz[i1]};
    double u2[3] = {st->u[i2], st->v[i2], st->w[i2]}, o2[3] = {st->ox[i2], st->oy[i2], st->oz[i2]};
    double q1[4] = {st->qa[i1], st->qb[i1], st->qc[i1], st->qd[i1]};
    double q2[4] = {st->qa[i2], st->qb[i2], st->qc[i2], st->qd[i2]};
    int rc = orc_collision_response(s, p->ipxx[i1], p->ipyy[i1], p->ipzz[i1], u1, o1, q1, u2, o2, q2,
                                    r->rx1, r->rx2, r->cn);
    st->u[i1] = u1[0]; st->v[i1] = u1[1]; st->w[i1] = u1[2];
    st->ox[i1] = o1[0]; st->oy[i1] = o1[1]; st->oz[i1] = o1[2];
    st->u[i2] = u2[0]; st->v[i2] = u2[1]; st->w[i2] = u2[2];
    st->ox[i2] = o2[0]; st->oy[i2] = o2[1]; st->oz[i2] = o2[2];
    return rc;
}

static int collision_impl(const orc_setup *s, const orc_props *p, const orc_boxgrid *g,
                          const int32_t *ncon, const int32_t *con, orc_state *st,
                          int32_t prefilter, int32_t nthreads,
                          int64_t coll_cap, int32_t *coll_home, int32_t *coll_near,
                          int64_t *n_coll, int64_t *n_candidates, int64_t *n_contacts,
                          int64_t *err_id, const int32_t *group, int32_t ngroups, double *colstat) {
    const int64_t n = st->n;
    if (colstat) nthreads = 1;   /* the statistics follow the serial walk */
    int rc_out = ORC_OK;
    if (err_id) *err_id = -1;
    int32_t *ijk = (int32_t *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int32_t));
    if (!ijk) return ORC_EBADARG;
    int64_t eid;
    if (orc_box_index(g, n, st->x, st->y, st->z, ijk, &eid)) {
        free(ijk);
        if (err_id) *err_id = eid;
        return ORC_EOUT_OF_GRID;
    }
    int64_t *start; int32_t *list;
    if (build_box_lists(g, n, ijk, &start, &list)) { free(ijk); return ORC_EBADARG; }
    int64_t ncand = 0, ncontact = 0, ncoll = 0;

    if (nthreads <= 1) {
        /* Faithful serial loop (collision_interaction.f90:190-419): pairs in list order,
         * evaluated only while both particles are uncoloured. */
        signed char *color = (signed char *)malloc((size_t)(n > 0 ? n : 1));
        memset(color, 1, (size_t)(n > 0 ? n : 1));
        for (int64_t b = 0; b < g->nbox; ++b) {
            int64_t s0 = start[b], s1 = start[b + 1];
            for (int64_t a = s0; a < s1; ++a) {
                int64_t i1 = list[a];
                for (int slot = 0; slot <= ncon[b]; ++slot) {
                    int64_t c0, c1;
                    if (slot == 0) { c0 = a + 1; c1 = s1; }
                    else { int64_t nb = con[b * 27 + slot - 1] - 1; c0 = start[nb]; c1 = start[nb + 1]; }
                    for (int64_t c = c0; c < c1; ++c) {
                        int64_t i2 = list[c];
                        ncand++;
                        if (!(color[i1] == 1 && color[i2] == 1)) continue;
                        if (prefilter && !prefilter_pass(s, p, st, i1, i2)) continue;
                        coll_rec r;
                        int32_t flag;
                        double nvrel = 0.0, nrm = 0.0;
                        int hit = pair_eval_full(s, p, st, i1, i2, r.ept1, r.ept2, r.cn, r.rx1, r.rx2, &flag,
                                                 &nvrel, &nrm);
                        ncontact += flag;
                        if (colstat && flag) {
                            /* collision_interaction.f90:330-345 and :397-398 */
                            int g1 = group ? group[i1] - 1 : 0, g2 = group ? group[i2] - 1 : 0;
                            double *a = colstat + ((int64_t)g1 * ngroups + g2) * 8;
                            double v0 = r.ept1[0] - r.ept2[0], v1 = r.ept1[1] - r.ept2[1], v2 = r.ept1[2] - r.ept2[2];
                            a[0] = a[0] + 1.0;
                            a[3] = a[3] + sqrt(v0 * v0 + v1 * v1 + v2 * v2);
                            a[5] = a[5] + nvrel;
                            a[6] = a[6] + nrm;
                            a[7] = a[7] + acos(nvrel / nrm);
                            if (hit) a[1] = a[1] + 1.0;
                        }
                        if (!hit) continue;
                        r.home = (int32_t)i1; r.near = (int32_t)i2;
                        int rc = apply_response(s, p, st, &r);
                        if (rc && rc_out == ORC_OK) { rc_out = rc; if (err_id) *err_id = i1; }
                        color[i1] = -1; color[i2] = -1;
                        if (coll_home && ncoll < coll_cap) { coll_home[ncoll] = r.home; coll_near[ncoll] = r.near; }
                        ncoll++;
                    }
                }
            }
        }
        free(color);
    } else {
        /* Parallel evaluation on the pre-collision state, then the same greedy
         * acceptance in list order.  Equivalent to the serial loop: a pair is only
         * ever evaluated while both particles are uncoloured, i.e. unmodified. */
        int nt = nthreads;
        coll_rec **bufs = (coll_rec **)calloc((size_t)nt, sizeof(coll_rec *));
        int64_t *lens = (int64_t *)calloc((size_t)nt, sizeof(int64_t));
        int64_t *caps = (int64_t *)calloc((size_t)nt, sizeof(int64_t));
        int64_t cand_tot = 0, contact_tot = 0;
#ifdef _OPENMP
#pragma omp parallel num_threads(nt) reduction(+ : cand_tot, contact_tot)
#endif
        {
#ifdef _OPENMP
            int tid = omp_get_thread_num();
#else
            int tid = 0;
#endif
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 64)
#endif
            for (int64_t b = 0; b < g->nbox; ++b) {
                int64_t s0 = start[b], s1 = start[b + 1];
                for (int64_t a = s0; a < s1; ++a) {
                    int64_t i1 = list[a];
                    for (int slot = 0; slot <= ncon[b]; ++slot) {
                        int64_t c0, c1, nb = b;
                        if (slot == 0) { c0 = a + 1; c1 = s1; }
                        else { nb = con[b * 27 + slot - 1] - 1; c0 = start[nb]; c1 = start[nb + 1]; }
                        for (int64_t c = c0; c < c1; ++c) {
                            int64_t i2 = list[c];
                            cand_tot++;
                            if (prefilter && !prefilter_pass(s, p, st, i1, i2)) continue;
                            coll_rec r;
                            int32_t flag;
                            int hit = orc_pair_eval(s, p, st, i1, i2, r.ept1, r.ept2, r.cn, r.rx1, r.rx2, &flag);
                            contact_tot += flag;
                            if (!hit) continue;
                            r.box = b; r.a_rank = (int32_t)(a - s0); r.slot = slot;
                            r.c_rank = (int32_t)(c - start[nb]);
                            r.home = (int32_t)i1; r.near = (int32_t)i2;
                            if (lens[tid] == caps[tid]) {
                                caps[tid] = caps[tid] ? 2 * caps[tid] : 1024;
                                bufs[tid] = (coll_rec *)realloc(bufs[tid], (size_t)caps[tid] * sizeof(coll_rec));
                            }
                            bufs[tid][lens[tid]++] = r;
                        }
                    }
                }
            }
        }
        ncand = cand_tot;
        ncontact = contact_tot;
        int64_t tot = 0;
        for (int t = 0; t < nt; ++t) tot += lens[t];
        coll_rec *all = (coll_rec *)malloc((size_t)(tot > 0 ? tot : 1) * sizeof(coll_rec));
        int64_t o = 0;
        for (int t = 0; t < nt; ++t) { if (lens[t]) memcpy(all + o, bufs[t], (size_t)lens[t] * sizeof(coll_rec)); o += lens[t]; free(bufs[t]); }
        free(bufs); free(lens); free(caps);
        qsort(all, (size_t)tot, sizeof(coll_rec), rec_cmp);
        signed char *color = (signed char *)malloc((size_t)(n > 0 ? n : 1));
        memset(color, 1, (size_t)(n > 0 ? n : 1));
        for (int64_t k = 0; k < tot; ++k) {
            coll_rec *r = &all[k];
            if (!(color[r->home] == 1 && color[r->near] == 1)) continue;
            int rc = apply_response(s, p, st, r);
            if (rc && rc_out == ORC_OK) { rc_out = rc; if (err_id) *err_id = r->home; }
            color[r->home] = -1; color[r->near] = -1;
            if (coll_home && ncoll < coll_cap) { coll_home[ncoll] = r->home; coll_near[ncoll] = r->near; }
            ncoll++;
        }
        free(color);
        free(all);
    }
    free(ijk); free(start); free(list);
    if (n_coll) *n_coll = ncoll;
    if (n_candidates) *n_candidates = ncand;
    if (n_contacts) *n_contacts = ncontact;
    return rc_out;
}

int orc_collision(const orc_setup *s, const orc_props *p, const orc_boxgrid *g,
                  const int32_t *ncon, const int32_t *con, orc_state *st,
                  int32_t prefilter, int32_t nthreads,
                  int64_t coll_cap, int32_t *coll_home, int32_t *coll_near,
                  int64_t *n_coll, int64_t *n_candidates, int64_t *n_contacts,
                  int64_t *err_id) {
    return collision_impl(s, p, g, ncon, con, st, prefilter, nthreads, coll_cap, coll_home, coll_near,
                          n_coll, n_candidates, n_contacts, err_id, NULL, 0, NULL);
}

int orc_collision_stats(const orc_setup *s, const orc_props *p, const orc_boxgrid *g,
                        const int32_t *ncon, const int32_t *con, orc_state *st, int32_t prefilter,
                        const int32_t *group, int32_t ngroups, double *colstat, int64_t *n_coll,
                        int64_t *err_id) {
    for (int64_t k = 0; k < (int64_t)ngroups * ngroups * 8; ++k) colstat[k] = 0.0;
    int rc = collision_impl(s, p, g, ncon, con, st, prefilter, 1, 0, NULL, NULL, n_coll, NULL, NULL,
                            err_id, group, ngroups, colstat);
    /* collision_interaction.f90:429-430 */
    for (int64_t k = 0; k < (int64_t)ngroups * ngroups; ++k) {
        double *a = colstat + k * 8;
        a[2] = 2.0 * a[1] / s->dtime;
        a[4] = a[3] / a[0];
    }
    return rc;
}

/* ---- exported pieces of the contact solve, for the scipy MINPACK cross-check ---- */
static void make_prob(double emaj1, double apr1, double emaj2, double apr2,
                      const double b1[3], const double q1[4], const double b2[3],
                      const double q2[4], contact_prob *P) {
    ellipsoid_matrix(emaj1, apr1, q1, P->e1);
    ellipsoid_matrix(emaj2, apr2, q2, P->e2);
    for (int i = 0; i < 3; ++i) { P->b1[i] = b1[i]; P->b2[i] = b2[i]; }
}

void orc_contact_residual(double emaj1, double apr1, double emaj2, double apr2,
                          const double b1[3], const double q1[4], const double b2[3],
                          const double q2[4], const double x[2], double fvec[3]) {
    contact_prob P;
    make_prob(emaj1, apr1, emaj2, apr2, b1, q1, b2, q2, &P);
    fcn_f(&P, x, fvec);
}

void orc_contact_jacobian(double emaj1, double apr1, double emaj2, double apr2,
                          const double b1[3], const double q1[4], const double b2[3],
                          const double q2[4], const double x[2], double fjac[6]) {
    contact_prob P;
    make_prob(emaj1, apr1, emaj2, apr2, b1, q1, b2, q2, &P);
    fcn_j(&P, x, fjac);
}

int32_t orc_contact_lm(double emaj1, double apr1, double emaj2, double apr2,
                       const double b1[3], const double q1[4], const double b2[3],
                       const double q2[4], double x[2], double tol, int32_t *nfev) {
    contact_prob P;
    make_prob(emaj1, apr1, emaj2, apr2, b1, q1, b2, q2, &P);
    int nf = 0;
    int info = lm_lmder(&P, x, tol, &nf);
    if (nfev) *nfev = nf;
    return info;
}
