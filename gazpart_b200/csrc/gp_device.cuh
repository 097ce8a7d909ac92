// gp_device.cuh -- per-particle and per-pair device routines of the frozen-flow
// ellipsoidal-particle step, FP64, register resident.
//
// Each routine restates the reference routine named beside it (paths relative to the
// reference's source/ directory) with the reference's evaluation order, so that the
// FP64 path agrees with an IEEE restatement to rounding.  3x3 matrices are column
// major: m[i + 3*j] = M(i+1, j+1).
#pragma once
#include <cstdint>
#include <cmath>

#include "gp_types.h"

namespace gp {

constexpr double kZeroRef = 1.0e-33;   // ZERO, mod_dns_dim.f90:136

struct Quat { double a, b, c, d; };

__host__ __device__ inline Quat conj(const Quat& q) { return {q.a, -q.b, -q.c, -q.d}; }

// R(q): transform_basis.f90:44-54 (same expressions in calculate_ellipsoid_matrix.f90:54-64
// and mod_particle_parallel.f90:176-186).
__host__ __device__ inline void rotmat(const Quat& q, double r[9]) {
  const double q0 = q.a, q1 = q.b, q2 = q.c, q3 = q.d;
  r[0] = 1.0 - 2.0 * (q2 * q2 + q3 * q3);
  r[3] = 2.0 * (q1 * q2 - q0 * q3);
  r[6] = 2.0 * (q1 * q3 + q0 * q2);
  r[1] = 2.0 * (q1 * q2 + q0 * q3);
  r[4] = 1.0 - 2.0 * (q1 * q1 + q3 * q3);
  r[7] = 2.0 * (q2 * q3 - q0 * q1);
  r[2] = 2.0 * (q1 * q3 - q0 * q2);
  r[5] = 2.0 * (q2 * q3 + q0 * q1);
  r[8] = 1.0 - 2.0 * (q1 * q1 + q2 * q2);
}

__host__ __device__ inline void matvec(const double m[9], const double v[3], double o[3]) {
  const double t0 = m[0] * v[0] + m[3] * v[1] + m[6] * v[2];
  const double t1 = m[1] * v[0] + m[4] * v[1] + m[7] * v[2];
  const double t2 = m[2] * v[0] + m[5] * v[1] + m[8] * v[2];
  o[0] = t0; o[1] = t1; o[2] = t2;
}

// transform_basis.f90:77 (vector case)
__host__ __device__ inline void rot_vec(const Quat& q, double v[3]) {
  double r[9];
  rotmat(q, r);
  matvec(r, v, v);
}

__host__ __device__ inline void matmul(const double a[9], const double b[9], double c[9]) {
  double t[9];
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int i = 0; i < 3; ++i)
      t[i + 3 * j] = a[i] * b[3 * j] + a[i + 3] * b[1 + 3 * j] + a[i + 6] * b[2 + 3 * j];
#pragma unroll
  for (int k = 0; k < 9; ++k) c[k] = t[k];
}

// transform_basis.f90:82 for a diagonal input: R*(diag(d)*R^T).  With the zero
// off-diagonal entries the inner product is exactly d_k*R(j,k).
__host__ __device__ inline void rot_diag(const Quat& q, double d0, double d1, double d2, double o[9]) {
  double r[9];
  rotmat(q, r);
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const double t0 = d0 * r[j], t1 = d1 * r[j + 3], t2 = d2 * r[j + 6];
#pragma unroll
    for (int i = 0; i < 3; ++i) o[i + 3 * j] = r[i] * t0 + r[i + 3] * t1 + r[i + 6] * t2;
  }
}

// invert_ndim3_matrix.f90:1-39.  Returns false where the reference stops.
__host__ __device__ inline bool invert3(const double m[9], double inv[9]) {
#define M(i, j) m[((i)-1) + 3 * ((j)-1)]
  const double detinv = 1.0 / (M(1, 1) * M(2, 2) * M(3, 3) - M(1, 1) * M(2, 3) * M(3, 2) -
                               M(1, 2) * M(2, 1) * M(3, 3) + M(1, 2) * M(2, 3) * M(3, 1) +
                               M(1, 3) * M(2, 1) * M(3, 2) - M(1, 3) * M(2, 2) * M(3, 1));
  if (detinv == 0.0) return false;
  inv[0] = +detinv * (M(2, 2) * M(3, 3) - M(2, 3) * M(3, 2));
  inv[1] = -detinv * (M(2, 1) * M(3, 3) - M(2, 3) * M(3, 1));
  inv[2] = +detinv * (M(2, 1) * M(3, 2) - M(2, 2) * M(3, 1));
  inv[3] = -detinv * (M(1, 2) * M(3, 3) - M(1, 3) * M(3, 2));
  inv[4] = +detinv * (M(1, 1) * M(3, 3) - M(1, 3) * M(3, 1));
  inv[5] = -detinv * (M(1, 1) * M(3, 2) - M(1, 2) * M(3, 1));
  inv[6] = +detinv * (M(1, 2) * M(2, 3) - M(1, 3) * M(2, 2));
  inv[7] = -detinv * (M(1, 1) * M(2, 3) - M(1, 3) * M(2, 1));
  inv[8] = +detinv * (M(1, 1) * M(2, 2) - M(1, 2) * M(2, 1));
#undef M
  return true;
}

// mod_quaternion.f90:136-145
__host__ __device__ inline Quat mult_quat(const Quat& x, const Quat& y) {
  return {x.a * y.a - x.b * y.b - x.c * y.c - x.d * y.d,
          x.a * y.b + x.b * y.a + x.c * y.d - x.d * y.c,
          x.a * y.c - x.b * y.d + x.c * y.a + x.d * y.b,
          x.a * y.d + x.b * y.c - x.c * y.b + x.d * y.a};
}

// adv_quaternion.f90:39-84 (direct multiplication, no renormalisation)
__host__ __device__ __forceinline__ void quaternion_integration(Quat& q, double ox, double oy, double oz, double dt) {
  double omg[3] = {ox, oy, oz};
  rot_vec(q, omg);
  const double nrm = sqrt(omg[0] * omg[0] + omg[1] * omg[1] + omg[2] * omg[2]);
  Quat map;
  if (nrm != 0.0) {
    const double h = (nrm * dt) / 2.0;
    double s, c;
    sincos(h, &s, &c);
    map = {c, s * (omg[0] / nrm), s * (omg[1] / nrm), s * (omg[2] / nrm)};
  } else {
    map = {1.0, 0.0, 0.0, 0.0};
  }
  q = mult_quat(map, q);
}

// adv_angular_velocity.f90:113-149 (METHOD=2)
__host__ __device__ inline void euler_integration(double ipxx, double ipyy, double ipzz, double dt,
                                                  double& ox, double& oy, double& oz) {
  const double w0x = ox, w0y = oy, w0z = oz;
  const double cx = (ipyy - ipzz) / ipxx, cy = (ipzz - ipxx) / ipyy, cz = (ipxx - ipyy) / ipzz;
  const double k1x = dt * (w0y * w0z * cx), k1y = dt * (w0z * w0x * cy), k1z = dt * (w0x * w0y * cz);
  const double k2x = dt * ((w0y + 0.5 * k1y) * (w0z + 0.5 * k1z) * cx);
  const double k2y = dt * ((w0z + 0.5 * k1z) * (w0x + 0.5 * k1x) * cy);
  const double k2z = dt * ((w0x + 0.5 * k1x) * (w0y + 0.5 * k1y) * cz);
  const double k3x = dt * ((w0y + 0.5 * k2y) * (w0z + 0.5 * k2z) * cx);
  const double k3y = dt * ((w0z + 0.5 * k2z) * (w0x + 0.5 * k2x) * cy);
  const double k3z = dt * ((w0x + 0.5 * k2x) * (w0y + 0.5 * k2y) * cz);
  const double k4x = dt * ((w0y + k3y) * (w0z + k3z) * cx);
  const double k4y = dt * ((w0z + k3z) * (w0x + k3x) * cy);
  const double k4z = dt * ((w0x + k3x) * (w0y + k3y) * cz);
  ox = w0x + (k1x + 2.0 * k2x + 2.0 * k3x + k4x) / 6.0;
  oy = w0y + (k1y + 2.0 * k2y + 2.0 * k3y + k4y) / 6.0;
  oz = w0z + (k1z + 2.0 * k2z + 2.0 * k3z + k4z) / 6.0;
}

// Per-particle constants hoisted out of the force/torque routines.  Each is a prefix
// of the reference's left-to-right product, so hoisting does not change a bit.
struct PartConst {
  double a, b;        // semi-axes: EMAJ, EMAJ/APR
  double deq;         // d_eq = 2a/APR^(2/3)            fluid_force_ellipsoid.f90:70
  double cdrag;       // (1/2)(RHOF/PMASS)(1/4)(PPI d^2)  fluid_force_ellipsoid.f90:119
  double cpitch;      // (1/4)(RHOF/PMASS)(1/4) PPI d^3   fluid_torque_ellipsoid.f90:147
  double crot;        // 0.5 RHOF/PMASS                   fluid_torque_ellipsoid.f90:158
  double h5;          // (d/2)^5
  double ipxx, ipyy, ipzz;
};

// R(q)^T v.  R(conj(q)) is R(q)^T bit for bit (conjugation only flips the signs of
// exact products), so this is rot_vec(conj(q), v) of transform_basis.f90:77.
__host__ __device__ inline void matvec_t(const double m[9], const double v[3], double o[3]) {
  const double t0 = m[0] * v[0] + m[1] * v[1] + m[2] * v[2];
  const double t1 = m[3] * v[0] + m[4] * v[1] + m[5] * v[2];
  const double t2 = m[6] * v[0] + m[7] * v[1] + m[8] * v[2];
  o[0] = t0; o[1] = t1; o[2] = t2;
}

// The particle's slip through the fluid as fluid_force_ellipsoid.f90:63-90 and
// fluid_torque_ellipsoid.f90:88-124 both form it, with the same operations: u_f - u_p,
// its magnitude, the Reynolds number, the slip in the body frame, its transverse part,
// the incidence angle's sine and cosine.  Formed once where the force and the torque
// see the same particle velocity.  (rep, umag and the angle are only read when umag0
// and, for the torque, syz are non-zero, as the reference reads them.)
struct Slip64 {
  double p[3];   // body frame
  double umag0, rep, syz, umag, sphi, cphi;
};

static __device__ __forceinline__ void slip64(const PartConst& pc, double visc, const double u[3],
                                              const double uf[3], const double r[9], Slip64& s) {
  double p[3] = {uf[0] - u[0], uf[1] - u[1], uf[2] - u[2]};
  s.umag0 = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
  s.rep = (s.umag0 * pc.deq) / visc;
  matvec_t(r, p, s.p);
  s.syz = sqrt(s.p[1] * s.p[1] + s.p[2] * s.p[2]);
  const double phi = fabs(atan(s.syz / s.p[0]));
  s.umag = sqrt(s.p[0] * s.p[0] + s.p[1] * s.p[1] + s.p[2] * s.p[2]);
  sincos(phi, &s.sphi, &s.cphi);
}

// fluid_force_ellipsoid.f90:1-161 (guards: zero relative speed -> zero force; zero
// transverse speed -> zero transverse lift; the reference stops or yields NaN there).
// Returns false if CDRAG is NaN (the reference's stop at :150-159).  r = R(q).
static __device__ __forceinline__ bool fluid_force(const PartConst& pc, const Slip64& s, const double r[9],
                                                   double fd[3], double fl[3]) {
  constexpr double a0 = 1.95, a1 = 18.12, a2 = 1.023, a3 = 4.26, a4 = 0.384;
  constexpr double a5 = 21.52, a6 = 0.990, a7 = 2.86, a8 = 0.260;
  constexpr double b1 = 0.083, b2 = -0.21, b3 = 1.582, b4 = 0.851, b5 = 1.842;
  constexpr double b6 = -0.802, b7 = -0.006, b8 = 0.874, b9 = 0.009, b10 = 0.570;
  fd[0] = fd[1] = fd[2] = 0.0;
  fl[0] = fl[1] = fl[2] = 0.0;
  if (s.umag0 == 0.0) return true;
  const double rep = s.rep, sphi = s.sphi, cphi = s.cphi, umag = s.umag;
  const double cd0 = (a1 / pow(rep, a2)) + (a3 / pow(rep, a4));
  const double cd90 = (a5 / pow(rep, a6)) + (a7 / pow(rep, a8));
  const double cdrag = cd0 + (cd90 - cd0) * pow(sphi, a0);
  const double clift = ((b1 / pow(rep, b2)) + (b3 / pow(rep, b4))) * pow(sphi, b5 + b6 * pow(rep, b7)) *
                       pow(cphi, b8 + b9 * pow(rep, b10));
  const double kd = pc.cdrag * cdrag * umag;
  fd[0] = kd * s.p[0];
  fd[1] = kd * s.p[1];
  fd[2] = kd * s.p[2];
  const double kl = pc.cdrag * clift * (umag * umag);
  fl[0] = kl * sphi * copysign(1.0, -s.p[0]);
  fl[1] = 0.0;
  fl[2] = 0.0;
  if (s.syz != 0.0) {
    fl[1] = kl * cphi * (s.p[1] / s.syz);
    fl[2] = kl * cphi * (s.p[2] / s.syz);
  }
  matvec(r, fd, fd);
  matvec(r, fl, fl);
  return !(cdrag != cdrag);
}

// fluid_torque_ellipsoid.f90:1-190.  Slip from the particle's stored velocity u_n
// (:88-105).  Guards as in fluid_force.  Pitching and rotation torques.  r = R(q).
static __device__ __forceinline__ void fluid_torque(const PartConst& pc, double visc, const Slip64& s,
                                                    double wx, double wy, double wz, double ox, double oy,
                                                    double oz, const double r[9], double tp[3], double tr[3]) {
  constexpr double c1 = 0.935, c2 = 0.146, c3 = -0.469, c4 = 0.145, c5 = 0.116;
  constexpr double c6 = 0.748, c7 = 0.041, c8 = 0.221, c9 = 0.657, c10 = 0.044;
  constexpr double r1 = 0.573, r2 = -0.154, r3 = 116.61;
  constexpr double r1_ = 1.244, r2_ = 0.239, r3_ = 378.12, r4_ = 0.789;
  const double wv[3] = {wx, wy, wz};
  double curl[3];
  matvec_t(r, wv, curl);
  const double o0 = 0.5 * curl[0] - ox, o1 = 0.5 * curl[1] - oy, o2 = 0.5 * curl[2] - oz;
  const double omag = sqrt(o0 * o0 + o1 * o1 + o2 * o2);
  const double oyz = sqrt(o2 * o2 + o1 * o1);
  const double re_r = (omag * (pc.deq * pc.deq)) / visc;
  double tp1 = 0.0, tp2 = 0.0, tr0 = 0.0, tr1 = 0.0, tr2 = 0.0;
  if (s.umag0 != 0.0 && s.syz != 0.0) {
    const double rep = s.rep, sphi = s.sphi, cphi = s.cphi, umag = s.umag;
    const double ctp = (c1 / pow(rep, c2) + c3 / pow(rep, c4)) * (pow(sphi, c5 + c6 * pow(rep, c7))) *
                       (pow(cphi, c8 + c9 * pow(rep, c10)));
    const double cp = pc.cpitch * ctp * (umag * umag);
    tp1 = cp * (fabs(s.p[2]) / s.syz) * copysign(1.0, s.p[0] * s.p[2]);
    tp2 = cp * (fabs(s.p[1]) / s.syz) * copysign(1.0, s.p[0] * s.p[1]);
  }
  if (re_r != 0.0) {
    const double ctr = r1 * pow(re_r, r2) + r3 / re_r;
    const double ctr2 = r1_ * pow(re_r, r2_) + r3_ / pow(re_r, r4_);
    tr0 = ctr * pc.crot * pc.h5 * fabs(o0) * o0;
    tr1 = ctr2 * pc.crot * pc.h5 * oyz * o1;
    tr2 = ctr2 * pc.crot * pc.h5 * oyz * o2;
  }
  tp[0] = 0.0; tp[1] = tp1; tp[2] = tp2;
  tr[0] = tr0; tr[1] = tr1; tr[2] = tr2;
}

// Skew matrix [r]x as in wall_ellipsoid_rebound.f90:176-186 / collision_response.f90:163-173
__host__ __device__ inline void skew(const double r[3], double m[9]) {
  m[0] = 0.0;   m[3] = -r[2]; m[6] = r[1];
  m[1] = r[2];  m[4] = 0.0;   m[7] = -r[0];
  m[2] = -r[1]; m[5] = r[0];  m[8] = 0.0;
}

// K = I + [r]x^T Ip^-1 [r]x   (wall_ellipsoid_rebound.f90:194, collision_response.f90:181)
__host__ __device__ inline void k_matrix(const double inv_ip[9], const double rx[9], double k[9]) {
  double t[9], rxt[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) rxt[i + 3 * j] = rx[j + 3 * i];
  matmul(inv_ip, rx, t);
  matmul(rxt, t, t);
#pragma unroll
  for (int i = 0; i < 9; ++i) k[i] = ((i % 4) == 0 ? 1.0 : 0.0) + t[i];
}

// ellipsoid_wall_boundary_new.f90 + closest_point_plane.f90 + max_encroachment_ellipsoid.f90.
// A centre farther than 1.5 bounding radii from the chosen plane cannot give margin<1
// (margin >= dist^2/rmax^2 = 2.25), so that case skips the matrix work with the same
// outcome.  Returns error code (0 ok, GP_ESINGULAR).
static __device__ __forceinline__ int wall_test(double lx, const PartConst& pc, double rmax, double xp, double yp, double zp,
                                const Quat& q, double wn[3], double arm[3], double& delta_x, bool& isect) {
  arm[0] = arm[1] = arm[2] = 0.0;
  isect = false;
  double wpos0;
  if (xp < lx / 2.0) { wpos0 = 0.0; wn[0] = 1.0; } else { wpos0 = lx; wn[0] = -1.0; }
  wn[1] = 0.0; wn[2] = 0.0;
  if (fabs(xp - wpos0) > 1.5 * rmax) return 0;
  double ell[9], inv[9];
  rot_diag(q, 1.0 / (pc.a * pc.a), 1.0 / (pc.b * pc.b), 1.0 / (pc.b * pc.b), ell);
  if (!invert3(ell, inv)) return GP_ESINGULAR;
  double ivn[3];
  matvec(inv, wn, ivn);
  const double tn = wn[0] * ivn[0] + wn[1] * ivn[1] + wn[2] * ivn[2];
  const double ellc[3] = {xp, yp, zp};
  const double d0 = wpos0 - ellc[0], d1 = yp - ellc[1], d2 = zp - ellc[2];
  const double tw = wn[0] * d0 + wn[1] * d1 + wn[2] * d2;
  const double lag = tw / tn;
  double vec[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) vec[i] = (ellc[i] + lag * ivn[i]) - ellc[i];
  double e_[3];
  matvec(ell, vec, e_);
  const double margin = vec[0] * e_[0] + vec[1] * e_[1] + vec[2] * e_[2];
  if (margin < 1.0) {
    isect = true;
    const double s = sqrt(tn);
    double pt[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) pt[i] = ellc[i] - ivn[i] / s;
    arm[0] = (xp - pt[0]);
    arm[1] = (yp - pt[1]);
    arm[2] = (zp - pt[2]);
    delta_x = wpos0 - pt[0];
  }
  return 0;
}

// wall_ellipsoid_rebound.f90:1-387.  Returns 0, GP_ESINGULAR or GP_EENERGY.
static __device__ __forceinline__ int wall_rebound(double ecw, double muw, const PartConst& pc, double& u, double& v, double& w,
                                   double& ox, double& oy, double& oz, const Quat& q, const double ri[3],
                                   const double nw[3]) {
  double omg[3] = {ox, oy, oz};
  rot_vec(q, omg);
  double vpc[3];
  vpc[0] = u + (omg[1] * ri[2] - omg[2] * ri[1]);
  vpc[1] = v + (omg[2] * ri[0] - omg[0] * ri[2]);
  vpc[2] = w + (omg[0] * ri[1] - omg[1] * ri[0]);
  const double vrn = vpc[0] * nw[0] + vpc[1] * nw[1] + vpc[2] * nw[2];
  double delv[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) delv[i] = vpc[i] + ecw * vrn * nw[i];
  double ip[9], inv_ip[9], rx[9], k[9], k1[9];
  rot_diag(q, pc.ipxx, pc.ipyy, pc.ipzz, ip);
  if (!invert3(ip, inv_ip)) return GP_ESINGULAR;
  skew(ri, rx);
  k_matrix(inv_ip, rx, k);
  if (!invert3(k, k1)) return GP_ESINGULAR;
  double pcv[3];
  matvec(k1, delv, pcv);
  pcv[0] = -pcv[0]; pcv[1] = -pcv[1]; pcv[2] = -pcv[2];
  double pcn = pcv[0] * nw[0] + pcv[1] * nw[1] + pcv[2] * nw[2];
  const double px = pcv[0] - pcn * nw[0], py = pcv[1] - pcn * nw[1], pz = pcv[2] - pcn * nw[2];
  const double pct = sqrt(px * px + py * py + pz * pz);
  if (pct > muw * pcn) {
    double tw[3] = {vpc[0] - vrn * nw[0], vpc[1] - vrn * nw[1], vpc[2] - vrn * nw[2]};
    const double nrm = sqrt(tw[0] * tw[0] + tw[1] * tw[1] + tw[2] * tw[2]);
    if (nrm != 0.0) { tw[0] = -tw[0] / nrm; tw[1] = -tw[1] / nrm; tw[2] = -tw[2] / nrm; }
    const double vimp[3] = {nw[0] + muw * tw[0], nw[1] + muw * tw[1], nw[2] + muw * tw[2]};
    double kn[3];
    matvec(k, vimp, kn);
    const double kndn = kn[0] * nw[0] + kn[1] * nw[1] + kn[2] * nw[2];
    pcn = -1.0 * (delv[0] * nw[0] + delv[1] * nw[1] + delv[2] * nw[2]);
#pragma unroll
    for (int i = 0; i < 3; ++i) pcv[i] = (pcn / kndn) * vimp[i];
  }
  double am[3];
  const double eit = 0.5 * (u * u + v * v + w * w);
  matvec(ip, omg, am);
  const double eir = 0.5 * (omg[0] * am[0] + omg[1] * am[1] + omg[2] * am[2]);
  const double ei = eit + eir;
  u = u + pcv[0]; v = v + pcv[1]; w = w + pcv[2];
  double tmp[3], dom[3];
  matvec(rx, pcv, tmp);
  matvec(inv_ip, tmp, dom);
#pragma unroll
  for (int i = 0; i < 3; ++i) omg[i] = omg[i] + dom[i];
  const double eft = 0.5 * (u * u + v * v + w * w);
  matvec(ip, omg, am);
  const double efr = 0.5 * (omg[0] * am[0] + omg[1] * am[1] + omg[2] * am[2]);
  const double ef = eft + efr;
  rot_vec(conj(q), omg);
  ox = omg[0]; oy = omg[1]; oz = omg[2];
  if (fabs((ei - ef) / ei) * 100.0 > 1.0e-9) return GP_EENERGY;
  return 0;
}

// collision_response.f90:1-437 (inertia of particle 1 for both bodies, :140-145).
static __device__ __noinline__ int collision_response(double ecp, double mup, double ipxx, double ipyy, double ipzz,
                                         double u1[3], double o1[3], const Quat& q1,
                                         double u2[3], double o2[3], const Quat& q2,
                                         const double r1[3], const double r2[3], const double n[3]) {
  double om1[3] = {o1[0], o1[1], o1[2]}, om2[3] = {o2[0], o2[1], o2[2]};
  rot_vec(q1, om1);
  rot_vec(q2, om2);
  double upc1[3], upc2[3];
  upc1[0] = u1[0] + (om1[1] * r1[2] - om1[2] * r1[1]);
  upc1[1] = u1[1] + (om1[2] * r1[0] - om1[0] * r1[2]);
  upc1[2] = u1[2] + (om1[0] * r1[1] - om1[1] * r1[0]);
  upc2[0] = u2[0] + (om2[1] * r2[2] - om2[2] * r2[1]);
  upc2[1] = u2[1] + (om2[2] * r2[0] - om2[0] * r2[2]);
  upc2[2] = u2[2] + (om2[0] * r2[1] - om2[1] * r2[0]);
  const double urel[3] = {upc2[0] - upc1[0], upc2[1] - upc1[1], upc2[2] - upc1[2]};
  const double urn = urel[0] * n[0] + urel[1] * n[1] + urel[2] * n[2];
  double delu[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) delu[i] = urel[i] + ecp * urn * n[i];
  double ip1[9], ip2[9], inv1[9], inv2[9], rx1[9], rx2[9], k1[9], k2[9], k[9], invk[9];
  rot_diag(q1, ipxx, ipyy, ipzz, ip1);
  rot_diag(q2, ipxx, ipyy, ipzz, ip2);
  if (!invert3(ip1, inv1)) return GP_ESINGULAR;
  if (!invert3(ip2, inv2)) return GP_ESINGULAR;
  skew(r1, rx1);
  k_matrix(inv1, rx1, k1);
  skew(r2, rx2);
  k_matrix(inv2, rx2, k2);
#pragma unroll
  for (int i = 0; i < 9; ++i) k[i] = k1[i] + k2[i];
  if (!invert3(k, invk)) return GP_ESINGULAR;
  double pc[3];
  matvec(invk, delu, pc);
  pc[0] = -pc[0]; pc[1] = -pc[1]; pc[2] = -pc[2];
  double pcn = pc[0] * n[0] + pc[1] * n[1] + pc[2] * n[2];
  const double px = pc[0] - pcn * n[0], py = pc[1] - pcn * n[1], pz = pc[2] - pcn * n[2];
  const double pct = sqrt(px * px + py * py + pz * pz);
  if (pct > mup * pcn) {
    double tw[3] = {urel[0] - urn * n[0], urel[1] - urn * n[1], urel[2] - urn * n[2]};
    const double nrm = sqrt(tw[0] * tw[0] + tw[1] * tw[1] + tw[2] * tw[2]);
    if (nrm != 0.0) { tw[0] = -tw[0] / nrm; tw[1] = -tw[1] / nrm; tw[2] = -tw[2] / nrm; }
    const double vimp[3] = {n[0] + mup * tw[0], n[1] + mup * tw[1], n[2] + mup * tw[2]};
    double kn[3];
    matvec(k, vimp, kn);
    const double kndn = kn[0] * n[0] + kn[1] * n[1] + kn[2] * n[2];
    pcn = -1.0 * (delu[0] * n[0] + delu[1] * n[1] + delu[2] * n[2]);
#pragma unroll
    for (int i = 0; i < 3; ++i) pc[i] = (pcn / kndn) * vimp[i];
  }
  double am[3];
  const double eit1 = 0.5 * (u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]);
  matvec(ip1, om1, am);
  const double eir1 = 0.5 * (om1[0] * am[0] + om1[1] * am[1] + om1[2] * am[2]);
  const double eit2 = 0.5 * (u2[0] * u2[0] + u2[1] * u2[1] + u2[2] * u2[2]);
  matvec(ip2, om2, am);
  const double eir2 = 0.5 * (om2[0] * am[0] + om2[1] * am[1] + om2[2] * am[2]);
  const double ei = (eit1 + eir1) + (eit2 + eir2);
  u1[0] = u1[0] - pc[0]; u1[1] = u1[1] - pc[1]; u1[2] = u1[2] - pc[2];
  double mpc[3] = {-pc[0], -pc[1], -pc[2]}, tmp[3], dom[3];
  matvec(rx1, mpc, tmp);
  matvec(inv1, tmp, dom);
#pragma unroll
  for (int i = 0; i < 3; ++i) om1[i] = om1[i] + dom[i];
  u2[0] = u2[0] + pc[0]; u2[1] = u2[1] + pc[1]; u2[2] = u2[2] + pc[2];
  matvec(rx2, pc, tmp);
  matvec(inv2, tmp, dom);
#pragma unroll
  for (int i = 0; i < 3; ++i) om2[i] = om2[i] + dom[i];
  const double eft1 = 0.5 * (u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]);
  matvec(ip1, om1, am);
  const double efr1 = 0.5 * (om1[0] * am[0] + om1[1] * am[1] + om1[2] * am[2]);
  const double eft2 = 0.5 * (u2[0] * u2[0] + u2[1] * u2[1] + u2[2] * u2[2]);
  matvec(ip2, om2, am);
  const double efr2 = 0.5 * (om2[0] * am[0] + om2[1] * am[1] + om2[2] * am[2]);
  const double ef = (eft1 + efr1) + (eft2 + efr2);
  rot_vec(conj(q1), om1);
  rot_vec(conj(q2), om2);
  o1[0] = om1[0]; o1[1] = om1[1]; o1[2] = om1[2];
  o2[0] = om2[0]; o2[1] = om2[1]; o2[2] = om2[2];
  if (fabs((ei - ef) / ei) > 1.0e-9) return GP_EENERGY;
  return 0;
}

}  // namespace gp
