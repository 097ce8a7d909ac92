// gp_advance.cuh -- fused ADV_PARTICLE_ELLP kernel body: 64-point Lagrange gather of
// the six field components at x_n, RK2 predictor/corrector with the wall test and
// rebound, periodic wrap.  Included by the FP64 (plain) and the mixed translation units.
#pragma once
#include <math_constants.h>

#include "gp_device.cuh"

namespace gp {

// Internal field layout: [k: nz+4][j: ny+4][i: nx+3][c: kFieldStride].  Reference
// index (I, J, K) with J, K in -1..N+2 (NGHTCELL=2 ghost planes) and I in 1..NX maps
// to (I, J+1, K+1); x ghost columns 0, NX+1, NX+2 hold columns NX, 1, 2 so that the
// periodic x wrap of interp_lag3.f90:132-154 reads four contiguous points.  The six
// components of a point are padded to eight, so a point is one 32-byte sector (FP32)
// and a stencil row of four points is 128 contiguous, aligned bytes.
__device__ __forceinline__ int64_t field_point(const InstDev& I, int ix, int jy, int kz) {
  return ((int64_t)(kz + 1) * (I.ny + 4) + (jy + 1)) * (int64_t)(I.nx + 3) + ix;
}

// Cubic Lagrange weights (interp_lag3.f90:196-211), FP64.
__device__ __forceinline__ void lag3_w(double a, double f[4]) {
  f[0] = -1. / 6. * (a - 2.) * (a - 1.) * a;
  f[1] = 1. / 2. * (a - 2.) * (a - 1.) * (a + 1.);
  f[2] = -1. / 2. * (a - 2.) * a * (a + 1.);
  f[3] = 1. / 6. * (a - 1.) * a * (a + 1.);
}
__device__ __forceinline__ void lag3_wf(float a, float f[4]) {
  f[0] = -1.f / 6.f * (a - 2.f) * (a - 1.f) * a;
  f[1] = 0.5f * (a - 2.f) * (a - 1.f) * (a + 1.f);
  f[2] = -0.5f * (a - 2.f) * a * (a + 1.f);
  f[3] = 1.f / 6.f * (a - 1.f) * a * (a + 1.f);
}

struct Stencil {
  int ix[4], j0, k0;
  double alfa, beta, gama;
  bool contiguous;
};

// Stencil nodes of interp_lag3.f90:124-190.  Returns false if the stencil leaves the
// array (the reference would read out of bounds).
__device__ __forceinline__ bool stencil(const InstDev& I, double x, double y, double z, Stencil& s) {
  const double dxa = I.dx, dya = I.dy, dza = I.dz;   // XAIN(2)-XAIN(1) = DX
  const double fx = x / dxa, fy = y / dya, fz = z / dza;
  if (!(fx > -2.0 && fx < 2147483000.0 && fy > -2.0 && fy < 2147483000.0 && fz > -2.0 &&
        fz < 2147483000.0))
    return false;
  const int i0 = (int)fx + 1, j0 = (int)fy + 1, k0 = (int)fz + 1;
  if (i0 < 1 || i0 > I.nx || j0 < 0 || j0 > I.ny || k0 < 0 || k0 > I.nz) return false;
  if (I.wall_boundary) {
    const int iend = I.nx;
    int ip1 = (i0 == iend) ? iend - 1 : i0 + 1;
    int ip2 = (ip1 == iend) ? iend - 1 : ip1 + 1;
    int im1 = (i0 == 1) ? 2 : i0 - 1;
    s.ix[0] = im1; s.ix[1] = i0; s.ix[2] = ip1; s.ix[3] = ip2;
    s.contiguous = (ip2 == i0 + 2) && (im1 == i0 - 1);
  } else {
    s.ix[0] = i0 - 1; s.ix[1] = i0; s.ix[2] = i0 + 1; s.ix[3] = i0 + 2;
    s.contiguous = true;
  }
  s.j0 = j0;
  s.k0 = k0;
  // explicit IEEE roundings: identical offsets whether or not the translation unit
  // contracts multiply-adds (the FP64 and mixed paths share this routine)
  s.alfa = __ddiv_rn(__dsub_rn(x, __dmul_rn((double)(i0 - 1), I.dx)), dxa);
  s.beta = __ddiv_rn(__dsub_rn(y, __dmul_rn(I.dy, (double)(j0 - 1))), dya);
  s.gama = __ddiv_rn(__dsub_rn(z, __dmul_rn(I.dz, (double)(k0 - 1))), dza);
  return true;
}

// FP64 gather of the six components with the reference's nesting z(y(x))
// (interp_lag3.f90:220-288).
__device__ __forceinline__ void gather6_fp64(const InstDev& I, const Stencil& s, double out[6]) {
  const double* __restrict__ F = static_cast<const double*>(I.field);
  double fx[4], fy[4], fz[4];
  lag3_w(s.alfa, fx);
  lag3_w(s.beta, fy);
  lag3_w(s.gama, fz);
  double zs[6];
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
    double ys[6];
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      double xs[6];
      const int64_t p0 = field_point(I, s.ix[0], s.j0 - 1 + jj, s.k0 - 1 + kk);
      if (s.contiguous) {
        const double2* row = reinterpret_cast<const double2*>(F + p0 * kFieldStride);
        double v[24];
#pragma unroll
        for (int ii = 0; ii < 4; ++ii)
#pragma unroll
          for (int t = 0; t < 3; ++t) {
            const double2 d = __ldg(row + ii * (kFieldStride / 2) + t);
            v[6 * ii + 2 * t] = d.x;
            v[6 * ii + 2 * t + 1] = d.y;
          }
#pragma unroll
        for (int c = 0; c < 6; ++c)
          xs[c] = fx[0] * v[c] + fx[1] * v[6 + c] + fx[2] * v[12 + c] + fx[3] * v[18 + c];
      } else {
        double v[24];
#pragma unroll
        for (int ii = 0; ii < 4; ++ii) {
          const int64_t pp = field_point(I, s.ix[ii], s.j0 - 1 + jj, s.k0 - 1 + kk);
#pragma unroll
          for (int c = 0; c < 6; ++c) v[6 * ii + c] = __ldg(F + pp * kFieldStride + c);
        }
#pragma unroll
        for (int c = 0; c < 6; ++c)
          xs[c] = fx[0] * v[c] + fx[1] * v[6 + c] + fx[2] * v[12 + c] + fx[3] * v[18 + c];
      }
#pragma unroll
      for (int c = 0; c < 6; ++c) ys[c] = (jj == 0) ? fy[0] * xs[c] : ys[c] + fy[jj] * xs[c];
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) zs[c] = (kk == 0) ? fz[0] * ys[c] : zs[c] + fz[kk] * ys[c];
  }
#pragma unroll
  for (int c = 0; c < 6; ++c) out[c] = zs[c];
}

// FP32 field, FP32 weights, Kahan-compensated FP32 accumulation of the 64 products
// w_x w_y w_z U.  Result returned in double.
__device__ __forceinline__ void gather6_fp32(const InstDev& I, const Stencil& s, double out[6]) {
  const float* __restrict__ F = static_cast<const float*>(I.field);
  float fx[4], fy[4], fz[4];
  lag3_wf((float)s.alfa, fx);
  lag3_wf((float)s.beta, fy);
  lag3_wf((float)s.gama, fz);
  float sum[6], cmp[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) { sum[c] = 0.f; cmp[c] = 0.f; }
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      const float wyz = fz[kk] * fy[jj];
      const int64_t p0 = field_point(I, s.ix[0], s.j0 - 1 + jj, s.k0 - 1 + kk);
      float v[24];
      if (s.contiguous) {
        const float4* row = reinterpret_cast<const float4*>(F + p0 * kFieldStride);
#pragma unroll
        for (int ii = 0; ii < 4; ++ii) {
          const float4 d = __ldg(row + 2 * ii);
          const float2 e = __ldg(reinterpret_cast<const float2*>(row + 2 * ii + 1));
          v[6 * ii + 0] = d.x; v[6 * ii + 1] = d.y; v[6 * ii + 2] = d.z; v[6 * ii + 3] = d.w;
          v[6 * ii + 4] = e.x; v[6 * ii + 5] = e.y;
        }
      } else {
#pragma unroll
        for (int ii = 0; ii < 4; ++ii) {
          const int64_t pp = field_point(I, s.ix[ii], s.j0 - 1 + jj, s.k0 - 1 + kk);
#pragma unroll
          for (int c = 0; c < 6; ++c) v[6 * ii + c] = __ldg(F + pp * kFieldStride + c);
        }
      }
#pragma unroll
      for (int ii = 0; ii < 4; ++ii) {
        const float w = wyz * fx[ii];
#pragma unroll
        for (int c = 0; c < 6; ++c) {
          // Kahan step: sum += w*v with the lost low part carried in cmp
          const float y = __fmaf_rn(w, v[6 * ii + c], -cmp[c]);
          const float t = __fadd_rn(sum[c], y);
          cmp[c] = __fsub_rn(__fsub_rn(t, sum[c]), y);
          sum[c] = t;
        }
      }
    }
  }
#pragma unroll
  for (int c = 0; c < 6; ++c) out[c] = (double)sum[c] - (double)cmp[c];
}

// ---------------------------------------------------------------------------
// Mixed-precision force and torque.  The Zastawny correlation coefficients are FP32 and
// bound the relative error of every force and torque near 1e-7, so the rest of the
// force and torque is formed in FP32 too: the slip u_f - u_p and the spin are taken as
// FP64 differences of the FP64 state and then rounded, and the rotation R(q), the
// body-frame slip, its magnitudes and reciprocals, the per-particle constants
// (MixedConst) and the assembled force and torque are FP32.  The state they advance
// stays FP64.  The body-frame flow is shared by the force and the torque when both see
// the same particle velocity (the first RK2 stage).
// ---------------------------------------------------------------------------
// Everything the mixed form's common path needs of a particle's constants, formed once:
// the full PartConst is not kept, and the rare wall branches read it again from the pool,
// so that the integrate holds fewer registers.
struct MixedConst {
  float dv;               // deq / visc: particle Reynolds number per unit slip speed
  float d2v;              // deq^2 / visc: rotational Reynolds number per unit spin
  float cd, cp, krot;     // cdrag, cpitch and crot * h5 in FP32
  float rix, riy, riz;    // 1 / principal moments of inertia (FP32 reciprocals)
  double dyz, dzx, dxy;   // ipyy - ipzz, ipzz - ipxx, ipxx - ipyy
  double rmax;            // bounding radius max(a, b)
};

__device__ __forceinline__ void mixed_const(const PartConst& pc, double visc, MixedConst& mc) {
  const float vi = __frcp_rn((float)visc), d = (float)pc.deq;
  mc.dv = d * vi;
  mc.d2v = (d * d) * vi;
  mc.cd = (float)pc.cdrag;
  mc.cp = (float)pc.cpitch;
  mc.krot = (float)(pc.crot * pc.h5);
  mc.rix = __frcp_rn((float)pc.ipxx);
  mc.riy = __frcp_rn((float)pc.ipyy);
  mc.riz = __frcp_rn((float)pc.ipzz);
  mc.dyz = pc.ipyy - pc.ipzz;
  mc.dzx = pc.ipzz - pc.ipxx;
  mc.dxy = pc.ipxx - pc.ipyy;
  mc.rmax = fmax(pc.a, pc.b);
}

// The FP32 arithmetic of the mixed force, torque and rotation increment is written with
// explicit roundings (__fmaf_rn, __fmul_rn): the plain and the speculative integrate are
// separate kernels, and a multiply-add that the compiler fused in one and not in the
// other would make the two give different bits for the same particle.
__device__ __forceinline__ float dot3f(float a0, float a1, float a2, float b0, float b1, float b2) {
  return __fmaf_rn(a2, b2, __fmaf_rn(a1, b1, __fmul_rn(a0, b0)));
}

// R(q) of transform_basis.f90:44-54 in FP32 (same layout as rotmat: r[i + 3j] = R_ij).
__device__ __forceinline__ void rotmat_f(const Quat& q, float r[9]) {
  const float q0 = (float)q.a, q1 = (float)q.b, q2 = (float)q.c, q3 = (float)q.d;
  r[0] = __fsub_rn(1.f, __fmul_rn(2.f, __fmaf_rn(q2, q2, __fmul_rn(q3, q3))));
  r[3] = __fmul_rn(2.f, __fmaf_rn(q1, q2, -__fmul_rn(q0, q3)));
  r[6] = __fmul_rn(2.f, __fmaf_rn(q1, q3, __fmul_rn(q0, q2)));
  r[1] = __fmul_rn(2.f, __fmaf_rn(q1, q2, __fmul_rn(q0, q3)));
  r[4] = __fsub_rn(1.f, __fmul_rn(2.f, __fmaf_rn(q1, q1, __fmul_rn(q3, q3))));
  r[7] = __fmul_rn(2.f, __fmaf_rn(q2, q3, -__fmul_rn(q0, q1)));
  r[2] = __fmul_rn(2.f, __fmaf_rn(q1, q3, -__fmul_rn(q0, q2)));
  r[5] = __fmul_rn(2.f, __fmaf_rn(q2, q3, __fmul_rn(q0, q1)));
  r[8] = __fsub_rn(1.f, __fmul_rn(2.f, __fmaf_rn(q1, q1, __fmul_rn(q2, q2))));
}

// 2^x and the square root as one hardware instruction each (ex2.approx, sqrt.approx):
// relative errors near 2^-22, below the FP32 correlations' own 1e-7; sqrt(0) = 0 and
// 2^-inf = 0 as the force and torque need.
__device__ __forceinline__ float ex2_fast(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float sqrt_fast(float x) {
  float y;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Slip velocity u_f - u_p in the body frame (R^T p), its magnitude, the magnitude of its
// transverse part and the incidence angle phi = |atan(syz / b0)| in [0, pi/2].
struct RelFlow {
  float b0, b1, b2;       // body frame
  float umag, syz, inv_syz;
  float lr, sphi, cphi;   // log2 of the particle Reynolds number, sin and cos of phi
};

static __device__ __forceinline__ void rel_flow(const MixedConst& mc, const double u[3], const double uf[3],
                                                const float r[9], RelFlow& q) {
  const float p0 = (float)(uf[0] - u[0]), p1 = (float)(uf[1] - u[1]), p2 = (float)(uf[2] - u[2]);
  q.umag = sqrt_fast(dot3f(p0, p1, p2, p0, p1, p2));
  q.b0 = dot3f(r[0], r[1], r[2], p0, p1, p2);
  q.b1 = dot3f(r[3], r[4], r[5], p0, p1, p2);
  q.b2 = dot3f(r[6], r[7], r[8], p0, p1, p2);
  const float s2 = __fmaf_rn(q.b2, q.b2, __fmul_rn(q.b1, q.b1));
  q.syz = sqrt_fast(s2);
  q.inv_syz = __frcp_rn(q.syz);   // used only where syz != 0
  // phi = |atan(syz / b0)| (pi/2 where b0 = 0) has sin(phi) = syz / |b| and
  // cos(phi) = |b0| / |b|: no angle needs forming (|b| = 0 gives phi = 0)
  const float bb = __fmaf_rn(q.b0, q.b0, s2);
  if (bb > 0.f) {
    const float inv = rsqrtf(bb);
    q.sphi = fminf(__fmul_rn(q.syz, inv), 1.f);
    q.cphi = fminf(__fmul_rn(fabsf(q.b0), inv), 1.f);
  } else {
    q.sphi = 0.f;
    q.cphi = 1.f;
  }
  q.lr = __log2f(__fmul_rn(q.umag, mc.dv));
}

// x^y for x in [0, 1] and y > 0 (sines and cosines of the incidence angle raised to the
// correlations' exponents) as 2^(y log2 x) with the hardware log2 and exp2: an absolute
// error of a few 1e-7 of the result where it is not negligible against the rest of the
// coefficient, the size of the FP32 correlations' own rounding.  x = 0 gives 0.
__device__ __forceinline__ float pow_unit(float x, float y) { return ex2_fast(y * __log2f(x)); }

static __device__ __forceinline__ bool fluid_force_mixed(const MixedConst& mc, const RelFlow& q, const float r[9],
                                                         double f[3]) {
  f[0] = f[1] = f[2] = 0.0;
  if (q.umag == 0.f) return true;
  const float lr = q.lr, sphi = q.sphi, cphi = q.cphi;
  const float cd0 = __fmaf_rn(18.12f, ex2_fast(-1.023f * lr), __fmul_rn(4.26f, ex2_fast(-0.384f * lr)));
  const float cd90 = __fmaf_rn(21.52f, ex2_fast(-0.990f * lr), __fmul_rn(2.86f, ex2_fast(-0.260f * lr)));
  const float cdrag = __fmaf_rn(__fsub_rn(cd90, cd0), pow_unit(sphi, 1.95f), cd0);
  const float clift = __fmul_rn(__fmul_rn(__fmaf_rn(0.083f, ex2_fast(0.21f * lr), __fmul_rn(1.582f, ex2_fast(-0.851f * lr))),
                                          pow_unit(sphi, __fmaf_rn(-0.802f, ex2_fast(-0.006f * lr), 1.842f))),
                                pow_unit(cphi, __fmaf_rn(0.009f, ex2_fast(0.570f * lr), 0.874f)));
  const float cd = mc.cd;
  const float kd = __fmul_rn(__fmul_rn(cd, cdrag), q.umag);
  const float kl = __fmul_rn(__fmul_rn(cd, clift), __fmul_rn(q.umag, q.umag));
  const float fb0 = __fmaf_rn(kd, q.b0, __fmul_rn(__fmul_rn(kl, sphi), copysignf(1.f, -q.b0)));
  float fb1 = __fmul_rn(kd, q.b1), fb2 = __fmul_rn(kd, q.b2);
  if (q.syz != 0.f) {
    const float kc = __fmul_rn(__fmul_rn(kl, cphi), q.inv_syz);
    fb1 = __fmaf_rn(kc, q.b1, fb1);
    fb2 = __fmaf_rn(kc, q.b2, fb2);
  }
  f[0] = (double)dot3f(r[0], r[3], r[6], fb0, fb1, fb2);
  f[1] = (double)dot3f(r[1], r[4], r[7], fb0, fb1, fb2);
  f[2] = (double)dot3f(r[2], r[5], r[8], fb0, fb1, fb2);
  return !(cdrag != cdrag) && isfinite(f[0]) && isfinite(f[1]) && isfinite(f[2]);
}

static __device__ __forceinline__ void fluid_torque_mixed(const MixedConst& mc, const RelFlow& q,
                                                          const double wv[3], double ox, double oy, double oz,
                                                          const float r[9], double t[3]) {
  const float w0 = (float)wv[0], w1 = (float)wv[1], w2 = (float)wv[2];
  const float c0 = dot3f(r[0], r[1], r[2], w0, w1, w2);
  const float c1 = dot3f(r[3], r[4], r[5], w0, w1, w2);
  const float c2 = dot3f(r[6], r[7], r[8], w0, w1, w2);
  const float o0 = __fmaf_rn(0.5f, c0, -(float)ox), o1 = __fmaf_rn(0.5f, c1, -(float)oy);
  const float o2 = __fmaf_rn(0.5f, c2, -(float)oz);
  const float omag = sqrt_fast(dot3f(o0, o1, o2, o0, o1, o2));
  const float oyz = sqrt_fast(__fmaf_rn(o2, o2, __fmul_rn(o1, o1)));
  t[0] = t[1] = t[2] = 0.0;
  if (q.umag != 0.f && q.syz != 0.f) {
    const float lr = q.lr, sphi = q.sphi, cphi = q.cphi;
    const float ctp =
        __fmul_rn(__fmul_rn(__fmaf_rn(0.935f, ex2_fast(-0.146f * lr), __fmul_rn(-0.469f, ex2_fast(-0.145f * lr))),
                            pow_unit(sphi, __fmaf_rn(0.748f, ex2_fast(0.041f * lr), 0.116f))),
                  pow_unit(cphi, __fmaf_rn(0.657f, ex2_fast(0.044f * lr), 0.221f)));
    const float cp = __fmul_rn(__fmul_rn(__fmul_rn(mc.cp, ctp), __fmul_rn(q.umag, q.umag)), q.inv_syz);
    t[1] = (double)(cp * fabsf(q.b2) * copysignf(1.f, q.b0 * q.b2));
    t[2] = (double)(cp * fabsf(q.b1) * copysignf(1.f, q.b0 * q.b1));
  }
  const float re_r = __fmul_rn(omag, mc.d2v);
  if (re_r != 0.f) {
    const float lr = __log2f(re_r);
    const float ctr = __fmaf_rn(0.573f, ex2_fast(-0.154f * lr), __fmul_rn(116.61f, __frcp_rn(re_r)));
    const float ctr2 = __fmaf_rn(1.244f, ex2_fast(0.239f * lr), __fmul_rn(378.12f, ex2_fast(-0.789f * lr)));
    const float k = mc.krot;
    t[0] += (double)(ctr * k * fabsf(o0) * o0);
    t[1] += (double)(ctr2 * k * oyz * o1);
    t[2] += (double)(ctr2 * k * oyz * o2);
  }
}

template <bool kMixed>
struct Forces {
  // F (lab frame, per unit mass) and T (body frame) for stage velocities: the force
  // sees the stage velocity u, the torque the velocity un at the start of the step
  // (same_u: u and un are the same values).  r = R(q) in FP32 (mixed form only).
  __device__ __forceinline__ static bool eval(const PartConst& pc, double visc, const MixedConst& mc,
                                              const double u[3], const double un[3], bool same_u,
                                              const double uf[3], const double wv[3], double ox, double oy,
                                              double oz, const Quat& q, const float r[9], double f[3],
                                              double t[3]) {
    if (kMixed) {
      RelFlow qf;
      rel_flow(mc, u, uf, r, qf);
      const bool ok = fluid_force_mixed(mc, qf, r, f);
      if (same_u) {
        fluid_torque_mixed(mc, qf, wv, ox, oy, oz, r, t);
      } else {
        RelFlow qt;
        rel_flow(mc, un, uf, r, qt);
        fluid_torque_mixed(mc, qt, wv, ox, oy, oz, r, t);
      }
      return ok;
    } else {
      // one R(q) and, where u and un are the same values, one slip for both routines
      double rq[9];
      rotmat(q, rq);
      double fd[3], fl[3], tp[3], tr[3];
      Slip64 sf;
      slip64(pc, visc, u, uf, rq, sf);
      const bool ok = fluid_force(pc, sf, rq, fd, fl);
      if (same_u) {
        fluid_torque(pc, visc, sf, wv[0], wv[1], wv[2], ox, oy, oz, rq, tp, tr);
      } else {
        Slip64 st;
        slip64(pc, visc, un, uf, rq, st);
        fluid_torque(pc, visc, st, wv[0], wv[1], wv[2], ox, oy, oz, rq, tp, tr);
      }
      f[0] = fd[0] + fl[0]; f[1] = fd[1] + fl[1]; f[2] = fd[2] + fl[2];
      t[0] = tp[0] + tr[0]; t[1] = tp[1] + tr[1]; t[2] = tp[2] + tr[2];
      return ok;
    }
  }
};

// adv_particle_new.f90:305-307; the mixed form multiplies by the reciprocal moments.
template <bool kMixed>
__device__ __forceinline__ void k_omega(const double t[3], double ox, double oy, double oz, const PartConst& pc,
                                        const MixedConst& mc, double k[3]) {
  if (kMixed) {
    k[0] = (t[0] + oy * oz * mc.dyz) * (double)mc.rix;
    k[1] = (t[1] + oz * ox * mc.dzx) * (double)mc.riy;
    k[2] = (t[2] + ox * oy * mc.dxy) * (double)mc.riz;
  } else {
    k[0] = (t[0] + oy * oz * (pc.ipyy - pc.ipzz)) / pc.ipxx;
    k[1] = (t[1] + oz * ox * (pc.ipzz - pc.ipxx)) / pc.ipyy;
    k[2] = (t[2] + ox * oy * (pc.ipxx - pc.ipyy)) / pc.ipzz;
  }
}

// Quaternion step of adv_quaternion.f90:39-84 followed by renormalisation (mixed form).
// r = R(q) in FP32: the body-to-lab rotation that the stage's force evaluation already
// built.  The increment (the spin in the lab frame, the half angle's sine and cosine) is
// FP32: a relative error of a few 1e-8 of one step's rotation; the product with q and
// the renormalisation are FP64.
__device__ __forceinline__ void quaternion_step_mixed(Quat& q, const float r[9], double ox, double oy, double oz,
                                                      double dt) {
  const float w0 = (float)ox, w1 = (float)oy, w2 = (float)oz;
  const float g0 = dot3f(r[0], r[3], r[6], w0, w1, w2);
  const float g1 = dot3f(r[1], r[4], r[7], w0, w1, w2);
  const float g2 = dot3f(r[2], r[5], r[8], w0, w1, w2);
  const float n2 = dot3f(g0, g1, g2, g0, g1, g2);
  Quat map = {1.0, 0.0, 0.0, 0.0};
  if (n2 > 0.f) {
    const float inv = rsqrtf(n2);
    const float h = __fmul_rn(__fmul_rn(n2, inv), (float)(dt * 0.5));
    float s, c;
    if (h <= 0.785f) {
      // Taylor series of sin and cos about 0, nested in h^2 up to the h^9 and h^10 terms:
      // sin h = h (1 - h^2/(2.3) (1 - h^2/(4.5) (1 - h^2/(6.7) (1 - h^2/(8.9))))),
      // cos h = 1 - h^2/(1.2) (1 - h^2/(3.4) (...(1 - h^2/(9.10)))); the first term left
      // out is below 3e-9 for h <= pi/4, under FP32's rounding
      const float h2 = __fmul_rn(h, h);
      float ps = __fmaf_rn(-h2, 1.f / 72.f, 1.f);
      ps = __fmaf_rn(__fmul_rn(-h2, 1.f / 42.f), ps, 1.f);
      ps = __fmaf_rn(__fmul_rn(-h2, 1.f / 20.f), ps, 1.f);
      ps = __fmaf_rn(__fmul_rn(-h2, 1.f / 6.f), ps, 1.f);
      s = __fmul_rn(h, ps);
      float pc = __fmaf_rn(-h2, 1.f / 90.f, 1.f);
      pc = __fmaf_rn(__fmul_rn(-h2, 1.f / 56.f), pc, 1.f);
      pc = __fmaf_rn(__fmul_rn(-h2, 1.f / 30.f), pc, 1.f);
      pc = __fmaf_rn(__fmul_rn(-h2, 1.f / 12.f), pc, 1.f);
      c = __fmaf_rn(__fmul_rn(-h2, 0.5f), pc, 1.f);
    } else {
      sincosf(h, &s, &c);
    }
    const float si = __fmul_rn(s, inv);
    map = {(double)c, (double)__fmul_rn(si, g0), (double)__fmul_rn(si, g1), (double)__fmul_rn(si, g2)};
  }
  q = mult_quat(map, q);
  const double inv = rsqrt(q.a * q.a + q.b * q.b + q.c * q.c + q.d * q.d);
  q.a *= inv; q.b *= inv; q.c *= inv; q.d *= inv;
}

// One quaternion update; r = R(q) is used by the mixed form only.
template <bool kMixed>
__device__ __forceinline__ void quat_advance(Quat& q, const float r[9], double ox, double oy, double oz, double dt) {
  if (kMixed) quaternion_step_mixed(q, r, ox, oy, oz, dt);
  else quaternion_integration(q, ox, oy, oz, dt);
}

// One particle of adv_particle_new.f90:268-637.  State in/out in registers.
// Returns 0 or an error code.
__device__ __forceinline__ void load_pc(const PoolView& P, int64_t i, PartConst& pc) {
  pc.a = P.pc[0][i]; pc.b = P.pc[1][i]; pc.deq = P.pc[2][i]; pc.cdrag = P.pc[3][i];
  pc.cpitch = P.pc[4][i]; pc.crot = P.pc[5][i]; pc.h5 = P.pc[6][i];
  pc.ipxx = P.pc[7][i]; pc.ipyy = P.pc[8][i]; pc.ipzz = P.pc[9][i];
}

// wall_test for the advance: the FP64 form has the particle's constants at hand; the
// mixed form takes wall_test's own early exit (centre farther than 1.5 bounding radii
// from the chosen plane: no intersection) before it reads them back from the pool.
template <bool kMixed>
__device__ __forceinline__ int wall_test_adv(double lx, const PartConst& pc, const PoolView& S, int64_t si,
                                             double rmax, double xp, double yp, double zp, const Quat& q,
                                             double wn[3], double arm[3], double& delta_x, bool& isect) {
  if (kMixed) {
    const double wpos0 = (xp < lx / 2.0) ? 0.0 : lx;
    if (fabs(xp - wpos0) > 1.5 * rmax) {
      arm[0] = arm[1] = arm[2] = 0.0;
      isect = false;
      wn[0] = (xp < lx / 2.0) ? 1.0 : -1.0;
      wn[1] = 0.0; wn[2] = 0.0;
      return 0;
    }
    PartConst full;
    load_pc(S, si, full);
    return wall_test(lx, full, rmax, xp, yp, zp, q, wn, arm, delta_x, isect);
  }
  return wall_test(lx, pc, rmax, xp, yp, zp, q, wn, arm, delta_x, isect);
}

// One particle of adv_particle_new.f90:268-637.  State in/out in registers.  The FP64
// form takes the particle's constants in pc; the mixed form takes them formed in mc, and
// reads them again from the pool (S, slot si) in the rare wall branches.
// Returns 0 or an error code.
template <bool kMixed>
__device__ __forceinline__ int advance_particle(const InstDev& I, const PartConst& pc, const MixedConst& mc,
                                                const PoolView& S, int64_t si, const double uf[3],
                                                const double wv[3], double X[3], double U[3], double O[3],
                                                Quat& Q) {
  const double dt = I.dtime;
  const double rmax = kMixed ? mc.rmax : fmax(pc.a, pc.b);
  const double un[3] = {U[0], U[1], U[2]};
  double f[3], t[3];
  float r0[9], r1[9];   // R(Q) and R(q1) in FP32, mixed form only
  if (kMixed) rotmat_f(Q, r0);
  int err = 0;
  if (!Forces<kMixed>::eval(pc, I.visc, mc, un, un, true, uf, wv, O[0], O[1], O[2], Q, r0, f, t)) err = GP_ENAN_FORCE;
  if (O[0] != O[0] && !err) err = GP_ENAN_TORQUE;
  const double k1x[3] = {U[0], U[1], U[2]};
  const double k1u[3] = {f[0], f[1], f[2] + I.gravity};
  double k1o[3];
  k_omega<kMixed>(t, O[0], O[1], O[2], pc, mc, k1o);
  double xp1 = X[0] + dt * k1x[0], yp1 = X[1] + dt * k1x[1], zp1 = X[2] + dt * k1x[2];
  double u1[3] = {U[0] + dt * k1u[0], U[1] + dt * k1u[1], U[2] + dt * k1u[2]};
  double o1[3] = {O[0] + dt * k1o[0], O[1] + dt * k1o[1], O[2] + dt * k1o[2]};
  Quat q1 = Q;
  quat_advance<kMixed>(q1, r0, o1[0], o1[1], o1[2], dt);
  double wn[3], arm[3], delta_x = 0.0;
  bool isect;
  int rc = wall_test_adv<kMixed>(I.lx, pc, S, si, rmax, xp1, yp1, zp1, q1, wn, arm, delta_x, isect);
  if (rc && !err) err = rc;
  if (isect && u1[0] * wn[0] < 0.0) {
    // rebound branch, adv_particle_new.f90:358-511
    double ol[3] = {o1[0], o1[1], o1[2]};
    rot_vec(q1, ol);
    double vpc[3];
    vpc[0] = u1[0] + (ol[1] * arm[2] - ol[2] * arm[1]);
    vpc[1] = u1[1] + (ol[2] * arm[0] - ol[0] * arm[2]);
    vpc[2] = u1[2] + (ol[0] * arm[1] - ol[1] * arm[0]);
    xp1 = xp1 + delta_x;
    const double delt = fabs(delta_x) / sqrt(vpc[0] * vpc[0] + vpc[1] * vpc[1] + vpc[2] * vpc[2]);
    yp1 = X[1] + (dt - delt) * k1x[1];
    zp1 = X[2] + (dt - delt) * k1x[2];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      u1[i] = U[i] + (dt - delt) * k1u[i];
      o1[i] = O[i] + (dt - delt) * k1o[i];
    }
    q1 = Q;
    if (kMixed) rotmat_f(Q, r0);   // rebuilt here, so that R(Q) need not stay live on the common path
    quat_advance<kMixed>(q1, r0, o1[0], o1[1], o1[2], dt - delt);
    if (kMixed) {
      PartConst full;
      load_pc(S, si, full);
      rc = wall_rebound(I.ecw, I.muw, full, u1[0], u1[1], u1[2], o1[0], o1[1], o1[2], q1, arm, wn);
    } else {
      rc = wall_rebound(I.ecw, I.muw, pc, u1[0], u1[1], u1[2], o1[0], o1[1], o1[2], q1, arm, wn);
    }
    if (rc && !err) err = rc;
    if (kMixed) rotmat_f(q1, r1);
    if (!Forces<kMixed>::eval(pc, I.visc, mc, u1, un, false, uf, wv, o1[0], o1[1], o1[2], q1, r1, f, t) && !err)
      err = GP_ENAN_FORCE;
    if (o1[0] != o1[0] && !err) err = GP_ENAN_TORQUE;
    const double k2u[3] = {f[0], f[1], f[2] + I.gravity};
    double k2o[3];
    k_omega<kMixed>(t, o1[0], o1[1], o1[2], pc, mc, k2o);
    X[0] = xp1 + (delt) * u1[0];
    X[1] = yp1 + (delt) * u1[1];
    X[2] = zp1 + (delt) * u1[2];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      U[i] = u1[i] + (delt) * k2u[i];
      O[i] = o1[i] + (delt) * k2o[i];
    }
    Q = q1;
    quat_advance<kMixed>(Q, r1, O[0], O[1], O[2], delt);
    return err;
  }
  // unbounced second stage, adv_particle_new.f90:513-637
  if (kMixed) rotmat_f(q1, r1);
  if (!Forces<kMixed>::eval(pc, I.visc, mc, u1, un, false, uf, wv, o1[0], o1[1], o1[2], q1, r1, f, t) && !err)
    err = GP_ENAN_FORCE;
  if (o1[0] != o1[0] && !err) err = GP_ENAN_TORQUE;
  const double k2x[3] = {u1[0], u1[1], u1[2]};
  const double k2u[3] = {f[0], f[1], f[2] + I.gravity};
  double k2o[3];
  k_omega<kMixed>(t, o1[0], o1[1], o1[2], pc, mc, k2o);
  const double xp2 = X[0] + 0.5 * dt * (k1x[0] + k2x[0]);
  const double yp2 = X[1] + 0.5 * dt * (k1x[1] + k2x[1]);
  const double zp2 = X[2] + 0.5 * dt * (k1x[2] + k2x[2]);
  rc = wall_test_adv<kMixed>(I.lx, pc, S, si, rmax, xp2, yp2, zp2, q1, wn, arm, delta_x, isect);
  if (rc && !err) err = rc;
  if (isect) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      X[i] = X[i] + dt * k1x[i];
      U[i] = U[i] + dt * k1u[i];
      O[i] = O[i] + dt * k1o[i];
    }
  } else {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      X[i] = X[i] + 0.5 * dt * (k1x[i] + k2x[i]);
      U[i] = U[i] + 0.5 * dt * (k1u[i] + k2u[i]);
      O[i] = O[i] + 0.5 * dt * (k1o[i] + k2o[i]);
    }
  }
  Q = q1;
  quat_advance<kMixed>(Q, r1, O[0], O[1], O[2], dt);
  return err;
}

__device__ __forceinline__ float pick4(const float f[4], int k) {
  return k == 0 ? f[0] : (k == 1 ? f[1] : (k == 2 ? f[2] : f[3]));
}

// Warp-cooperative FP32 gather for the 32 particles of one warp.  Eight lanes serve one
// particle: lane t of the group loads float4 (t & 1) of point (t >> 1) of each of the 16
// stencil rows (one aligned 128-byte row per group and load instruction, instead of 32
// scattered 8-byte loads).  A lane sums its point's column: the four y rows of each z
// plane weighted by w_y, then the four planes weighted by w_z (FP32 multiply-adds, 4-term
// sums), then the product with w_x exactly in double; the four x points are summed in
// double across the group.  (interp_lag3.f90:220-288 nests the same sums with x
// innermost; the FP64 form keeps that order.)
// Its rounding error (a few FP32 ulps of sum |w u|) stays far below the FP32 drag
// correlations' 1e-7, and it takes a quarter of the instructions of a compensated
// (Kahan) sum of the 64 products.  mode: 0 no gather, 1 cooperative (contiguous row),
// 2 left to the lane itself.
__device__ __forceinline__ void gather_warp_fp32(const InstDev* __restrict__ insts, int mode, int inst,
                                                 int64_t b, float al, float be, float ga, int64_t j0,
                                                 double* const* __restrict__ fluid) {
  constexpr unsigned kFull = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int t = lane & 7, k = t >> 1, half = t & 1;
#pragma unroll 1
  for (int g = 0; g < 8; ++g) {
    const int o = g * 4 + (lane >> 3);
    const int mo = __shfl_sync(kFull, mode, o);
    const int io = __shfl_sync(kFull, inst, o);
    const long long bo = __shfl_sync(kFull, (long long)b, o);
    const float alo = __shfl_sync(kFull, al, o), beo = __shfl_sync(kFull, be, o), gao = __shfl_sync(kFull, ga, o);
    float4 zs = make_float4(0.f, 0.f, 0.f, 0.f);
    float wxl = 0.f;
    if (mo == 1) {
      const InstDev& I = insts[io];
      const float* __restrict__ F = static_cast<const float*>(I.field);
      const int64_t sy = I.nx + 3, sz = (int64_t)(I.ny + 4) * sy;
      float fx[4], fy[4], fz[4];
      lag3_wf(alo, fx);
      lag3_wf(beo, fy);
      lag3_wf(gao, fz);
      const float wx = pick4(fx, k);
      const float* __restrict__ p = F + (bo + k) * kFieldStride + 4 * half;
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        float4 ys = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          const float4 v = __ldg(reinterpret_cast<const float4*>(p + (kk * sz + jj * sy) * kFieldStride));
          ys.x = __fmaf_rn(fy[jj], v.x, ys.x);
          ys.y = __fmaf_rn(fy[jj], v.y, ys.y);
          ys.z = __fmaf_rn(fy[jj], v.z, ys.z);
          ys.w = __fmaf_rn(fy[jj], v.w, ys.w);
        }
        zs.x = __fmaf_rn(fz[kk], ys.x, zs.x);
        zs.y = __fmaf_rn(fz[kk], ys.y, zs.y);
        zs.z = __fmaf_rn(fz[kk], ys.z, zs.z);
        zs.w = __fmaf_rn(fz[kk], ys.w, zs.w);
      }
      wxl = wx;
    }
    const double wd = (double)wxl;
    double d0 = (double)zs.x * wd, d1 = (double)zs.y * wd;
    double d2 = (double)zs.z * wd, d3 = (double)zs.w * wd;
#pragma unroll
    for (int m = 2; m <= 4; m <<= 1) {
      d0 += __shfl_xor_sync(kFull, d0, m);
      d1 += __shfl_xor_sync(kFull, d1, m);
      d2 += __shfl_xor_sync(kFull, d2, m);
      d3 += __shfl_xor_sync(kFull, d3, m);
    }
    if (mo == 1 && t < 2) {
      const int64_t jo = j0 + o;
      if (half == 0) {
        fluid[0][jo] = d0; fluid[1][jo] = d1; fluid[2][jo] = d2; fluid[3][jo] = d3;
      } else {
        fluid[4][jo] = d0; fluid[5][jo] = d1;
      }
    }
  }
}

// ADV_PARTICLE_ELLP, first half: the six field components at x_n
// (adv_particle_new.f90:139-206) of the particle that the next integrate pass will
// place in slot j, perm[j] of the current buffer (the last binning's cell order, so
// that neighbouring stencils are gathered together).  Reads only positions, instance
// and id, so it may run while the collision phase updates velocities.  kMixed: every
// instance holds an FP32 field (warp-cooperative gather); otherwise FP64 fields,
// gathered per lane in the reference's summation order.
// Each warp takes the next 32 slots from *ticket (zero at launch), so the slots in
// flight at any time are one contiguous run of the cell order whatever the grid: the
// field rows that neighbouring stencils share stay in L2 between their uses, where a
// grid-stride loop over many blocks spreads the resident warps over the pool.
// two blocks of 256 per SM: 128 registers, no spills (at three, 80 registers spill)
#ifndef GP_GATHER_MIN_BLOCKS
#define GP_GATHER_MIN_BLOCKS 2
#endif
template <bool kMixed>
__global__ void __launch_bounds__(256, GP_GATHER_MIN_BLOCKS) k_gather(const InstDev* __restrict__ insts,
                                                const PoolView* __restrict__ src_pv,
                                                const int32_t* __restrict__ perm, int64_t n,
                                                double* const* __restrict__ fluid,
                                                unsigned long long* __restrict__ ticket, Status* st) {
  if (step_halted(st)) return;
  const int lane = threadIdx.x & 31;
  for (;;) {
    unsigned long long wt = 0;
    if (lane == 0) wt = atomicAdd(ticket, 1ull);
    const int64_t w = (int64_t)__shfl_sync(0xffffffffu, wt, 0);
    if (w * 32 >= n) break;
    const int64_t j = w * 32 + lane;
    int inst = -1;
    int64_t i = 0;
    if (j < n) {
      i = perm[j];
      inst = src_pv->inst[i];
    }
    int mode = 0;
    Stencil s;
    if (inst >= 0) {
      const InstDev& I = insts[inst];
      if (stencil(I, src_pv->st[0][i], src_pv->st[1][i], src_pv->st[2][i], s)) {
        mode = (kMixed && s.contiguous) ? 1 : 2;
      } else {
        set_error(st, GP_EOUT_OF_GRID, (long long)src_pv->id[i], inst);
      }
    }
    if (j < n && mode == 0) {
#pragma unroll
      for (int c = 0; c < 6; ++c) fluid[c][j] = CUDART_NAN;
    }
    if (kMixed) {
      const int64_t b = (mode == 1) ? field_point(insts[inst], s.ix[0], s.j0 - 1, s.k0 - 1) : 0;
      gather_warp_fp32(insts, mode, inst, b, (float)s.alfa, (float)s.beta, (float)s.gama, w * 32, fluid);
    }
    if (mode == 2) {
      const InstDev& I = insts[inst];
      double g[6];
      if (kMixed) gather6_fp32(I, s, g); else gather6_fp64(I, s, g);
#pragma unroll
      for (int c = 0; c < 6; ++c) fluid[c][j] = g[c];
    }
  }
}

// ADV_PARTICLE_ELLP, second half, for one particle: particle i of the source buffer is
// advanced and written to slot j of the destination buffer with its properties, id and
// instance (any permutation is correct: every particle carries its own record).  The
// RK2 predictor/corrector with wall handling (adv_particle_new.f90:268-637) and
// BOUNDARY_PARTICLE's periodic wrap (boundary_particle.f90:50-59).  A particle whose
// stencil left the field (NaN fluid values, reported by the gather) is copied unchanged.
template <bool kMixed>
__device__ __forceinline__ void integrate_slot(const InstDev* __restrict__ insts, const PoolView* __restrict__ S,
                                               const PoolView* __restrict__ D, int64_t i, int64_t j,
                                               const double* const* __restrict__ fluid, Status* st) {
  const int inst = S->inst[i];
  D->inst[j] = inst;
  D->id[j] = S->id[i];
  PartConst pc;
  load_pc(*S, i, pc);
#pragma unroll 1
  for (int c = 0; c < kNConst; ++c) D->pc[c][j] = S->pc[c][i];
  MixedConst mc;
  double X[3] = {S->st[0][i], S->st[1][i], S->st[2][i]};
  double U[3] = {S->st[3][i], S->st[4][i], S->st[5][i]};
  Quat Q = {S->st[6][i], S->st[7][i], S->st[8][i], S->st[9][i]};
  double O[3] = {S->st[10][i], S->st[11][i], S->st[12][i]};
  const double uf[3] = {fluid[0][j], fluid[1][j], fluid[2][j]};
  const double wv[3] = {fluid[3][j], fluid[4][j], fluid[5][j]};
  // stencil out of range (reported by the gather): carried over unchanged
  if (inst >= 0 && !(uf[0] != uf[0] && wv[0] != wv[0])) {
    const InstDev& I = insts[inst];
    if (kMixed) mixed_const(pc, I.visc, mc);
    const int err = advance_particle<kMixed>(I, pc, mc, *S, i, uf, wv, X, U, O, Q);
    if (err) set_error(st, err, (long long)S->id[i], inst);
    // adv_particle_new.f90:685-686: the channel wraps y and z only
    // (boundary_particle_yz.f90:44-70), the others every direction when periodic
    if (I.frozen_flow == 3) {
      if (X[1] > I.ly) X[1] = X[1] - I.ly;
      else if (X[1] < 0.) X[1] = X[1] + I.ly;
      if (X[2] > I.lz) X[2] = X[2] - I.lz;
      else if (X[2] < 0.) X[2] = X[2] + I.lz;
    } else if (I.periodicity) {
      if (X[0] > I.lx) X[0] = X[0] - I.lx;
      if (X[0] < 0.) X[0] = X[0] + I.lx;
      if (X[1] > I.ly) X[1] = X[1] - I.ly;
      if (X[1] < 0.) X[1] = X[1] + I.ly;
      if (X[2] > I.lz) X[2] = X[2] - I.lz;
      if (X[2] < 0.) X[2] = X[2] + I.lz;
    }
  }
  D->st[0][j] = X[0]; D->st[1][j] = X[1]; D->st[2][j] = X[2];
  D->st[3][j] = U[0]; D->st[4][j] = U[1]; D->st[5][j] = U[2];
  D->st[6][j] = Q.a; D->st[7][j] = Q.b; D->st[8][j] = Q.c; D->st[9][j] = Q.d;
  D->st[10][j] = O[0]; D->st[11][j] = O[1]; D->st[12][j] = O[2];
}

// The pass over the pool: particle perm[j] of the source buffer goes to slot j of the
// destination.  With mark non-null (the speculative pass, run while the previous step's
// contact solves and response are still going) a particle that the last search marked
// (it is in a candidate pair, so the response may still change its velocity) is left
// alone: mark[i] receives j + 1 and k_integrate_fix advances it once the response is
// done.  Unmarked particles are ones the response never touches, so both passes read
// exactly the state a single pass after the response would read.
#ifndef GP_INTEGRATE_MIN_BLOCKS
#define GP_INTEGRATE_MIN_BLOCKS 4
#endif
template <bool kMixed>
__global__ void __launch_bounds__(128, GP_INTEGRATE_MIN_BLOCKS) k_integrate(const InstDev* __restrict__ insts,
                                                                           const PoolView* __restrict__ src_pv,
                                                                           const PoolView* __restrict__ dst_pv,
                                                                           const int32_t* __restrict__ perm, int64_t n,
                                                                           const double* const* __restrict__ fluid,
                                                                           uint32_t* __restrict__ mark, Status* st) {
  if (step_halted(st)) return;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = perm[j];
    if (mark != nullptr && mark[i] != 0u) {
      mark[i] = (uint32_t)(j + 1);
      continue;
    }
    integrate_slot<kMixed>(insts, src_pv, dst_pv, i, j, fluid, st);
  }
}

// The rest of a speculative pass, after the response: every particle of the stored
// candidate pairs (pairs[0, min(*npairs, cap))) that the search marked, once each (the
// first lane to clear its mark takes it), into the slot the speculative pass recorded.
// The marks are all zero again afterwards.
template <bool kMixed>
__global__ void __launch_bounds__(128, GP_INTEGRATE_MIN_BLOCKS) k_integrate_fix(const InstDev* __restrict__ insts,
                                                                               const PoolView* __restrict__ src_pv,
                                                                               const PoolView* __restrict__ dst_pv,
                                                                               const PairRec* __restrict__ pairs,
                                                                               const unsigned long long* npairs,
                                                                               int64_t cap,
                                                                               const double* const* __restrict__ fluid,
                                                                               uint32_t* __restrict__ mark, Status* st) {
  if (step_halted(st)) return;
  const int64_t np = (int64_t)min(*npairs, (unsigned long long)cap);
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < 2 * np; e += (int64_t)gridDim.x * blockDim.x) {
    const PairRec& r = pairs[e >> 1];
    const int64_t i = (e & 1) ? r.near : r.home;
    const uint32_t v = atomicExch(&mark[i], 0u);
    if (v != 0u) integrate_slot<kMixed>(insts, src_pv, dst_pv, i, (int64_t)v - 1, fluid, st);
  }
}

// After an advance the destination buffer becomes the current one (not after an advance
// that a halted step skipped).
static __global__ void k_swap_pool(PoolView* a, PoolView* b, const Status* st) {
  if (step_halted(st)) return;
  const PoolView t = *a;
  *a = *b;
  *b = t;
}

}  // namespace gp
