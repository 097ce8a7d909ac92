// gp_lm.cuh -- ellipsoid contact detection with a register-resident Levenberg-
// Marquardt solve (FP64), one pair per thread.
//
// ellipsoid_contact_detection.f90:1-187 parametrises the common normal by two angles
// and minimises the squared components of the gap between the two support points
// with lmder1 (minpack_reduc.f90:652-757: ftol=xtol=sqrt(eps), gtol=0,
// maxfev=100(n+1), mode=1, factor=100).  The solver below is the MINPACK
// Levenberg-Marquardt method (Moré 1978; MINPACK-1 user guide, ANL-80-74: QR with
// column pivoting, Levenberg-Marquardt parameter by the secular-equation iteration,
// Givens-rotation least-squares update, trust-region step control) for the fixed size
// n=2 variables, m=3 residuals; every loop bound is a compile-time constant.
#pragma once
#include <cfloat>
#include <math_constants.h>

#include "gp_device.cuh"

namespace gp {

// Linkage of the solver's building blocks.  Out-of-line calls keep the register count
// of the pair-search and batch kernels low; GP_LM_INLINE folds the whole solve into
// its caller, which shortens the dependent-latency chain of one iteration.
#ifdef GP_LM_INLINE
#define GP_LM_FN static __device__ __forceinline__
#else
#define GP_LM_FN static __device__ __noinline__
#endif
// The pieces of one iteration are folded into the iteration itself.
#define GP_LM_INNER static __device__ __forceinline__
// Once per solve (set-up and the final contact test): out of line in every build, so
// that they do not add to the register pressure of the iteration they bracket.
#define GP_LM_COLD static __device__ __noinline__

// Correctly rounded FP64 division and square root of the solver, one place for every
// site of the iteration.  They are in line by default.  Out of line
// (GP_LM_CALLED_ARITH) each site becomes a call and the iteration's code shrinks by a
// quarter, but on the B200 the bulk of 150k solves like those of the 512^3 /
// 16.8 M-spheroid workload then took 4.45 ms against 3.72 ms in line: the calls cost
// more than the smaller code saves once the norm's rare paths are out of line
// (lm_enorm).
#ifdef GP_LM_CALLED_ARITH
#define GP_LM_ARITH static __device__ __noinline__
#else
#define GP_LM_ARITH static __device__ __forceinline__
#endif
GP_LM_ARITH double lm_div(double a, double b) { return a / b; }
GP_LM_ARITH double lm_sqrt(double a) { return sqrt(a); }

// MINPACK's scaled Euclidean norm (minpack_reduc.f90:180-232): three accumulators
// for tiny, mid-range and huge components.
template <int N>
__device__ __noinline__ double lm_enorm_general(const double* x) {
  constexpr double rdwarf = 3.834e-20, rgiant = 1.304e19;
  double s1 = 0.0, s2 = 0.0, s3 = 0.0, x1max = 0.0, x3max = 0.0;
  const double agiant = rgiant / (double)N;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const double xabs = fabs(x[i]);
    if (xabs > rdwarf && xabs < agiant) {
      s2 = s2 + xabs * xabs;
    } else if (xabs <= rdwarf) {
      if (xabs <= x3max) {
        if (xabs != 0.0) { const double r = xabs / x3max; s3 = s3 + r * r; }
      } else {
        const double r = x3max / xabs;
        s3 = 1.0 + s3 * (r * r);
        x3max = xabs;
      }
    } else if (xabs <= x1max) {
      const double r = xabs / x1max;
      s1 = s1 + r * r;
    } else {
      const double r = x1max / xabs;
      s1 = 1.0 + s1 * (r * r);
      x1max = xabs;
    }
  }
  if (s1 != 0.0) return x1max * sqrt(s1 + (s2 / x1max) / x1max);
  if (s2 == 0.0) return x3max * sqrt(s3);
  if (s2 >= x3max) return sqrt(s2 * (1.0 + (x3max / s2) * (x3max * s3)));
  return sqrt(x3max * ((s2 / x3max) + (x3max * s3)));
}

// The same norm with its common case in line: when every component is zero or in the
// mid range, MINPACK's result is sqrt(s2 * (1 + (0/s2) * (0*0))), which is sqrt(s2)
// exactly (zero components add nothing to s2 and leave s3 and x3max at zero).  The
// tiny, huge and NaN cases go to the full routine above.  Keeping its divisions out of
// the iteration's code keeps that code small enough for the instruction caches.
template <int N>
__device__ __forceinline__ double lm_enorm(const double* x) {
  constexpr double rdwarf = 3.834e-20, rgiant = 1.304e19;
  const double agiant = rgiant / (double)N;
  double s2 = 0.0;
  bool mid = true;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const double xabs = fabs(x[i]);
    mid = mid && ((xabs > rdwarf && xabs < agiant) || xabs == 0.0);
    s2 = s2 + xabs * xabs;
  }
  if (mid) return lm_sqrt(s2);
  return lm_enorm_general<N>(x);
}

// Trigonometric functions of the contact solve.  The reference calls libm's
// sin/cos/asin/acos there; the kernels and the oracle use these functions
// (same constants, same operation order, compiled without contraction) so that their
// Levenberg-Marquardt iterates agree bit for bit.  Method: Cody-Waite reduction by
// pi/2 split into three parts and Taylor polynomials on [-pi/4, pi/4]; asin by its
// Taylor series on |x| <= 1/2 and pi/2 - 2 asin(sqrt((1-x)/2)) above.  The solve
// resolves its angles only to xtol = sqrt(eps), far above one-ulp differences.
#define CT_QUAL __host__ __device__ __forceinline__
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
#ifdef GP_LM_INLINE
#define CT_SINCOS_QUAL CT_QUAL
#else
#define CT_SINCOS_QUAL inline __host__ __device__ __noinline__
#endif
CT_SINCOS_QUAL void ct_sincos(double x, double *s, double *c) {
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

struct ContactProb {
  double e1[9], e2[9];   // R diag(a^2,b^2,b^2) R^T (calculate_ellipsoid_matrix.f90:33-72)
  double b1[3], b2[3];
  // entry k of body W's matrix, coordinate i of body W's centre
  template <int W> __device__ __forceinline__ double e(int k) const { return W == 0 ? e1[k] : e2[k]; }
  template <int W> __device__ __forceinline__ double b(int i) const { return W == 0 ? b1[i] : b2[i]; }
};

// The same problem held in shared memory, one column per lane of a 128-thread block
// (entry m of the lane's problem at base[m * kProbLanes]; m = 0..8 E1, 9..17 E2,
// 18..20 b1, 21..23 b2): the solve reads it there and keeps its registers for its state.
constexpr int kProbLanes = 128;
constexpr int kProbWords = 24;
struct SmemProb {
  double* base;
  template <int W> __device__ __forceinline__ double e(int k) const { return base[(W * 9 + k) * kProbLanes]; }
  template <int W> __device__ __forceinline__ double b(int i) const { return base[(18 + W * 3 + i) * kProbLanes]; }
  __device__ __forceinline__ void store(const ContactProb& P) const {
#pragma unroll
    for (int k = 0; k < 9; ++k) { base[k * kProbLanes] = P.e1[k]; base[(9 + k) * kProbLanes] = P.e2[k]; }
#pragma unroll
    for (int i = 0; i < 3; ++i) { base[(18 + i) * kProbLanes] = P.b1[i]; base[(21 + i) * kProbLanes] = P.b2[i]; }
  }
};

// Everything the residual at x computes that the Jacobian at the same x needs again:
// the trigonometric values of the two angles, the support-function values lambda_1,
// lambda_2, the factors 1/(2 lambda_i) and the gap vector (whose squares are the
// residual).  The Jacobian is only ever taken at a point whose residual was the last
// one accepted, so keeping these avoids a second evaluation of the same expressions.
struct SupportEval {
  double s0, k0, s1, k1;   // sin, cos of x[0] and x[1]
  double l1, l2, f1, f2;   // lambda_i and 1/(2 lambda_i)
  double depth[3];         // pt1 - pt2
};

// E_W v, in matvec's order of terms
template <int W, class Prob>
__device__ __forceinline__ void prob_matvec(const Prob& P, const double v[3], double o[3]) {
  const double t0 = P.template e<W>(0) * v[0] + P.template e<W>(3) * v[1] + P.template e<W>(6) * v[2];
  const double t1 = P.template e<W>(1) * v[0] + P.template e<W>(4) * v[1] + P.template e<W>(7) * v[2];
  const double t2 = P.template e<W>(2) * v[0] + P.template e<W>(5) * v[1] + P.template e<W>(8) * v[2];
  o[0] = t0; o[1] = t1; o[2] = t2;
}

// Support points along +-c(x) (ellipsoid_pair_depth.f90:117-142): E receives the
// quantities above, pt1/pt2 the points themselves.
template <class Prob>
GP_LM_INNER void support_eval(const Prob& P, const double x[2], SupportEval& E, double pt1[3], double pt2[3]) {
  ct_sincos(x[0], &E.s0, &E.k0);
  ct_sincos(x[1], &E.s1, &E.k1);
  const double c1[3] = {E.k0 * E.k1, E.s0 * E.k1, E.s1};
  const double c2[3] = {-c1[0], -c1[1], -c1[2]};
  double t1[3], t2[3];
  prob_matvec<0>(P, c1, t1);
  prob_matvec<1>(P, c2, t2);
  E.l1 = lm_sqrt(0.25 * (c1[0] * t1[0] + c1[1] * t1[1] + c1[2] * t1[2]));
  E.l2 = lm_sqrt(0.25 * (c2[0] * t2[0] + c2[1] * t2[1] + c2[2] * t2[2]));
  E.f1 = lm_div(1.0, 2.0 * E.l1);
  E.f2 = lm_div(1.0, 2.0 * E.l2);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    pt1[i] = E.f1 * t1[i] + P.template b<0>(i);
    pt2[i] = E.f2 * t2[i] + P.template b<1>(i);
    E.depth[i] = pt1[i] - pt2[i];
  }
}

// Support points alone (the contact test after the solve).
template <class Prob>
GP_LM_INNER void support_points(const Prob& P, const double x[2], double c1[3], double pt1[3], double pt2[3]) {
  SupportEval E;
  support_eval(P, x, E, pt1, pt2);
  c1[0] = E.k0 * E.k1;
  c1[1] = E.s0 * E.k1;
  c1[2] = E.s1;
}

// fcn, iflag=1 (ellipsoid_contact_detection.f90:290-295): the squared gap components.
template <class Prob>
GP_LM_INNER void lm_fcn(const Prob& P, const double x[2], double fvec[3], SupportEval& E) {
  double pt1[3], pt2[3];
  support_eval(P, x, E, pt1, pt2);
#pragma unroll
  for (int i = 0; i < 3; ++i) fvec[i] = E.depth[i] * E.depth[i];
}

// d(support point)/dc = E/(2 lambda) - (E c)(E c)^T / (8 lambda^3), with s = 1/(2 lambda);
// E (outer) in matmul's order of terms.
template <int W, class Prob>
GP_LM_INNER void grad_coeff(const Prob& P, const double c[3], double l, double s, double co[9]) {
  double row[3];
#pragma unroll
  for (int j = 0; j < 3; ++j)
    row[j] = c[0] * P.template e<W>(3 * j) + c[1] * P.template e<W>(1 + 3 * j) + c[2] * P.template e<W>(2 + 3 * j);
  double outer[9];
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int i = 0; i < 3; ++i) outer[i + 3 * j] = c[i] * row[j];
  double eo[9];
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int i = 0; i < 3; ++i)
      eo[i + 3 * j] = P.template e<W>(i) * outer[3 * j] + P.template e<W>(i + 3) * outer[1 + 3 * j] +
                      P.template e<W>(i + 6) * outer[2 + 3 * j];
  const double t = lm_div(1.0, 8.0 * (l * l * l));   // lambda**3.0
#pragma unroll
  for (int k = 0; k < 9; ++k) co[k] = s * P.template e<W>(k) - t * eo[k];
}

// fcn, iflag=2: analytic Jacobian (ellipsoid_contact_detection.f90:296-332), 3x2
// column-major, at the point whose residual produced E.
template <class Prob>
GP_LM_INNER void lm_jac(const Prob& P, const SupportEval& E, double fj[6]) {
  const double g[6] = {-E.s0 * E.k1, E.k0 * E.k1, 0.0, -E.k0 * E.s1, -E.s0 * E.s1, E.k1};
  const double c1[3] = {E.k0 * E.k1, E.s0 * E.k1, E.s1};
  const double c2[3] = {-c1[0], -c1[1], -c1[2]};
  double co1[9], co2[9];
  grad_coeff<0>(P, c1, E.l1, E.f1, co1);
  grad_coeff<1>(P, c2, E.l2, E.f2, co2);
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const double gj[3] = {g[3 * j], g[3 * j + 1], g[3 * j + 2]};
    const double ng[3] = {-gj[0], -gj[1], -gj[2]};
    double gp1[3], gp2[3];
    matvec(co1, gj, gp1);
    matvec(co2, ng, gp2);
#pragma unroll
    for (int i = 0; i < 3; ++i) fj[i + 3 * j] = 2.0 * (E.depth[i] * (gp1[i] - gp2[i]));
  }
}

// The column pivot of the 3x2 QR is either the identity or the swap; `sw` records the
// swap (MINPACK's ipvt = (2, 1)).  sel(sw, a, b) is element ipvt[j] of a two-vector
// (a, b) for j = 0, and sel(!sw, a, b) for j = 1; keeping the pivot as a flag lets every
// index be a compile-time constant, so the solver's state stays in registers.
__device__ __forceinline__ double sel(bool sw, double a, double b) { return sw ? b : a; }

// QR with column pivoting (3x2), Householder vectors left in a.
GP_LM_INNER void lm_qrfac(double a[6], bool& sw, double rdiag[2], double acnorm[2]) {
  double wa[2];
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    acnorm[j] = lm_enorm<3>(a + 3 * j);
    rdiag[j] = acnorm[j];
    wa[j] = rdiag[j];
  }
  sw = false;
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    if (j == 0 && rdiag[1] > rdiag[0]) {
#pragma unroll
      for (int i = 0; i < 3; ++i) { const double t = a[i]; a[i] = a[i + 3]; a[i + 3] = t; }
      rdiag[1] = rdiag[0];
      wa[1] = wa[0];
      sw = true;
    }
    double ajnorm = (j == 0) ? lm_enorm<3>(a) : lm_enorm<2>(a + 4);
    if (ajnorm != 0.0) {
      if (a[j + 3 * j] < 0.0) ajnorm = -ajnorm;
#pragma unroll
      for (int i = j; i < 3; ++i) a[i + 3 * j] = lm_div(a[i + 3 * j], ajnorm);
      a[j + 3 * j] = a[j + 3 * j] + 1.0;
      if (j == 0) {
        double sum = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i) sum = sum + a[i] * a[i + 3];
        const double temp = lm_div(sum, a[0]);
#pragma unroll
        for (int i = 0; i < 3; ++i) a[i + 3] = a[i + 3] - temp * a[i];
        if (rdiag[1] != 0.0) {
          const double t2 = lm_div(a[3], rdiag[1]);
          const double f = 1.0 - t2 * t2;
          rdiag[1] = rdiag[1] * lm_sqrt(f > 0.0 ? f : 0.0);
          const double r = lm_div(rdiag[1], wa[1]);
          if (0.05 * (r * r) <= DBL_EPSILON) {
            rdiag[1] = lm_enorm<2>(a + 4);
            wa[1] = rdiag[1];
          }
        }
      }
    }
    rdiag[j] = -ajnorm;
  }
}

GP_LM_INNER void lm_qrsolv(double r[6], bool sw, const double diag[2], const double qtb[2], double x[2],
                           double sdiag[2]) {
  double wa[2];
#pragma unroll
  for (int j = 0; j < 2; ++j) {
#pragma unroll
    for (int i = j; i < 2; ++i) r[i + 3 * j] = r[j + 3 * i];
    x[j] = r[j + 3 * j];
    wa[j] = qtb[j];
  }
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const double dl = (j == 0) ? sel(sw, diag[0], diag[1]) : sel(!sw, diag[0], diag[1]);
    if (dl != 0.0) {
#pragma unroll
      for (int k = j; k < 2; ++k) sdiag[k] = 0.0;
      sdiag[j] = dl;
      double qtbpj = 0.0;
#pragma unroll
      for (int k = j; k < 2; ++k) {
        if (sdiag[k] == 0.0) continue;
        double cs, sn;
        if (fabs(r[k + 3 * k]) >= fabs(sdiag[k])) {
          const double tn = lm_div(sdiag[k], r[k + 3 * k]);
          cs = lm_div(0.5, lm_sqrt(0.25 + 0.25 * (tn * tn)));
          sn = cs * tn;
        } else {
          const double ct = lm_div(r[k + 3 * k], sdiag[k]);
          sn = lm_div(0.5, lm_sqrt(0.25 + 0.25 * (ct * ct)));
          cs = sn * ct;
        }
        r[k + 3 * k] = cs * r[k + 3 * k] + sn * sdiag[k];
        const double temp = cs * wa[k] + sn * qtbpj;
        qtbpj = -sn * wa[k] + cs * qtbpj;
        wa[k] = temp;
        if (k == 0) {
          const double t2 = cs * r[1] + sn * sdiag[1];
          sdiag[1] = -sn * r[1] + cs * sdiag[1];
          r[1] = t2;
        }
      }
    }
    sdiag[j] = r[j + 3 * j];
    r[j + 3 * j] = x[j];
  }
  int nsing = 2;
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    if (sdiag[j] == 0.0 && nsing == 2) nsing = j;
    if (nsing < 2) wa[j] = 0.0;
  }
  if (nsing >= 2) wa[1] = lm_div(wa[1], sdiag[1]);
  if (nsing >= 1) {
    double sum = 0.0;
    if (nsing >= 2) sum = sum + r[1] * wa[1];
    wa[0] = lm_div(wa[0] - sum, sdiag[0]);
  }
  // x[ipvt[j]] = wa[j]
  x[0] = sel(sw, wa[0], wa[1]);
  x[1] = sel(sw, wa[1], wa[0]);
}

GP_LM_INNER void lm_lmpar(double r[6], bool sw, const double diag[2], const double qtb[2], double delta,
                          double& par, double x[2], double sdiag[2]) {
  const double dwarf = DBL_MIN;
  double wa1[2], wa2[2];
  int nsing = 2;
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    wa1[j] = qtb[j];
    if (r[j + 3 * j] == 0.0 && nsing == 2) nsing = j;
    if (nsing < 2) wa1[j] = 0.0;
  }
  if (nsing >= 2) {
    wa1[1] = lm_div(wa1[1], r[4]);
    wa1[0] = wa1[0] - r[3] * wa1[1];
  }
  if (nsing >= 1) wa1[0] = lm_div(wa1[0], r[0]);
  x[0] = sel(sw, wa1[0], wa1[1]);
  x[1] = sel(sw, wa1[1], wa1[0]);
  wa2[0] = diag[0] * x[0];
  wa2[1] = diag[1] * x[1];
  double dxnorm = lm_enorm<2>(wa2);
  double fp = dxnorm - delta;
  if (fp <= 0.1 * delta) {
    par = 0.0;
    return;
  }
  // diag and wa2 in pivot order: element ipvt[j] for j = 0, 1
  const double dp0 = sel(sw, diag[0], diag[1]), dp1 = sel(!sw, diag[0], diag[1]);
  double parl = 0.0;
  if (nsing >= 2) {
    wa1[0] = dp0 * lm_div(sel(sw, wa2[0], wa2[1]), dxnorm);
    wa1[1] = dp1 * lm_div(sel(!sw, wa2[0], wa2[1]), dxnorm);
    wa1[0] = lm_div(wa1[0] - 0.0, r[0]);
    wa1[1] = lm_div(wa1[1] - (0.0 + r[3] * wa1[0]), r[4]);
    const double temp = lm_enorm<2>(wa1);
    parl = lm_div(lm_div(lm_div(fp, delta), temp), temp);
  }
  {
    const double s0 = 0.0 + r[0] * qtb[0];
    const double s1 = (0.0 + r[3] * qtb[0]) + r[4] * qtb[1];
    wa1[0] = lm_div(s0, dp0);
    wa1[1] = lm_div(s1, dp1);
  }
  const double gnorm = lm_enorm<2>(wa1);
  double paru = lm_div(gnorm, delta);
  if (paru == 0.0) paru = lm_div(dwarf, delta < 0.1 ? delta : 0.1);
  double p = par;
  p = (p > parl) ? p : parl;
  p = (p < paru) ? p : paru;
  if (p == 0.0) p = lm_div(gnorm, dxnorm);
  for (int iter = 1;; ++iter) {
    if (p == 0.0) { const double t = 0.001 * paru; p = (dwarf > t) ? dwarf : t; }
    const double sp = lm_sqrt(p);
    wa1[0] = sp * diag[0];
    wa1[1] = sp * diag[1];
    lm_qrsolv(r, sw, wa1, qtb, x, sdiag);
    wa2[0] = diag[0] * x[0];
    wa2[1] = diag[1] * x[1];
    dxnorm = lm_enorm<2>(wa2);
    const double told = fp;
    fp = dxnorm - delta;
    if (fabs(fp) <= 0.1 * delta || (parl == 0.0 && fp <= told && told < 0.0) || iter == 10) break;
    wa1[0] = dp0 * lm_div(sel(sw, wa2[0], wa2[1]), dxnorm);
    wa1[1] = dp1 * lm_div(sel(!sw, wa2[0], wa2[1]), dxnorm);
    wa1[0] = lm_div(wa1[0], sdiag[0]);
    wa1[1] = wa1[1] - r[1] * wa1[0];
    wa1[1] = lm_div(wa1[1], sdiag[1]);
    const double temp = lm_enorm<2>(wa1);
    const double parc = lm_div(lm_div(lm_div(fp, delta), temp), temp);
    if (fp > 0.0) parl = (parl > p) ? parl : p;
    if (fp < 0.0) paru = (paru < p) ? paru : p;
    const double t2 = p + parc;
    p = (parl > t2) ? parl : t2;
  }
  par = p;
}

// lmder (minpack_reduc.f90:243-640) as a resumable state machine: lm_begin evaluates
// the residual at the starting point; each lm_step runs, when the previous trial was
// accepted (or at the start), the Jacobian/QR block of lmder's outer loop, then one
// trial step of its inner loop, and returns 0 to continue or lmder's info code (8
// mapped to 4 as lmder1 does) when lmder would return.  The sequence of operations per
// pair is lmder's; the split lets a warp refill a lane with a new pair as soon as its
// pair converges.
struct LmState {
  double x[2], fjac[6], diag[2], qtf[2];
  double fnorm, xnorm, delta, par, temp, gnorm;
  SupportEval E;   // residual evaluation at x (for the next Jacobian; fvec = E.depth^2)
  int nfev, iter;
  bool swapped;    // column pivot of the last QR: ipvt = (2, 1)
  bool need_jac;
};

template <class Prob>
GP_LM_FN void lm_begin(const Prob& P, LmState& S) {
  double fvec[3];
  lm_fcn(P, S.x, fvec, S.E);
  S.nfev = 1;
  S.fnorm = lm_enorm<3>(fvec);
  S.par = 0.0;
  S.iter = 1;
  S.xnorm = 0.0;
  S.delta = 0.0;
  S.temp = 0.0;
  S.gnorm = 0.0;
  S.diag[0] = S.diag[1] = 0.0;
  S.swapped = false;
  S.need_jac = true;
}

template <class Prob>
GP_LM_FN int lm_step(const Prob& P, LmState& S, double tol) {
  constexpr int maxfev = 300;
  const double ftol = tol, xtol = tol;
  double wa1[2], wa2[2], wa3[2], wa4[3];
  if (S.need_jac) {
    lm_jac(P, S.E, S.fjac);
    lm_qrfac(S.fjac, S.swapped, wa1, wa2);
    if (S.iter == 1) {
#pragma unroll
      for (int j = 0; j < 2; ++j) { S.diag[j] = wa2[j]; if (wa2[j] == 0.0) S.diag[j] = 1.0; }
      wa3[0] = S.diag[0] * S.x[0];
      wa3[1] = S.diag[1] * S.x[1];
      S.xnorm = lm_enorm<2>(wa3);
      S.delta = 100.0 * S.xnorm;
      if (S.delta == 0.0) S.delta = 100.0;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) wa4[i] = S.E.depth[i] * S.E.depth[i];   // fvec at x
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      if (S.fjac[j + 3 * j] != 0.0) {
        double sum = 0.0;
#pragma unroll
        for (int i = j; i < 3; ++i) sum = sum + S.fjac[i + 3 * j] * wa4[i];
        const double t = lm_div(-sum, S.fjac[j + 3 * j]);
#pragma unroll
        for (int i = j; i < 3; ++i) wa4[i] = wa4[i] + S.fjac[i + 3 * j] * t;
      }
      S.fjac[j + 3 * j] = wa1[j];
      S.qtf[j] = wa4[j];
    }
    double gnorm = 0.0;
    if (S.fnorm != 0.0) {
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        // acnorm of the original column ipvt[j]
        const double acn = (j == 0) ? sel(S.swapped, wa2[0], wa2[1]) : sel(!S.swapped, wa2[0], wa2[1]);
        if (acn != 0.0) {
          double sum = 0.0;
#pragma unroll
          for (int i = 0; i <= j; ++i) sum = sum + S.fjac[i + 3 * j] * lm_div(S.qtf[i], S.fnorm);
          const double g = fabs(lm_div(sum, acn));
          gnorm = (gnorm > g) ? gnorm : g;
        }
      }
    }
    S.gnorm = gnorm;
    if (gnorm <= 0.0) return 4;
    S.diag[0] = (S.diag[0] > wa2[0]) ? S.diag[0] : wa2[0];
    S.diag[1] = (S.diag[1] > wa2[1]) ? S.diag[1] : wa2[1];
    S.need_jac = false;
  }
  // one trial step (the body of lmder's inner loop)
  lm_lmpar(S.fjac, S.swapped, S.diag, S.qtf, S.delta, S.par, wa1, wa2);
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    wa1[j] = -wa1[j];
    wa2[j] = S.x[j] + wa1[j];
    wa3[j] = S.diag[j] * wa1[j];
  }
  const double pnorm = lm_enorm<2>(wa3);
  if (S.iter == 1) S.delta = (S.delta < pnorm) ? S.delta : pnorm;
  SupportEval E2;
  lm_fcn(P, wa2, wa4, E2);
  ++S.nfev;
  const double fnorm1 = lm_enorm<3>(wa4);
  double actred = -1.0;
  if (0.1 * fnorm1 < S.fnorm) { const double r = lm_div(fnorm1, S.fnorm); actred = 1.0 - r * r; }
  // wa1 in pivot order: element ipvt[j]
  const double p0 = sel(S.swapped, wa1[0], wa1[1]);
  const double p1 = sel(!S.swapped, wa1[0], wa1[1]);
  wa3[0] = 0.0 + S.fjac[0] * p0;
  wa3[1] = 0.0;
  wa3[0] = wa3[0] + S.fjac[3] * p1;
  wa3[1] = wa3[1] + S.fjac[4] * p1;
  const double temp1 = lm_div(lm_enorm<2>(wa3), S.fnorm);
  const double temp2 = lm_div(lm_sqrt(S.par) * pnorm, S.fnorm);
  const double prered = temp1 * temp1 + (temp2 * temp2) / 0.5;
  const double dirder = -(temp1 * temp1 + temp2 * temp2);
  double ratio = 0.0;
  if (prered != 0.0) ratio = lm_div(actred, prered);
  if (ratio <= 0.25) {
    if (actred >= 0.0) S.temp = 0.5;
    if (actred < 0.0) S.temp = lm_div(0.5 * dirder, dirder + 0.5 * actred);
    if (0.1 * fnorm1 >= S.fnorm || S.temp < 0.1) S.temp = 0.1;
    const double pt = lm_div(pnorm, 0.1);
    const double m = (S.delta < pt) ? S.delta : pt;
    S.delta = S.temp * m;
    S.par = lm_div(S.par, S.temp);
  } else if (S.par == 0.0 || ratio >= 0.75) {
    S.delta = pnorm / 0.5;
    S.par = 0.5 * S.par;
  }
  if (ratio >= 1.0e-4) {
#pragma unroll
    for (int j = 0; j < 2; ++j) { S.x[j] = wa2[j]; wa2[j] = S.diag[j] * S.x[j]; }
    S.E = E2;
    S.xnorm = lm_enorm<2>(wa2);
    S.fnorm = fnorm1;
    ++S.iter;
  }
  int info = 0;
  if (fabs(actred) <= ftol && prered <= ftol && 0.5 * ratio <= 1.0) info = 1;
  if (S.delta <= xtol * S.xnorm) info = 2;
  if (fabs(actred) <= ftol && prered <= ftol && 0.5 * ratio <= 1.0 && info == 2) info = 3;
  if (info != 0) return info;
  if (S.nfev >= maxfev) info = 5;
  if (fabs(actred) <= DBL_EPSILON && prered <= DBL_EPSILON && 0.5 * ratio <= 1.0) info = 6;
  if (S.delta <= DBL_EPSILON * S.xnorm) info = 7;
  if (S.gnorm <= DBL_EPSILON) info = 8;
  if (info != 0) return info == 8 ? 4 : info;
  if (ratio >= 1.0e-4) S.need_jac = true;
  return 0;
}

// Margin function mod_particle_parallel.f90:145-201: v^T (R diag(1/a^2,1/b^2,1/b^2) R^T) v
// Separating-direction test for two spheroids whose bounding spheres overlap and whose
// extents along the centre line do too.  With support functions
// h_i(n) = sqrt(b_i^2 + (a_i^2 - b_i^2) (e_i.n)^2), the bodies are disjoint if some unit
// n has g(n) = n.d - h_1(n) - h_2(n) > 0 (d from body 1 to body 2).  g is concave, so
// a few projected-gradient steps from the centre line (the best of four step lengths
// each) find such an n for nearly every disjoint pair.  Disjoint bodies cannot hold
// each other's support points, so ellipsoid_contact_detection.f90:125 cannot flag the
// pair.  The test runs in FP32: its rounding moves g by about 1e-6 of its terms (the
// inputs rounded to FP32, 3-term dot products, square roots, a unit vector normalised
// to 1e-7), so g must exceed 1e-4 of its terms, and a pair is dropped only when it is
// disjoint; pairs closer than that to touching are left to the solver, as are pairs
// whose g turns NaN.  It never decides a contact, so its precision changes which pairs
// are solved, not a result.
static __device__ __forceinline__ float support_gap(const float n[3], const float d[3], const float e1[3],
                                                    float a1, float b1, const float e2[3], float a2, float b2,
                                                    float &h1, float &h2, float &c1, float &c2) {
  c1 = e1[0] * n[0] + e1[1] * n[1] + e1[2] * n[2];
  c2 = e2[0] * n[0] + e2[1] * n[1] + e2[2] * n[2];
  h1 = sqrtf(fmaxf(b1 + (a1 - b1) * c1 * c1, 0.f));
  h2 = sqrtf(fmaxf(b2 + (a2 - b2) * c2 * c2, 0.f));
  return n[0] * d[0] + n[1] * d[1] + n[2] * d[2] - h1 - h2;
}

// (dx, dy, dz): centre of body 2 minus centre of body 1; e1, e2 unit axes; a, b the
// squared semi-axes along and across the axis.
static __device__ __noinline__ bool separated(double dx, double dy, double dz, const double e1d[3], double a1d,
                                              double b1d, const double e2d[3], double a2d, double b2d) {
  const float d[3] = {(float)dx, (float)dy, (float)dz};
  const float e1[3] = {(float)e1d[0], (float)e1d[1], (float)e1d[2]};
  const float e2[3] = {(float)e2d[0], (float)e2d[1], (float)e2d[2]};
  const float a1 = (float)a1d, b1 = (float)b1d, a2 = (float)a2d, b2 = (float)b2d;
  const float dist = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  if (!(dist > 0.f)) return false;
  const float idist = __frcp_rn(dist);
  float n[3] = {d[0] * idist, d[1] * idist, d[2] * idist};
  float h1, h2, c1, c2;
  float g = support_gap(n, d, e1, a1, b1, e2, a2, b2, h1, h2, c1, c2);
  for (int it = 0; it < 4; ++it) {
    // gradient of g: d - E1 n / h1 - E2 n / h2, with E n = b^2 n + (a^2 - b^2)(e.n) e
    const float i1 = __frcp_rn(h1), i2 = __frcp_rn(h2);
    float gr[3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
      gr[k] = d[k] - (b1 * n[k] + (a1 - b1) * c1 * e1[k]) * i1 - (b2 * n[k] + (a2 - b2) * c2 * e2[k]) * i2;
    const float gn = gr[0] * n[0] + gr[1] * n[1] + gr[2] * n[2];
    const float t[3] = {(gr[0] - gn * n[0]) * idist, (gr[1] - gn * n[1]) * idist, (gr[2] - gn * n[2]) * idist};
    float best = -3.0e38f, bn[3] = {n[0], n[1], n[2]}, bh1 = h1, bh2 = h2, bc1 = c1, bc2 = c2;
#pragma unroll
    for (int ka = 0; ka < 4; ++ka) {
      const float alpha = 0.25f * (float)(1 << ka);
      float m[3] = {n[0] + alpha * t[0], n[1] + alpha * t[1], n[2] + alpha * t[2]};
      const float inv = rsqrtf(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
      m[0] *= inv; m[1] *= inv; m[2] *= inv;
      float mh1, mh2, mc1, mc2;
      const float gm = support_gap(m, d, e1, a1, b1, e2, a2, b2, mh1, mh2, mc1, mc2);
      if (gm > best) {
        best = gm;
        bn[0] = m[0]; bn[1] = m[1]; bn[2] = m[2];
        bh1 = mh1; bh2 = mh2; bc1 = mc1; bc2 = mc2;
      }
    }
    if (!(best > g)) return false;   // no progress (or NaN): keep the pair
    n[0] = bn[0]; n[1] = bn[1]; n[2] = bn[2];
    h1 = bh1; h2 = bh2; c1 = bc1; c2 = bc2;
    g = best;
    const float scale = fabsf(n[0] * d[0] + n[1] * d[1] + n[2] * d[2]) + h1 + h2;
    if (g > 1.0e-4f * scale) return true;
  }
  return false;
}

GP_LM_COLD double fmargin(double a, double b, const double pt[3], const double c[3], const Quat& q) {
  double ell[9];
  rot_diag(q, 1.0 / (a * a), 1.0 / (b * b), 1.0 / (b * b), ell);
  const double v[3] = {pt[0] - c[0], pt[1] - c[1], pt[2] - c[2]};
  double e_[3];
  matvec(ell, v, e_);
  return v[0] * e_[0] + v[1] * e_[1] + v[2] * e_[2];
}

// Set-up of ellipsoid_contact_detection.f90:72-95: the two rotated ellipsoid matrices
// and the starting angles from the centre line (:77-87).  Returns false when a starting
// angle is NaN (acos of a ratio just above 1): every iterate would stay NaN and the
// reference reports no contact, so the caller skips the solve.
GP_LM_FN bool contact_setup(double a1, double bb1, double a2, double bb2, const double c1[3],
                                                  const Quat& q1, const double c2[3], const Quat& q2, ContactProb& P,
                                                  double x[2]) {
  double nrm[3] = {c1[0] - c2[0], c1[1] - c2[1], c1[2] - c2[2]};
  const double c_norm = sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
  if (c_norm != 0.0) { nrm[0] = nrm[0] / c_norm; nrm[1] = nrm[1] / c_norm; nrm[2] = nrm[2] / c_norm; }
  x[1] = ct_asin(nrm[2]);
  x[0] = ct_acos(nrm[0] / ct_cos(x[1]));
  rot_diag(q1, a1 * a1, bb1 * bb1, bb1 * bb1, P.e1);
  rot_diag(q2, a2 * a2, bb2 * bb2, bb2 * bb2, P.e2);
#pragma unroll
  for (int i = 0; i < 3; ++i) { P.b1[i] = c1[i]; P.b2[i] = c2[i]; }
  return !(x[0] != x[0] || x[1] != x[1]);
}

// pair_depth at the solution and the contact test (ellipsoid_contact_detection.f90:104-179)
GP_LM_COLD bool contact_finish(double a1, double bb1, double a2, double bb2, const Quat& q1,
                                                   const Quat& q2, const ContactProb& P, const double x[2],
                                                   double ept1[3], double ept2[3], double cn[3]) {
  double cc[3], pt1[3], pt2[3];
  support_points(P, x, cc, pt1, pt2);
  const double d[3] = {pt1[0] - pt2[0], pt1[1] - pt2[1], pt1[2] - pt2[2]};
  const double contact = d[0] * cc[0] + d[1] * cc[1] + d[2] * cc[2];
#pragma unroll
  for (int i = 0; i < 3; ++i) { ept1[i] = pt1[i]; ept2[i] = pt2[i]; cn[i] = cc[i]; }
  return (contact > 0) && (fmargin(a1, bb1, pt2, P.b1, q1) < 1.0) && (fmargin(a2, bb2, pt1, P.b2, q2) < 1.0);
}

constexpr double kContactTol = 1.4901161193847656e-08;   // sqrt(epsilon(1.0_8))

// ellipsoid_contact_detection.f90:1-187 for one pair, start to finish.
GP_LM_FN bool contact_detection(double a1, double bb1, double a2, double bb2,
                                                      const double c1[3], const Quat& q1, const double c2[3],
                                                      const Quat& q2, double ept1[3], double ept2[3], double cn[3]) {
  ContactProb P;
  LmState S;
  if (!contact_setup(a1, bb1, a2, bb2, c1, q1, c2, q2, P, S.x)) {
#pragma unroll
    for (int i = 0; i < 3; ++i) { ept1[i] = CUDART_NAN; ept2[i] = CUDART_NAN; cn[i] = CUDART_NAN; }
    return false;
  }
  lm_begin(P, S);
  while (lm_step(P, S, kContactTol) == 0) {
  }
  return contact_finish(a1, bb1, a2, bb2, q1, q2, P, S.x, ept1, ept2, cn);
}

}  // namespace gp
