// gp_kernels_fp64.cu -- FP64 kernels compiled without FMA contraction (-fmad=false),
// so that every rounded operation matches an IEEE restatement of the reference:
// the fused ADV_PARTICLE_ELLP step, the interpolation drop-ins, the contact solve and
// the collision response, and the per-routine batched entry points.
#include <math_constants.h>

#include "gp_advance.cuh"
#include "gp_lm.cuh"
#include "gp_launch.h"

namespace gp {

template __global__ void k_integrate<false>(const InstDev *, const PoolView *, const PoolView *, const int32_t *,
                                            int64_t, const double *const *, uint32_t *, Status *);
template __global__ void k_integrate_fix<false>(const InstDev *, const PoolView *, const PoolView *, const PairRec *,
                                                const unsigned long long *, int64_t, const double *const *,
                                                uint32_t *, Status *);
template __global__ void k_gather<false>(const InstDev *, const PoolView *, const int32_t *, int64_t,
                                         double *const *, unsigned long long *, Status *);

void launch_gather_fp64(const InstDev *insts, const PoolView *pv, const int32_t *perm, int64_t n,
                      double *const *fluid, unsigned long long *ticket, Status *st, int grid, cudaStream_t s) {
  cudaMemsetAsync(ticket, 0, sizeof(unsigned long long), s);
  k_gather<false><<<grid, 256, 0, s>>>(insts, pv, perm, n, fluid, ticket, st);
}

void launch_integrate_fp64(const InstDev *insts, PoolView *pv, PoolView *pv_alt, const int32_t *perm, int64_t n,
                         double *const *fluid, Status *st, int grid, cudaStream_t s, uint32_t *mark) {
  k_integrate<false><<<grid, 128, 0, s>>>(insts, pv, pv_alt, perm, n, fluid, mark, st);
  if (mark == nullptr) k_swap_pool<<<1, 1, 0, s>>>(pv, pv_alt, st);
}

void launch_integrate_fix_fp64(const InstDev *insts, PoolView *pv, PoolView *pv_alt, const PairRec *pairs,
                             const unsigned long long *npairs, int64_t cap_pairs, double *const *fluid,
                             uint32_t *mark, Status *st, int grid, cudaStream_t s) {
  k_integrate_fix<false><<<grid, 128, 0, s>>>(insts, pv, pv_alt, pairs, npairs, cap_pairs, fluid, mark, st);
  k_swap_pool<<<1, 1, 0, s>>>(pv, pv_alt, st);
}

// INTERP_LAG3 (interp_lag3.f90:11-298) for one component at arbitrary points.
__global__ void k_interp(const InstDev *__restrict__ inst, int comp, int64_t n, const double *__restrict__ x,
                         const double *__restrict__ y, const double *__restrict__ z, double *__restrict__ out,
                         Status *st) {
  const InstDev I = *inst;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    Stencil s;
    if (!stencil(I, x[p], y[p], z[p], s)) {
      out[p] = CUDART_NAN;
      set_error(st, GP_EOUT_OF_GRID, p);
      continue;
    }
    double g[6];
    if (I.fprec == GP_PREC_MIXED) gather6_fp32(I, s, g); else gather6_fp64(I, s, g);
    out[p] = g[comp];
  }
}

void launch_interp(const InstDev *inst, int comp, int64_t n, const double *x, const double *y, const double *z,
                   double *out, Status *st, cudaStream_t s) {
  if (n <= 0) return;
  const int grid = (int)((n + 255) / 256 < 148 * 16 ? (n + 255) / 256 : 148 * 16);
  k_interp<<<grid, 256, 0, s>>>(inst, comp, n, x, y, z, out, st);
}

// FROZEN_INTERP_LAG3 (frozen_interp_lag3.f90:11-274): plain (NX,NY,NZ) array, mirror
// boundaries (the JP2 test compares with NZ, as the reference does at :148).
__global__ void k_frozen_interp(const double *__restrict__ xain, const double *__restrict__ yain,
                                const double *__restrict__ zain, int nx, int ny, int nz,
                                const double *__restrict__ uain, int64_t n, const double *__restrict__ xi,
                                const double *__restrict__ yi, const double *__restrict__ zi,
                                double *__restrict__ out, Status *st) {
  const double dxa = xain[1] - xain[0], dya = yain[1] - yain[0], dza = zain[1] - zain[0];
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    const double fx = xi[p] / dxa, fy = yi[p] / dya, fz = zi[p] / dza;
    bool bad = !(fx > -2.0 && fx < 2147483000.0 && fy > -2.0 && fy < 2147483000.0 && fz > -2.0 && fz < 2147483000.0);
    int i0 = 0, j0 = 0, k0 = 0;
    if (!bad) { i0 = (int)fx + 1; j0 = (int)fy + 1; k0 = (int)fz + 1; }
    int ip1 = i0 + 1; if (i0 == nx) ip1 = nx - 1;
    int ip2 = ip1 + 1; if (ip1 == nx) ip2 = nx - 1;
    int im1 = i0 - 1; if (i0 == 1) im1 = 2;
    int jm1 = j0 - 1; if (j0 == 1) jm1 = 2;
    int jp1 = j0 + 1; if (j0 == ny) jp1 = ny - 1;
    int jp2 = jp1 + 1; if (jp1 == nz) jp2 = ny - 1;
    int km1 = k0 - 1; if (k0 == 1) km1 = 2;
    int kp1 = k0 + 1; if (k0 == nz) kp1 = nz - 1;
    int kp2 = kp1 + 1; if (kp1 == nz) kp2 = nz - 1;
    const int ix[4] = {im1, i0, ip1, ip2}, jy[4] = {jm1, j0, jp1, jp2}, kz[4] = {km1, k0, kp1, kp2};
#pragma unroll
    for (int t = 0; t < 4; ++t)
      if (ix[t] < 1 || ix[t] > nx || jy[t] < 1 || jy[t] > ny || kz[t] < 1 || kz[t] > nz) bad = true;
    if (bad) {
      out[p] = CUDART_NAN;
      set_error(st, GP_EOUT_OF_GRID, p);
      continue;
    }
    double wx[4], wy[4], wz[4];
    lag3_w((xi[p] - xain[i0 - 1]) / dxa, wx);
    lag3_w((yi[p] - yain[j0 - 1]) / dya, wy);
    lag3_w((zi[p] - zain[k0 - 1]) / dza, wz);
    double zs = 0.0;
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      double ys = 0.0;
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) {
        const int64_t row = ((int64_t)(kz[kk] - 1) * ny + (jy[jj] - 1)) * (int64_t)nx;
        const double xs = wx[0] * uain[row + ix[0] - 1] + wx[1] * uain[row + ix[1] - 1] +
                          wx[2] * uain[row + ix[2] - 1] + wx[3] * uain[row + ix[3] - 1];
        ys = (jj == 0) ? wy[0] * xs : ys + wy[jj] * xs;
      }
      zs = (kk == 0) ? wz[0] * ys : zs + wz[kk] * ys;
    }
    out[p] = zs;
  }
}

void launch_frozen_interp(const double *xain, const double *yain, const double *zain, int nx, int ny, int nz,
                          const double *uain, int64_t n, const double *x, const double *y, const double *z,
                          double *out, Status *st, cudaStream_t s) {
  if (n <= 0) return;
  const int grid = (int)((n + 255) / 256 < 148 * 16 ? (n + 255) / 256 : 148 * 16);
  k_frozen_interp<<<grid, 256, 0, s>>>(xain, yain, zain, nx, ny, nz, uain, n, x, y, z, out, st);
}

// COLLISION_RESPONSE (collision_response.f90) for the accepted pairs; each particle is
// in at most one accepted pair.
__global__ void k_response(const InstDev *__restrict__ insts, const PoolView *__restrict__ pv,
                           const CollRec *__restrict__ coll, const unsigned long long *__restrict__ ncoll,
                           int64_t cap_coll, const int8_t *__restrict__ state, int32_t *acc_list,
                           unsigned long long *nacc, Status *st) {
  if (step_halted(st)) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&st->steps_done, 1ull);
  const PoolView P = *pv;
  const int64_t nc = (int64_t)min(*ncoll, (unsigned long long)cap_coll);
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nc; e += (int64_t)gridDim.x * blockDim.x) {
    if (state[e] != 1) continue;
    const CollRec r = coll[e];
    const int i1 = r.home, i2 = r.near;
    const InstDev &I = insts[P.inst[i1]];
    double u1[3] = {P.st[3][i1], P.st[4][i1], P.st[5][i1]}, o1[3] = {P.st[10][i1], P.st[11][i1], P.st[12][i1]};
    double u2[3] = {P.st[3][i2], P.st[4][i2], P.st[5][i2]}, o2[3] = {P.st[10][i2], P.st[11][i2], P.st[12][i2]};
    const Quat q1 = {P.st[6][i1], P.st[7][i1], P.st[8][i1], P.st[9][i1]};
    const Quat q2 = {P.st[6][i2], P.st[7][i2], P.st[8][i2], P.st[9][i2]};
    const int rc = collision_response(I.ecp, I.mup, P.pc[7][i1], P.pc[8][i1], P.pc[9][i1], u1, o1, q1, u2, o2, q2,
                                      r.rx1, r.rx2, r.cn);
    if (rc) set_error(st, rc, (long long)P.id[i1], P.inst[i1]);
    P.st[3][i1] = u1[0]; P.st[4][i1] = u1[1]; P.st[5][i1] = u1[2];
    P.st[10][i1] = o1[0]; P.st[11][i1] = o1[1]; P.st[12][i1] = o1[2];
    P.st[3][i2] = u2[0]; P.st[4][i2] = u2[1]; P.st[5][i2] = u2[2];
    P.st[10][i2] = o2[0]; P.st[11][i2] = o2[1]; P.st[12][i2] = o2[2];
    const unsigned long long k = atomicAdd(nacc, 1ull);
    if (acc_list != nullptr && (int64_t)k < cap_coll) acc_list[k] = (int32_t)e;
  }
}

void launch_response(const InstDev *insts, const PoolView *pv, const CollRec *coll, const unsigned long long *ncoll,
                     int64_t cap_coll, const int8_t *state, int32_t *acc_list, unsigned long long *nacc, Status *st,
                     int grid, cudaStream_t s) {
  k_response<<<grid, 128, 0, s>>>(insts, pv, coll, ncoll, cap_coll, state, acc_list, nacc, st);
}

// ---------------------------------------------------------------------------
// Per-routine batched entry points
// ---------------------------------------------------------------------------
__device__ __forceinline__ PartConst pc_from(const double *pcs, int64_t i) {
  const double *c = pcs + 10 * i;
  PartConst pc;
  pc.a = c[0]; pc.b = c[1]; pc.deq = c[2]; pc.cdrag = c[3]; pc.cpitch = c[4];
  pc.crot = c[5]; pc.h5 = c[6]; pc.ipxx = c[7]; pc.ipyy = c[8]; pc.ipzz = c[9];
  return pc;
}

__global__ void k_force_batch(int64_t n, const double *pcs, double visc, const double *up, const double *uf,
                              const double *quat, double *fdrag, double *flift, Status *st) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const PartConst pc = pc_from(pcs, i);
    const Quat q = {quat[4 * i], quat[4 * i + 1], quat[4 * i + 2], quat[4 * i + 3]};
    double r[9];
    rotmat(q, r);
    Slip64 sl;
    slip64(pc, visc, up + 3 * i, uf + 3 * i, r, sl);
    double fd[3], fl[3];
    if (!fluid_force(pc, sl, r, fd, fl)) set_error(st, GP_ENAN_FORCE, i);
#pragma unroll
    for (int k = 0; k < 3; ++k) { fdrag[3 * i + k] = fd[k]; flift[3 * i + k] = fl[k]; }
  }
}

__global__ void k_torque_batch(int64_t n, const double *pcs, double visc, const double *om, const double *quat,
                               const double *pup, const double *pufap, const double *pvort, double *tp, double *tr,
                               Status *st) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const PartConst pc = pc_from(pcs, i);
    const Quat q = {quat[4 * i], quat[4 * i + 1], quat[4 * i + 2], quat[4 * i + 3]};
    double r[9];
    rotmat(q, r);
    Slip64 sl;
    slip64(pc, visc, pup + 3 * i, pufap + 3 * i, r, sl);
    double a[3], b[3];
    fluid_torque(pc, visc, sl, pvort[3 * i], pvort[3 * i + 1], pvort[3 * i + 2], om[3 * i], om[3 * i + 1],
                 om[3 * i + 2], r, a, b);
    if (om[3 * i] != om[3 * i]) set_error(st, GP_ENAN_TORQUE, i);
#pragma unroll
    for (int k = 0; k < 3; ++k) { tp[3 * i + k] = a[k]; tr[3 * i + k] = b[k]; }
  }
}

__global__ void k_quat_batch(int64_t n, double *quat, const double *om, double dt) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    Quat q = {quat[4 * i], quat[4 * i + 1], quat[4 * i + 2], quat[4 * i + 3]};
    quaternion_integration(q, om[3 * i], om[3 * i + 1], om[3 * i + 2], dt);
    quat[4 * i] = q.a; quat[4 * i + 1] = q.b; quat[4 * i + 2] = q.c; quat[4 * i + 3] = q.d;
  }
}

__global__ void k_euler_batch(int64_t n, const double *ip, double dt, double *om) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double x = om[3 * i], y = om[3 * i + 1], z = om[3 * i + 2];
    euler_integration(ip[3 * i], ip[3 * i + 1], ip[3 * i + 2], dt, x, y, z);
    om[3 * i] = x; om[3 * i + 1] = y; om[3 * i + 2] = z;
  }
}

__global__ void __launch_bounds__(128, 8) k_contact_batch(int64_t n, const double *shapes, const double *centres, const double *quats,
                                int32_t *flag, double *e1, double *e2, double *cn) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double *s = shapes + 4 * i, *c = centres + 6 * i, *q = quats + 8 * i;
    const Quat q1 = {q[0], q[1], q[2], q[3]}, q2 = {q[4], q[5], q[6], q[7]};
    double a[3], b[3], nn[3];
    flag[i] = contact_detection(s[0], s[1], s[2], s[3], c, q1, c + 3, q2, a, b, nn) ? 1 : 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) { e1[3 * i + k] = a[k]; e2[3 * i + k] = b[k]; cn[3 * i + k] = nn[k]; }
  }
}

__global__ void k_response_batch(int64_t n, double ecp, double mup, const double *ip, double *p1, double *p2,
                                 const double *r1, const double *r2, const double *nrm, Status *st) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double *a = p1 + 10 * i, *b = p2 + 10 * i;
    double u1[3] = {a[0], a[1], a[2]}, o1[3] = {a[3], a[4], a[5]};
    double u2[3] = {b[0], b[1], b[2]}, o2[3] = {b[3], b[4], b[5]};
    const Quat q1 = {a[6], a[7], a[8], a[9]}, q2 = {b[6], b[7], b[8], b[9]};
    const int rc = collision_response(ecp, mup, ip[3 * i], ip[3 * i + 1], ip[3 * i + 2], u1, o1, q1, u2, o2, q2,
                                      r1 + 3 * i, r2 + 3 * i, nrm + 3 * i);
    if (rc) set_error(st, rc, i);
#pragma unroll
    for (int k = 0; k < 3; ++k) { a[k] = u1[k]; a[3 + k] = o1[k]; b[k] = u2[k]; b[3 + k] = o2[k]; }
  }
}

static int grid_for(int64_t n) { return (int)((n + 127) / 128 < 148 * 8 ? (n + 127) / 128 : 148 * 8); }

void launch_force_batch(int64_t n, const double *pcs, double visc, const double *up, const double *uf,
                        const double *quat, double *fdrag, double *flift, Status *st, cudaStream_t s) {
  if (n > 0) k_force_batch<<<grid_for(n), 128, 0, s>>>(n, pcs, visc, up, uf, quat, fdrag, flift, st);
}
void launch_torque_batch(int64_t n, const double *pcs, double visc, const double *omega, const double *quat,
                         const double *pup, const double *pufap, const double *pvort, double *tp, double *tr,
                         Status *st, cudaStream_t s) {
  if (n > 0)
    k_torque_batch<<<grid_for(n), 128, 0, s>>>(n, pcs, visc, omega, quat, pup, pufap, pvort, tp, tr, st);
}
void launch_quat_batch(int64_t n, double *quat, const double *omega, double dt, cudaStream_t s) {
  if (n > 0) k_quat_batch<<<grid_for(n), 128, 0, s>>>(n, quat, omega, dt);
}
void launch_euler_batch(int64_t n, const double *ip, double dt, double *omega, cudaStream_t s) {
  if (n > 0) k_euler_batch<<<grid_for(n), 128, 0, s>>>(n, ip, dt, omega);
}
void launch_contact_batch(int64_t n, const double *shapes, const double *centres, const double *quats,
                          int32_t *flag, double *e1, double *e2, double *cn, cudaStream_t s) {
  if (n > 0) k_contact_batch<<<grid_for(n), 128, 0, s>>>(n, shapes, centres, quats, flag, e1, e2, cn);
}
void launch_response_batch(int64_t n, double ecp, double mup, const double *ip, double *p1, double *p2,
                           const double *r1, const double *r2, const double *nrm, Status *st, cudaStream_t s) {
  if (n > 0) k_response_batch<<<grid_for(n), 128, 0, s>>>(n, ecp, mup, ip, p1, p2, r1, r2, nrm, st);
}

}  // namespace gp
