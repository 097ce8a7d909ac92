// gp_stats.cu -- statistics computed beside the step, on the device.
//
//  - STAT_PARTFLUID (stat_partfluid.f90:1-472): 35 per-particle quantities of the
//    particle-fluid coupling (Re_p, drag and lift coefficients and forces, Re_R, torque
//    coefficients and torques, relaxation times, orientation, velocities), summed per
//    class and polydisperse index, with the particle count as the 36th entry.
//  - The collision statistics of COLLISION_INTERACTION (collision_interaction.f90:
//    171,330-345,397-398,423-450): per class and pair of polydisperse indices, the pairs
//    found in contact while both particles were uncoloured, the collisions among them,
//    and the sums of overlap depth, NVREL, |v_rel| and the collision angle.
//
// Both read only what the step already holds in HBM, so a run needs no state download
// to follow them.  Compiled without FMA contraction (-fmad=false), as the FP64 path is.
#include <cuda_runtime.h>

#include "gp_device.cuh"
#include "gp_launch.h"

namespace gp {

constexpr int kStatThreads = 128;
constexpr int kStatWarps = kStatThreads / 32;

// stat_partfluid.f90:122-293 for one particle.  The reference reads EMAJ_PART, APR_PART
// and RHOP of the particle's class and index; the pool keeps the derived constants, so
// RHOF/PMASS is 2*crot (bit for bit the reference's quotient: crot = (0.5*RHOF)/PMASS),
// d_eq and EMAJ/APR are stored as such, and APR = a/b, PMASS = RHOF/(RHOF/PMASS) and
// RHOP are recovered to within a few units in the last place.
__device__ __forceinline__ void partfluid_values(const PartConst &pc, double rhof, double visc, double ppi,
                                                 double gravity, const double U[3], const double O[3],
                                                 const Quat &q, const double uf[3], const double wv[3],
                                                 double v[kNStatPartfluid]) {
  constexpr double a0 = 1.95, a1 = 18.12, a2 = 1.023, a3 = 4.26, a4 = 0.384;
  constexpr double a5 = 21.52, a6 = 0.990, a7 = 2.86, a8 = 0.260;
  constexpr double b1 = 0.083, b2 = -0.21, b3 = 1.582, b4 = 0.851, b5 = 1.842;
  constexpr double b6 = -0.802, b7 = -0.006, b8 = 0.874, b9 = 0.009, b10 = 0.570;
  constexpr double c1 = 0.935, c2 = 0.146, c3 = -0.469, c4 = 0.145, c5 = 0.116;
  constexpr double c6 = 0.748, c7 = 0.041, c8 = 0.221, c9 = 0.657, c10 = 0.044;
  constexpr double r1 = 0.573, r2 = -0.154, r3 = 116.61, r4 = 1.0;
  constexpr double r1_ = 1.244, r2_ = 0.239, r3_ = 378.12, r4_ = 0.789;
  const double rp = 2.0 * pc.crot;      // RHOF/PMASS
  const double pmass = rhof / rp;
  const double apr = pc.a / pc.b;
  const double deq = pc.deq;
  double rt[9];
  rotmat(conj(q), rt);
  double p[3] = {uf[0] - U[0], uf[1] - U[1], uf[2] - U[2]};
  const double urel = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
  const double rep = (urel * deq) / visc;
  matvec(rt, p, p);
  const double phi = fabs(atan((sqrt(p[1] * p[1] + p[2] * p[2])) / (p[0])));
  const double umag = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
  const double sphi = sin(phi), cphi = cos(phi);
  const double cd0 = a1 / pow(rep, a2) + a3 / pow(rep, a4);
  const double cd90 = a5 / pow(rep, a6) + a7 / pow(rep, a8);
  const double cdrag = cd0 + (cd90 - cd0) * pow(sphi, a0);
  const double clift = (b1 / pow(rep, b2) + b3 / pow(rep, b4)) * pow(sphi, b5 + b6 * pow(rep, b7)) *
                       pow(cphi, b8 + b9 * pow(rep, b10));
  const double kf = 0.5 * rp * 0.25 * (ppi * (deq * deq));
  const double syz = sqrt(p[1] * p[1] + p[2] * p[2]);
  double fd[3], fl[3];
  for (int k = 0; k < 3; ++k) fd[k] = kf * cdrag * umag * p[k];
  fl[0] = kf * clift * (umag * umag) * sphi * copysign(1.0, -p[0]);
  fl[1] = kf * clift * (umag * umag) * cphi * (p[1] / syz);
  fl[2] = kf * clift * (umag * umag) * cphi * (p[2] / syz);
  double r[9];
  rotmat(q, r);
  matvec(r, fd, fd);
  matvec(r, fl, fl);
  v[0] = rep; v[1] = cdrag; v[2] = clift;
  v[3] = fd[0]; v[4] = fd[1]; v[5] = fd[2];
  v[6] = fl[0]; v[7] = fl[1]; v[8] = fl[2];
  v[9] = sqrt(fd[0] * fd[0] + fd[1] * fd[1] + fd[2] * fd[2]);
  v[10] = sqrt(fl[0] * fl[0] + fl[1] * fl[1] + fl[2] * fl[2]);
  double curl[3] = {wv[0], wv[1], wv[2]};
  matvec(rt, curl, curl);
  const double o0 = 0.5 * curl[0] - O[0], o1 = 0.5 * curl[1] - O[1], o2 = 0.5 * curl[2] - O[2];
  const double omag = sqrt(o0 * o0 + o1 * o1 + o2 * o2);
  const double oyz = sqrt(o2 * o2 + o1 * o1);
  const double re_r = (omag * (deq * deq)) / visc;
  const double ctp = (c1 / pow(rep, c2) + c3 / pow(rep, c4)) * pow(sphi, c5 + c6 * pow(rep, c7)) *
                     pow(cphi, c8 + c9 * pow(rep, c10));
  const double ctr = r1 * pow(re_r, r2) + r3 / pow(re_r, r4);
  const double ctr2 = r1_ * pow(re_r, r2_) + r3_ / pow(re_r, r4_);
  const double kp = 0.25 * rp * 0.25 * ppi * ((deq * deq) * deq);
  const double tp1 = kp * ctp * (umag * umag) * (fabs(p[2]) / syz) * copysign(1.0, p[0] * p[2]);
  const double tp2 = kp * ctp * (umag * umag) * (fabs(p[1]) / syz) * copysign(1.0, p[0] * p[1]);
  const double h = deq / 2.0, h2 = h * h, h5 = h2 * h2 * h;
  const double tr0 = ctr * rp / 2.0 * h5 * fabs(o0) * o0;
  const double tr1 = ctr2 * rp / 2.0 * h5 * oyz * o1;
  const double tr2 = ctr2 * rp / 2.0 * h5 * oyz * o2;
  v[11] = re_r; v[12] = ctp; v[13] = ctr;
  v[14] = 0.0; v[15] = tp1; v[16] = tp2;
  v[17] = tr0; v[18] = tr1; v[19] = tr2;
  v[20] = sqrt(0.0 * 0.0 + tp1 * tp1 + tp2 * tp2);
  v[21] = sqrt(tr0 * tr0 + tr1 * tr1 + tr2 * tr2);
  // stat_partfluid.f90:265-276
  const double minax = pc.b;
  double fbeta = 1.0;
  if (!(apr == 1.0)) fbeta = (apr * log(apr + sqrt(apr * apr - 1.0))) / (sqrt(apr * apr - 1.0));
  const double rhop = pmass * (apr * apr) / ((4.0 / 3.0) * ppi * pow(pc.a, 3.0));
  double taupf = (2.0 / 9.0) * (rhop * (minax * minax)) / (rhof * visc);
  taupf = taupf * fbeta;
  v[22] = taupf;
  v[23] = gravity;
  v[24] = phi;
  v[25] = r[0]; v[26] = r[1]; v[27] = r[2];   // R(q) (1,0,0)
  v[28] = (0.5 * rhof * cdrag * (ppi / 4.0) * (deq * deq) * umag) / pmass;
  v[29] = U[0]; v[30] = U[1]; v[31] = U[2];
  v[32] = O[0]; v[33] = O[1]; v[34] = O[2];
  v[35] = 1.0;
}

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// Block b sums the class's particles in pool slots [b*per, (b+1)*per), warp by warp in
// slot order and group by group, so the partial sums do not depend on scheduling.
__global__ void __launch_bounds__(kStatThreads) k_stat_partfluid(const InstDev *__restrict__ insts,
                                                                 const PoolView *__restrict__ pv, int64_t n,
                                                                 int inst, const double *const *fluid,
                                                                 const int32_t *__restrict__ groups, int ngroups,
                                                                 double rhof, double ppi, double *partial,
                                                                 Status *st) {
  __shared__ double acc[kStatWarps][kStatMaxGroups][kNStatPartfluid];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int t = threadIdx.x; t < kStatWarps * kStatMaxGroups * kNStatPartfluid; t += blockDim.x)
    (&acc[0][0][0])[t] = 0.0;
  __syncthreads();
  const PoolView *__restrict__ P = pv;
  const InstDev &I = insts[inst];
  const int64_t per = (n + gridDim.x - 1) / gridDim.x;
  const int64_t lo = (int64_t)blockIdx.x * per, hi = min(n, lo + per);
  for (int64_t base = lo + 32 * warp; base < hi; base += kStatThreads) {
    const int64_t i = base + lane;
    int g = -1;
    if (i < hi && P->inst[i] == inst) {
      const int32_t id = P->id[i];
      g = groups ? groups[id] - 1 : 0;
      if (g < 0 || g >= ngroups) {
        set_error(st, GP_EBADARG, id, inst);
        g = -1;
      }
    }
    double v[kNStatPartfluid];
    if (g >= 0) {
      PartConst pc;
      pc.a = P->pc[0][i]; pc.b = P->pc[1][i]; pc.deq = P->pc[2][i]; pc.cdrag = P->pc[3][i];
      pc.cpitch = P->pc[4][i]; pc.crot = P->pc[5][i]; pc.h5 = P->pc[6][i];
      pc.ipxx = P->pc[7][i]; pc.ipyy = P->pc[8][i]; pc.ipzz = P->pc[9][i];
      const double U[3] = {P->st[3][i], P->st[4][i], P->st[5][i]};
      const double O[3] = {P->st[10][i], P->st[11][i], P->st[12][i]};
      const Quat q = {P->st[6][i], P->st[7][i], P->st[8][i], P->st[9][i]};
      const double uf[3] = {fluid[0][i], fluid[1][i], fluid[2][i]};
      const double wv[3] = {fluid[3][i], fluid[4][i], fluid[5][i]};
      partfluid_values(pc, rhof, I.visc, ppi, I.gravity, U, O, q, uf, wv, v);
    }
    unsigned todo = __ballot_sync(0xffffffffu, g >= 0);
    while (todo) {
      const int gg = __shfl_sync(0xffffffffu, g, __ffs(todo) - 1);
      const bool mine = (g == gg);
      todo &= ~__ballot_sync(0xffffffffu, mine);
#pragma unroll
      for (int s = 0; s < kNStatPartfluid; ++s) {
        const double x = warp_sum(mine ? v[s] : 0.0);
        if (lane == 0) acc[warp][gg][s] += x;
      }
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < ngroups * kNStatPartfluid; t += blockDim.x) {
    const int g = t / kNStatPartfluid, s = t % kNStatPartfluid;
    double x = 0.0;
    for (int w = 0; w < kStatWarps; ++w) x += acc[w][g][s];
    partial[(size_t)blockIdx.x * ngroups * kNStatPartfluid + t] = x;
  }
}

// Partial sums of the blocks, added in block order.
__global__ void k_stat_blocks(const double *__restrict__ partial, int nblocks, int width, double *out) {
  for (int t = threadIdx.x; t < width; t += blockDim.x) {
    double x = 0.0;
    for (int b = 0; b < nblocks; ++b) x += partial[(size_t)b * width + t];
    out[t] = x;
  }
}

void launch_stat_partfluid(const InstDev *insts, const PoolView *pv, int64_t n, int inst, double *const *fluid,
                           const int32_t *groups, int ngroups, double rhof, double ppi, double *partial,
                           int nblocks, double *out, Status *st, cudaStream_t s) {
  k_stat_partfluid<<<nblocks, kStatThreads, 0, s>>>(insts, pv, n, inst, fluid, groups, ngroups, rhof, ppi, partial,
                                                    st);
  k_stat_blocks<<<1, 256, 0, s>>>(partial, nblocks, ngroups * kNStatPartfluid, out);
}

// ---------------------------------------------------------------------------
// Collision statistics
// ---------------------------------------------------------------------------
// The COLOR walk examines a pair while both particles are uncoloured, so a pair in
// contact is counted when neither particle was coloured by an accepted pair that comes
// before it in the list.  Accepted pairs (state 1 after k_match) leave their key at
// both particles (best1/best2, reset to all ones afterwards).
__global__ void k_colour_keys(const CollRec *__restrict__ coll, const unsigned long long *__restrict__ ncoll,
                              int64_t cap, const int8_t *__restrict__ state, unsigned long long *best1,
                              unsigned long long *best2, int set, unsigned long long *steps, const Status *st) {
  if (step_halted(st)) return;
  const int64_t nc = (int64_t)min(*ncoll, (unsigned long long)cap);
  if (steps && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(steps, 1ull);   // one more step in the sums
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nc; e += (int64_t)gridDim.x * blockDim.x) {
    if (state[e] != 1) continue;
    const CollRec &r = coll[e];
    const unsigned long long k1 = set ? r.k1 : ~0ull, k2 = set ? r.k2 : ~0ull;
    best1[r.home] = k1; best2[r.home] = k2;
    best1[r.near] = k1; best2[r.near] = k2;
  }
}

__device__ __forceinline__ bool key_le(unsigned long long a1, unsigned long long a2, unsigned long long b1,
                                       unsigned long long b2) {
  return a1 < b1 || (a1 == b1 && a2 <= b2);
}

// collision_interaction.f90:330-345 and :397-398 for the contacts the walk examines.
__global__ void k_collision_stats(const ContactStatRec *__restrict__ rec, const unsigned long long *__restrict__ nrec,
                                  int64_t cap, const PoolView *__restrict__ pv,
                                  const int32_t *const *__restrict__ group_tab, const int32_t *__restrict__ ngroups,
                                  const unsigned long long *__restrict__ best1,
                                  const unsigned long long *__restrict__ best2, double *acc, Status *st) {
  if (step_halted(st)) return;
  const int64_t nr = (int64_t)min(*nrec, (unsigned long long)cap);
  const PoolView *__restrict__ P = pv;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nr; e += (int64_t)gridDim.x * blockDim.x) {
    const ContactStatRec r = rec[e];
    if (!key_le(r.k1, r.k2, best1[r.home], best2[r.home]) || !key_le(r.k1, r.k2, best1[r.near], best2[r.near]))
      continue;
    const int inst = r.inst;
    const int ng = ngroups[inst];
    const int32_t *gt = group_tab[inst];
    const int g1 = gt ? gt[P->id[r.home]] - 1 : 0, g2 = gt ? gt[P->id[r.near]] - 1 : 0;
    if (g1 < 0 || g1 >= ng || g2 < 0 || g2 >= ng) {
      set_error(st, GP_EBADARG, P->id[r.home], inst);
      continue;
    }
    double *a = acc + ((size_t)inst * kStatMaxGroups * kStatMaxGroups + (size_t)g1 * kStatMaxGroups + g2) *
                          kNStatCollision;
    atomicAdd(&a[0], 1.0);
    atomicAdd(&a[3], r.depth);
    atomicAdd(&a[5], r.nvrel);
    atomicAdd(&a[6], r.nrm);
    atomicAdd(&a[7], acos(r.nvrel / r.nrm));
    if (r.nvrel < kZeroRef) atomicAdd(&a[1], 1.0);
  }
}

void launch_collision_stats(const CollRec *coll, const unsigned long long *ncoll, int64_t cap_coll,
                            const int8_t *state, unsigned long long *best1, unsigned long long *best2,
                            const ContactStatRec *rec, const unsigned long long *nrec, int64_t cap_rec,
                            const PoolView *pv, const int32_t *const *group_tab, const int32_t *ngroups, double *acc,
                            unsigned long long *steps, Status *st, cudaStream_t s) {
  k_colour_keys<<<148, 256, 0, s>>>(coll, ncoll, cap_coll, state, best1, best2, 1, steps, st);
  k_collision_stats<<<148 * 2, 256, 0, s>>>(rec, nrec, cap_rec, pv, group_tab, ngroups, best1, best2, acc, st);
  k_colour_keys<<<148, 256, 0, s>>>(coll, ncoll, cap_coll, state, best1, best2, 0, nullptr, st);
}

}  // namespace gp
