// gp_contact.cuh -- one candidate pair of collision_interaction.f90:216-348: its
// geometry, and what follows a finished contact solve.
#pragma once

#include "gp_lm.cuh"

namespace gp {

// A solve handed from one pass of k_contact to the next: the pair and the solver's state
// between two lm_step calls (the problem itself is rebuilt from the pool).
struct TailRec {
  int64_t e;                 // index of the pair in the candidate list
  LmState S;
};

// The pair's bodies as the contact test sees them (collision_interaction.f90:216-249):
// HOME at its position, NEAR at the minimum image, orientations and semi-axes.
struct PairBodies {
  double c1[3], c2[3];
  Quat q1, q2;
  double a1, b1, a2, b2;
};

__device__ __forceinline__ void pair_bodies(const InstDev *__restrict__ insts, const PoolView &P, int i1, int i2,
                                            PairBodies &B) {
  const InstDev &I = insts[P.inst[i1]];
  const double x1 = P.st[0][i1], y1 = P.st[1][i1], z1 = P.st[2][i1];
  double vkx = P.st[0][i2] - x1, vky = P.st[1][i2] - y1, vkz = P.st[2][i2] - z1;
  if ((fabs(vkx) > I.lx / 2) && I.periodicity) vkx = vkx - copysign(I.lx, vkx);
  if (fabs(vky) > I.ly / 2.) vky = vky - copysign(I.ly, vky);
  if (fabs(vkz) > I.lz / 2.) vkz = vkz - copysign(I.lz, vkz);
  B.c1[0] = x1; B.c1[1] = y1; B.c1[2] = z1;
  B.c2[0] = x1 + vkx; B.c2[1] = y1 + vky; B.c2[2] = z1 + vkz;
  B.q1 = {P.st[6][i1], P.st[7][i1], P.st[8][i1], P.st[9][i1]};
  B.q2 = {P.st[6][i2], P.st[7][i2], P.st[8][i2], P.st[9][i2]};
  B.a1 = P.pc[0][i1]; B.b1 = P.pc[1][i1]; B.a2 = P.pc[0][i2]; B.b2 = P.pc[1][i2];
}

// The solve of pair e has returned at angles (x0, x1) after nfev evaluations: contact
// test, contact-point velocities, NVREL, the contact record for the statistics and the
// colliding-pair record.  Out of line and given only the pair index and the solver's
// result, so that the solving loop never passes its state by address: the problem is
// rebuilt from the pool, which the contact phase does not change, by the same set-up
// (hence to the same values).  hist (optional): the queue order's record of the solve.
static __device__ __noinline__ void finish_pair(const InstDev *__restrict__ insts, const PoolView *__restrict__ pv,
                                         const PairRec *__restrict__ pairs, int64_t e, double x0, double x1,
                                         int nfev, CollRec *__restrict__ coll, unsigned long long *ncoll,
                                         int64_t cap_coll, ContactStatRec *__restrict__ cst,
                                         unsigned long long *ncst, int64_t cap_cst, uint32_t *hist,
                                         int64_t nhist, Status *st) {
  const PoolView P = *pv;
  atomicAdd(&st->n_solve, 1ull);
  atomicAdd(&st->n_eval, (unsigned long long)nfev);
  atomicMax(&st->max_eval, (unsigned long long)nfev);
  const PairRec pr = pairs[e];
  const int i1 = pr.home, i2 = pr.near;
  if (hist) {   // what this solve took, for the next collision phase's queue order
    const int64_t k0 = insts[P.inst[i1]].begin, g1 = k0 + P.id[i1], g2 = k0 + P.id[i2];
    if (g1 < nhist) atomicMax(&hist[g1], (uint32_t)nfev + 1u);
    if (g2 < nhist) atomicMax(&hist[g2], (uint32_t)nfev + 1u);
  }
  PairBodies B;
  pair_bodies(insts, P, i1, i2, B);
  ContactProb CP;
  double xs[2];
  contact_setup(B.a1, B.b1, B.a2, B.b2, B.c1, B.q1, B.c2, B.q2, CP, xs);
  const double x[2] = {x0, x1};
  double ept1[3], ept2[3], cn[3];
  if (!contact_finish(B.a1, B.b1, B.a2, B.b2, B.q1, B.q2, CP, x, ept1, ept2, cn)) return;
  atomicAdd(&st->n_contact, 1ull);
  // overlap depth |EPT1 - EPT2| for the collision statistics, while the points are at hand
  double depth = 0.0;
  if (cst != nullptr) {
    const double v0 = ept1[0] - ept2[0], v1 = ept1[1] - ept2[1], v2 = ept1[2] - ept2[2];
    depth = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
  }
  const double xh = CP.b1[0], yh = CP.b1[1], zh = CP.b1[2];
  double rx1[3] = {(ept1[0] - xh), (ept1[1] - yh), (ept1[2] - zh)};
  double om1[3] = {P.st[10][i1], P.st[11][i1], P.st[12][i1]};
  rot_vec(B.q1, om1);
  const double up1 = P.st[3][i1] + (om1[1] * rx1[2] - om1[2] * rx1[1]);
  const double vp1 = P.st[4][i1] + (om1[2] * rx1[0] - om1[0] * rx1[2]);
  const double wp1 = P.st[5][i1] + (om1[0] * rx1[1] - om1[1] * rx1[0]);
  double rx2[3] = {(ept2[0] - CP.b2[0]), (ept2[1] - CP.b2[1]), (ept2[2] - CP.b2[2])};
  double om2[3] = {P.st[10][i2], P.st[11][i2], P.st[12][i2]};
  rot_vec(B.q2, om2);
  const double up2 = P.st[3][i2] + (om2[1] * rx2[2] - om2[2] * rx2[1]);
  const double vp2 = P.st[4][i2] + (om2[2] * rx2[0] - om2[0] * rx2[2]);
  const double wp2 = P.st[5][i2] + (om2[0] * rx2[1] - om2[1] * rx2[0]);
  const double nvrel = (up2 - up1) * cn[0] + (vp2 - vp1) * cn[1] + (wp2 - wp1) * cn[2];
  if (cst != nullptr) {
    // every contact, for the collision statistics (collision_interaction.f90:253-328)
    const unsigned long long k = atomicAdd(ncst, 1ull);
    if ((int64_t)k < cap_cst) {
      ContactStatRec c;
      c.home = i1; c.near = i2; c.inst = P.inst[i1]; c.pad = 0; c.k1 = pr.k1; c.k2 = pr.k2;
      c.depth = depth;
      c.nvrel = nvrel;
      const double vx = up2 - up1, vy = vp2 - vp1, vz = wp2 - wp1;
      c.nrm = sqrt(vx * vx + vy * vy + vz * vz);
      cst[k] = c;
    } else {
      set_error(st, GP_EPAIR_OVERFLOW, (long long)P.id[i1], P.inst[i1]);
    }
  }
  if (!(nvrel < kZeroRef)) return;
  const unsigned long long slot = atomicAdd(ncoll, 1ull);
  if ((int64_t)slot >= cap_coll) {
    atomicAdd(&st->overflow, 1ull);
    set_error(st, GP_EPAIR_OVERFLOW, (long long)P.id[i1], P.inst[i1]);
    return;
  }
  CollRec r;
  r.home = i1; r.near = i2; r.k1 = pr.k1; r.k2 = pr.k2;
  r.inst = P.inst[i1]; r.pad = 0;
#pragma unroll
  for (int i = 0; i < 3; ++i) { r.rx1[i] = rx1[i]; r.rx2[i] = rx2[i]; r.cn[i] = cn[i]; }
  coll[slot] = r;
}

}  // namespace gp
