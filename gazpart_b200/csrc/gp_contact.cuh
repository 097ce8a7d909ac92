// gp_contact.cuh -- what follows a finished contact solve (collision_interaction.f90:
// 240-348), shared by the persistent contact kernel and the kernel that finishes the
// long solves it hands over.
#pragma once

#include "gp_lm.cuh"

namespace gp {

// A solve handed from k_contact to k_contact_tail: the pair, its problem and the
// solver's state between two lm_step calls.
struct TailRec {
  int64_t e;                 // index of the pair in the candidate list
  ContactProb CP;
  LmState S;
  Quat q1, q2;
  double a1, b1, a2, b2;
};

// The solve of pair e has returned: contact test, contact-point velocities, NVREL,
// the contact record for the statistics and the colliding-pair record.
__device__ __forceinline__ void finish_pair(const PoolView &P, const PairRec *__restrict__ pairs, int64_t e,
                                            const ContactProb &CP, const LmState &S, const Quat &q1,
                                            const Quat &q2, double a1, double b1, double a2, double b2,
                                            CollRec *__restrict__ coll, unsigned long long *ncoll,
                                            int64_t cap_coll, ContactStatRec *__restrict__ cst,
                                            unsigned long long *ncst, int64_t cap_cst, Status *st) {
  atomicAdd(&st->n_solve, 1ull);
  atomicAdd(&st->n_eval, (unsigned long long)S.nfev);
  atomicMax(&st->max_eval, (unsigned long long)S.nfev);
  double ept1[3], ept2[3], cn[3];
  if (!contact_finish(a1, b1, a2, b2, q1, q2, CP, S.x, ept1, ept2, cn)) return;
  atomicAdd(&st->n_contact, 1ull);
  // overlap depth |EPT1 - EPT2| for the collision statistics, while the points are at hand
  double depth = 0.0;
  if (cst != nullptr) {
    const double v0 = ept1[0] - ept2[0], v1 = ept1[1] - ept2[1], v2 = ept1[2] - ept2[2];
    depth = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
  }
  const PairRec pr = pairs[e];
  const int i1 = pr.home, i2 = pr.near;
  const double x1 = CP.b1[0], y1 = CP.b1[1], z1 = CP.b1[2];
  double rx1[3] = {(ept1[0] - x1), (ept1[1] - y1), (ept1[2] - z1)};
  double om1[3] = {P.st[10][i1], P.st[11][i1], P.st[12][i1]};
  rot_vec(q1, om1);
  const double up1 = P.st[3][i1] + (om1[1] * rx1[2] - om1[2] * rx1[1]);
  const double vp1 = P.st[4][i1] + (om1[2] * rx1[0] - om1[0] * rx1[2]);
  const double wp1 = P.st[5][i1] + (om1[0] * rx1[1] - om1[1] * rx1[0]);
  double rx2[3] = {(ept2[0] - CP.b2[0]), (ept2[1] - CP.b2[1]), (ept2[2] - CP.b2[2])};
  double om2[3] = {P.st[10][i2], P.st[11][i2], P.st[12][i2]};
  rot_vec(q2, om2);
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
