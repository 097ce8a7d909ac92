// gp_contact.cu -- the contact solves of one collision phase (collision_interaction.f90:
// 216-348), compiled without FMA contraction so that every rounded operation matches an
// IEEE restatement of the reference.
//
// One solve is a long chain of dependent FP64 operations (about 16k cycles per function
// evaluation on a lone lane, 3.0 M evaluations per step at 512^3/16.8 M spheroids), so
// the phase is bound by how many solves the SMs keep in flight: eight blocks of 128 per
// SM with the solver's pieces out of line (64 registers) finish the bulk sooner than two
// blocks with the whole iteration inlined in registers, although each lane then runs
// its own iteration faster.
#include <math_constants.h>

#include "gp_contact.cuh"
#include "gp_launch.h"

namespace gp {

// A solve handed over by an earlier pass: its pair and solver state, and the problem
// rebuilt from the pool by the same set-up (so to the same values).  Out of line: the
// solving loop only passes the state it already keeps in local memory.
static __device__ __noinline__ void resume_solve(const InstDev *__restrict__ insts, const PoolView *__restrict__ pv,
                                                 const PairRec *__restrict__ pairs, const TailRec *__restrict__ rec,
                                                 int64_t &e, ContactProb &CP, LmState &S) {
  e = rec->e;
  S = rec->S;
  const PairRec pr = pairs[e];
  PairBodies B;
  pair_bodies(insts, *pv, pr.home, pr.near, B);
  double xs[2];
  contact_setup(B.a1, B.b1, B.a2, B.b2, B.c1, B.q1, B.c2, B.q2, CP, xs);
}

// collision_interaction.f90:216-348 for every candidate pair: minimum image, contact
// (ellipsoid_contact_detection), contact-point velocities, NVREL.  Colliding pairs
// (flag && NVREL < ZERO) are appended.  Persistent warps with lane refill: a lane whose
// Levenberg-Marquardt solve has returned finishes its pair and takes the next one from
// a global queue, so warps do not idle on their slowest pair.
//
// Passes.  A warp runs as long as its slowest lane, and a C3 step has about one solve per
// lane of the persistent grid, so refilling cannot even out solves of 3 to 300
// evaluations.  With `out` set, a solve still running after `budget` evaluations is
// written there (pair and solver state) and the lane takes other work; a further pass
// of this kernel (`in` set) resumes those solves with every lane busy, under a larger
// budget or none.  The iterates are the same operations in the same order.
#ifndef GP_CONTACT_MIN_BLOCKS
#define GP_CONTACT_MIN_BLOCKS 8
#endif

__global__ void __launch_bounds__(128, GP_CONTACT_MIN_BLOCKS) k_contact(const InstDev *__restrict__ insts,
                                                    const PoolView *__restrict__ pv,
                                                    const PairRec *__restrict__ pairs,
                                                    const unsigned long long *__restrict__ npairs, int64_t cap_pairs,
                                                    const TailRec *__restrict__ in,
                                                    const unsigned long long *__restrict__ nin, int64_t cap_in,
                                                    CollRec *__restrict__ coll, unsigned long long *ncoll,
                                                    int64_t cap_coll, unsigned long long *queue,
                                                    ContactStatRec *__restrict__ cst, unsigned long long *ncst,
                                                    int64_t cap_cst, TailRec *__restrict__ out,
                                                    unsigned long long *nout, int64_t cap_out, int budget,
                                                    Status *st) {
  if (step_halted(st)) return;
  const int64_t np = in ? (int64_t)min(*nin, (unsigned long long)cap_in)
                        : (int64_t)min(*npairs, (unsigned long long)cap_pairs);
  const unsigned lane = threadIdx.x & 31u;
  constexpr unsigned kFull = 0xffffffffu;
  bool active = false, exhausted = false;
  int64_t e = 0;
  ContactProb CP;
  LmState S;
  for (;;) {
    if (!exhausted) {
      const unsigned want = __ballot_sync(kFull, !active);
      if (want) {
        const int leader = __ffs(want) - 1;
        unsigned long long base = 0;
        if ((int)lane == leader) base = atomicAdd(queue, (unsigned long long)__popc(want));
        base = __shfl_sync(kFull, base, leader);
        if ((int64_t)base >= np) {
          exhausted = true;
        } else if (!active) {
          const int64_t q = (int64_t)base + __popc(want & ((1u << lane) - 1u));
          if (q < np && in) {
            resume_solve(insts, pv, pairs, in + q, e, CP, S);
            active = true;
          } else if (q < np) {
            e = q;
            const PairRec pr = pairs[e];
            PairBodies B;
            pair_bodies(insts, *pv, pr.home, pr.near, B);
            const double vkx = B.c2[0] - B.c1[0], vky = B.c2[1] - B.c1[1], vkz = B.c2[2] - B.c1[2];
            const Quat &q1 = B.q1, &q2 = B.q2;
            // symmetry axes (first columns of R(q)); disjoint bodies need no solve
            const double e1[3] = {1.0 - 2.0 * (q1.c * q1.c + q1.d * q1.d), 2.0 * (q1.b * q1.c + q1.a * q1.d),
                                  2.0 * (q1.b * q1.d - q1.a * q1.c)};
            const double e2[3] = {1.0 - 2.0 * (q2.c * q2.c + q2.d * q2.d), 2.0 * (q2.b * q2.c + q2.a * q2.d),
                                  2.0 * (q2.b * q2.d - q2.a * q2.c)};
            const bool apart =
                separated(vkx, vky, vkz, e1, B.a1 * B.a1, B.b1 * B.b1, e2, B.a2 * B.a2, B.b2 * B.b2);
            if (!apart && contact_setup(B.a1, B.b1, B.a2, B.b2, B.c1, q1, B.c2, q2, CP, S.x)) {
              lm_begin(CP, S);
              active = true;
            }
          }
        }
      }
    }
    if (!__any_sync(kFull, active)) {
      if (exhausted) break;
      continue;
    }
    if (!active) continue;
    if (lm_step(CP, S, kContactTol) == 0) {
      // past the budget the solve moves on to the next pass and the lane takes other
      // work (with the hand-over buffer full, the lane keeps the solve)
      if (out != nullptr && S.nfev >= budget) {
        const unsigned long long k = atomicAdd(nout, 1ull);
        if ((int64_t)k < cap_out) {
          out[k].e = e;
          out[k].S = S;
          active = false;
        }
      }
      continue;
    }
    active = false;
    finish_pair(insts, pv, pairs, e, S.x[0], S.x[1], S.nfev, coll, ncoll, cap_coll, cst, ncst, cap_cst, st);
  }
}

// Persistent grid for k_contact: as many blocks as can be resident at once on the
// current device (looked up once, at context creation, outside any stream capture).
int contact_grid_blocks() {
  int per_sm = 0, dev = 0, sms = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_contact, 128, 0) != cudaSuccess ||
      cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || per_sm <= 0)
    return 0;
  return per_sm * sms;
}

void launch_contact(const InstDev *insts, const PoolView *pv, const PairRec *pairs, const unsigned long long *npairs,
                    int64_t cap_pairs, const TailRec *in, const unsigned long long *nin, int64_t cap_in,
                    CollRec *coll, unsigned long long *ncoll, int64_t cap_coll, unsigned long long *queue,
                    ContactStatRec *cst, unsigned long long *ncst, int64_t cap_cst, TailRec *out,
                    unsigned long long *nout, int64_t cap_out, int budget, Status *st, int grid, cudaStream_t s) {
  k_contact<<<grid, 128, 0, s>>>(insts, pv, pairs, npairs, cap_pairs, in, nin, cap_in, coll, ncoll, cap_coll, queue,
                                 cst, ncst, cap_cst, out, nout, cap_out, budget, st);
}

size_t tail_record_bytes() { return sizeof(TailRec); }

}  // namespace gp
