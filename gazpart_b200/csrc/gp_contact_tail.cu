// gp_contact_tail.cu -- the long contact solves, finished with the solver inlined.
//
// k_contact solves one pair per lane, many lanes per SM, which suits the bulk of short
// solves.  A solve still running after the contact-tail budget of evaluations can be
// handed over here: this kernel runs few threads, one per handed-over solve, spread over
// the SMs, with the whole Levenberg-Marquardt iteration inlined (this translation unit is
// compiled with GP_LM_INLINE).  The problem is rebuilt from the pool by the same set-up
// and the iterates are the same operations in the same order, so the results do not
// change.
#include "gp_contact.cuh"
#include "gp_launch.h"

namespace gp {

// One warp per block, at most 128 registers a thread by default: a block then fits in the
// registers the overlapped stencil gather leaves free on an SM (3 blocks of 256 threads
// at 80).
#ifndef GP_TAIL_MIN_BLOCKS
#define GP_TAIL_MIN_BLOCKS 16
#endif
__global__ void __launch_bounds__(32, GP_TAIL_MIN_BLOCKS) k_contact_tail(const InstDev *__restrict__ insts,
                               const PoolView *__restrict__ pv, const PairRec *__restrict__ pairs,
                               const TailRec *__restrict__ tail, const unsigned long long *__restrict__ ntail,
                               int64_t cap_tail, CollRec *__restrict__ coll, unsigned long long *ncoll,
                               int64_t cap_coll, ContactStatRec *__restrict__ cst, unsigned long long *ncst,
                               int64_t cap_cst, Status *st) {
  if (step_halted(st)) return;
  const int64_t nt = (int64_t)min(*ntail, (unsigned long long)cap_tail);
  // record r = thread * blocks + block: the records go round the SMs first
  for (int64_t r = (int64_t)threadIdx.x * gridDim.x + blockIdx.x; r < nt; r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = tail[r].e;
    LmState S = tail[r].S;
    const PairRec pr = pairs[e];
    PairBodies B;
    pair_bodies(insts, *pv, pr.home, pr.near, B);
    ContactProb CP;
    double xs[2];
    contact_setup(B.a1, B.b1, B.a2, B.b2, B.c1, B.q1, B.c2, B.q2, CP, xs);
    while (lm_step(CP, S, kContactTol) == 0) {
    }   // lm_step returns once nfev reaches maxfev = 300 at the latest
    finish_pair(insts, pv, pairs, e, S.x[0], S.x[1], S.nfev, coll, ncoll, cap_coll, cst, ncst, cap_cst, st);
  }
}

void launch_contact_tail(const InstDev *insts, const PoolView *pv, const PairRec *pairs, const TailRec *tail,
                         const unsigned long long *ntail, int64_t cap_tail, CollRec *coll, unsigned long long *ncoll,
                         int64_t cap_coll, ContactStatRec *cst, unsigned long long *ncst, int64_t cap_cst,
                         Status *st, cudaStream_t s) {
  k_contact_tail<<<148, 32, 0, s>>>(insts, pv, pairs, tail, ntail, cap_tail, coll, ncoll, cap_coll, cst, ncst, cap_cst,
                                    st);
}

size_t tail_record_bytes() { return sizeof(TailRec); }

}  // namespace gp
