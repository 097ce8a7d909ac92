// gp_contact_tail.cu -- the long contact solves, finished with the solver inlined.
//
// k_contact solves one pair per lane with the solver's pieces out of line (few
// registers, many resident warps), which suits the bulk of short solves.  A solve still
// running after GP contact-tail budget evaluations is handed over here: this kernel runs
// few threads, one per handed-over solve, spread over the SMs, with the whole
// Levenberg-Marquardt iteration inlined (this translation unit is compiled with
// GP_LM_INLINE), which shortens the dependent chain of one iteration.  The iterates are
// the same operations in the same order, so the results do not change.
#include "gp_contact.cuh"
#include "gp_launch.h"

namespace gp {

// One warp per block, at most 128 registers a thread by default: a block then fits in the
// registers the overlapped stencil gather leaves free on an SM (3 blocks of 256 threads
// at 80).
#ifndef GP_TAIL_MIN_BLOCKS
#define GP_TAIL_MIN_BLOCKS 16
#endif
__global__ void __launch_bounds__(32, GP_TAIL_MIN_BLOCKS) k_contact_tail(const PoolView *__restrict__ pv, const PairRec *__restrict__ pairs,
                               const TailRec *__restrict__ tail, const unsigned long long *__restrict__ ntail,
                               int64_t cap_tail, CollRec *__restrict__ coll, unsigned long long *ncoll,
                               int64_t cap_coll, ContactStatRec *__restrict__ cst, unsigned long long *ncst,
                               int64_t cap_cst, Status *st) {
  const PoolView P = *pv;
  const int64_t nt = (int64_t)min(*ntail, (unsigned long long)cap_tail);
  // record r = thread * blocks + block: the records go round the SMs first
  for (int64_t r = (int64_t)threadIdx.x * gridDim.x + blockIdx.x; r < nt; r += (int64_t)gridDim.x * blockDim.x) {
    TailRec t = tail[r];
    while (lm_step(t.CP, t.S, kContactTol) == 0) {
    }   // lm_step returns once nfev reaches maxfev = 300 at the latest
    finish_pair(P, pairs, t.e, t.CP, t.S, t.q1, t.q2, t.a1, t.b1, t.a2, t.b2, coll, ncoll, cap_coll, cst, ncst,
                cap_cst, st);
  }
}

void launch_contact_tail(const PoolView *pv, const PairRec *pairs, const TailRec *tail,
                         const unsigned long long *ntail, int64_t cap_tail, CollRec *coll, unsigned long long *ncoll,
                         int64_t cap_coll, ContactStatRec *cst, unsigned long long *ncst, int64_t cap_cst,
                         Status *st, cudaStream_t s) {
  k_contact_tail<<<148, 32, 0, s>>>(pv, pairs, tail, ntail, cap_tail, coll, ncoll, cap_coll, cst, ncst, cap_cst, st);
}

size_t tail_record_bytes() { return sizeof(TailRec); }

}  // namespace gp
