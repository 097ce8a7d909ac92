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

// ---------------------------------------------------------------------------
// Queue order.  A warp of k_contact runs as long as its slowest lane, and at 512^3 with
// 16.8 M spheroids a step holds about one solve per lane of the persistent grid, so the
// solves that share a warp decide how much of it idles: in queue order a warp holds 32
// solves of 3 to 300 evaluations.  A pair's solve takes about as many evaluations as it
// took in the last collision phase (the same two bodies, a few thousandths of their size
// further on; 98% of the pairs of a step were pairs in the step before), so the queue
// hands the pairs out in decreasing predicted length: long solves share warps and start
// first, short ones fill warps of their own.  The order decides only which lane solves a
// pair, never its result.
//
// hist[k] (k = the particle's instance begin + its id, below nhist) holds what the
// particle's solves took in the last collision phase: 0 nothing (no candidate pair), 1
// every pair proven apart before a solve, otherwise 1 + the largest evaluation count.  A
// pair's prediction is the smaller of its two particles' values, and a pair with no
// record at all (a new pair) is placed as a solve of typical length.
// ---------------------------------------------------------------------------
constexpr uint32_t kNewPairCost = 21;

__device__ __forceinline__ int64_t hist_index(const InstDev *__restrict__ insts, const PoolView &P, int slot) {
  return insts[P.inst[slot]].begin + P.id[slot];
}

// A pair proven apart without a solve, in the particles' record.  Out of line, so that
// the refill path keeps its registers.
static __device__ __noinline__ void record_apart(const InstDev *__restrict__ insts, const PoolView *__restrict__ pv,
                                                 const PairRec *__restrict__ pairs, int64_t e, uint32_t *hist,
                                                 int64_t nhist) {
  const PoolView &P = *pv;
  const PairRec pr = pairs[e];
  const int64_t g1 = hist_index(insts, P, pr.home), g2 = hist_index(insts, P, pr.near);
  if (g1 < nhist) atomicMax(&hist[g1], 1u);
  if (g2 < nhist) atomicMax(&hist[g2], 1u);
}

__global__ void k_queue_count(const InstDev *__restrict__ insts, const PoolView *__restrict__ pv,
                              const PairRec *__restrict__ pairs, const unsigned long long *__restrict__ npairs,
                              int64_t cap_pairs, const uint32_t *__restrict__ hist, int64_t nhist,
                              uint8_t *__restrict__ key, uint32_t *__restrict__ bins, const Status *st) {
  if (step_halted(st)) return;
  const PoolView P = *pv;
  const int64_t np = (int64_t)min(*npairs, (unsigned long long)cap_pairs);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t nround = (np + stride - 1) / stride * stride;   // whole warps stay in the loop
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nround; e += stride) {
    int k = -1;
    if (e < np) {
      const PairRec pr = pairs[e];
      const int64_t g1 = hist_index(insts, P, pr.home), g2 = hist_index(insts, P, pr.near);
      uint32_t p = (g1 < nhist && g2 < nhist) ? min(hist[g1], hist[g2]) : 0u;
      if (p == 0u) p = kNewPairCost;
      k = kQueueBins - 1 - (int)min(p, (uint32_t)(kQueueBins - 1));   // ascending bin = descending length
      key[e] = (uint8_t)k;
    }
    const unsigned peers = __match_any_sync(0xffffffffu, k);
    if (k >= 0 && (int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&bins[k], (uint32_t)__popc(peers));
  }
}

// order[start(bin) + fill] = e; every block forms the bins' starts itself (256 values).
// bins[0, kQueueBins) are the counts, bins[kQueueBins, 2 kQueueBins) the fill counters.
__global__ void k_queue_scatter(const unsigned long long *__restrict__ npairs, int64_t cap_pairs,
                                const uint8_t *__restrict__ key, uint32_t *__restrict__ bins,
                                uint32_t *__restrict__ order, const Status *st) {
  if (step_halted(st)) return;
  __shared__ uint32_t start[kQueueBins];
  if (threadIdx.x < 32) {
    uint32_t run = 0;
    for (int b0 = 0; b0 < kQueueBins; b0 += 32) {
      const uint32_t v = bins[b0 + threadIdx.x];
      uint32_t x = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if ((int)threadIdx.x >= o) x += y;
      }
      start[b0 + threadIdx.x] = run + x - v;
      run += __shfl_sync(0xffffffffu, x, 31);
    }
  }
  __syncthreads();
  const int64_t np = (int64_t)min(*npairs, (unsigned long long)cap_pairs);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t nround = (np + stride - 1) / stride * stride;
  const int lane = threadIdx.x & 31;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nround; e += stride) {
    const int k = (e < np) ? (int)key[e] : -1;
    const unsigned peers = __match_any_sync(0xffffffffu, k);
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (k >= 0 && lane == leader) base = atomicAdd(&bins[kQueueBins + k], (uint32_t)__popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (k >= 0) order[start[k] + base + __popc(peers & ((1u << lane) - 1u))] = (uint32_t)e;
  }
}

void launch_queue_order(const InstDev *insts, const PoolView *pv, const PairRec *pairs,
                        const unsigned long long *npairs, int64_t cap_pairs, const uint32_t *hist, int64_t nhist,
                        uint8_t *key, uint32_t *bins, uint32_t *order, const Status *st, int grid, cudaStream_t s) {
  k_queue_count<<<grid, 256, 0, s>>>(insts, pv, pairs, npairs, cap_pairs, hist, nhist, key, bins, st);
  k_queue_scatter<<<grid, 256, 0, s>>>(npairs, cap_pairs, key, bins, order, st);
}

// collision_interaction.f90:216-348 for every candidate pair: minimum image, contact
// (ellipsoid_contact_detection), contact-point velocities, NVREL.  Colliding pairs
// (flag && NVREL < ZERO) are appended.  Persistent warps with lane refill: a lane whose
// Levenberg-Marquardt solve has returned finishes its pair and takes the next one from
// a global queue, so warps do not idle on their slowest pair.  order (optional): the
// first pass takes the pairs in that order (the queue order above); hist (optional):
// each pair's outcome is recorded there for the next collision phase's order.
//
// Passes.  A warp runs as long as its slowest lane, and a step at 512^3 with 16.8 M
// spheroids has about one solve per lane of the persistent grid, so refilling cannot
// even out solves of 3 to 300 evaluations.  With `out` set, a solve still running after `budget` evaluations is
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
                                                    const uint32_t *__restrict__ order, uint32_t *hist,
                                                    int64_t nhist, Status *st) {
  if (step_halted(st)) return;
  const int64_t np = in ? (int64_t)min(*nin, (unsigned long long)cap_in)
                        : (int64_t)min(*npairs, (unsigned long long)cap_pairs);
  const unsigned lane = threadIdx.x & 31u;
  constexpr unsigned kFull = 0xffffffffu;
  bool active = false, exhausted = false;
  // With the order, each warp's first batch of 32 is fixed: warp w of block b takes batch
  // w * gridDim.x + b of the ordered pairs, so that every block holds one warp of the
  // longest solves, one of the next longest and so on.  Blocks then stay resident until
  // their longest solves end, as with the unordered queue, instead of short-solve blocks
  // leaving early and letting the overlapped gather take issue slots from the long
  // solves.  Later batches come from the counter, after the fixed ones.
  bool fixed = order != nullptr && in == nullptr;
  const unsigned long long lanes = (unsigned long long)gridDim.x * blockDim.x;
  int64_t e = 0;
  ContactProb CP;
  LmState S;
  for (;;) {
    if (!exhausted) {
      const unsigned want = __ballot_sync(kFull, !active);
      if (want) {
        unsigned long long base = 0;
        if (fixed) {
          base = ((unsigned long long)(threadIdx.x >> 5) * gridDim.x + blockIdx.x) * 32ull;
          fixed = false;
        } else {
          const int leader = __ffs(want) - 1;
          if ((int)lane == leader) base = atomicAdd(queue, (unsigned long long)__popc(want));
          base = __shfl_sync(kFull, base, leader);
          if (order != nullptr && in == nullptr) base += lanes;
        }
        if ((int64_t)base >= np) {
          exhausted = true;
        } else if (!active) {
          const int64_t q = (int64_t)base + __popc(want & ((1u << lane) - 1u));
          if (q < np && in) {
            resume_solve(insts, pv, pairs, in + q, e, CP, S);
            active = true;
          } else if (q < np) {
            e = order ? (int64_t)order[q] : q;
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
            } else if (hist) {
              record_apart(insts, pv, pairs, e, hist, nhist);
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
    finish_pair(insts, pv, pairs, e, S.x[0], S.x[1], S.nfev, coll, ncoll, cap_coll, cst, ncst, cap_cst, hist, nhist, st);
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
                    unsigned long long *nout, int64_t cap_out, int budget, const uint32_t *order,
                    uint32_t *hist, int64_t nhist, Status *st, int grid, cudaStream_t s) {
  k_contact<<<grid, 128, 0, s>>>(insts, pv, pairs, npairs, cap_pairs, in, nin, cap_in, coll, ncoll, cap_coll, queue,
                                 cst, ncst, cap_cst, out, nout, cap_out, budget, order, hist, nhist, st);
}

size_t tail_record_bytes() { return sizeof(TailRec); }

}  // namespace gp
