// gp_kernels_mixed.cu -- mixed-precision ADV_PARTICLE_ELLP: FP32 field and stencil
// weights with compensated FP32 sums, FP32 drag/lift/torque coefficients, FP64
// integration and renormalised quaternions.  Compiled with FMA contraction.
#include "gp_advance.cuh"
#include "gp_launch.h"

namespace gp {

template __global__ void k_integrate<true>(const InstDev *, const PoolView *, const PoolView *, const int32_t *,
                                            int64_t, const double *const *, uint32_t *, Status *);
template __global__ void k_integrate_fix<true>(const InstDev *, const PoolView *, const PoolView *, const PairRec *,
                                                const unsigned long long *, int64_t, const double *const *,
                                                uint32_t *, Status *);
template __global__ void k_gather<true>(const InstDev *, const PoolView *, const int32_t *, int64_t,
                                         double *const *, unsigned long long *, Status *);

void launch_gather_mixed(const InstDev *insts, const PoolView *pv, const int32_t *perm, int64_t n,
                      double *const *fluid, unsigned long long *ticket, Status *st, int grid, cudaStream_t s) {
  cudaMemsetAsync(ticket, 0, sizeof(unsigned long long), s);
  k_gather<true><<<grid, 256, 0, s>>>(insts, pv, perm, n, fluid, ticket, st);
}

void launch_integrate_mixed(const InstDev *insts, PoolView *pv, PoolView *pv_alt, const int32_t *perm, int64_t n,
                         double *const *fluid, Status *st, int grid, cudaStream_t s, uint32_t *mark) {
  k_integrate<true><<<grid, 128, 0, s>>>(insts, pv, pv_alt, perm, n, fluid, mark, st);
  if (mark == nullptr) k_swap_pool<<<1, 1, 0, s>>>(pv, pv_alt, st);
}

void launch_integrate_fix_mixed(const InstDev *insts, PoolView *pv, PoolView *pv_alt, const PairRec *pairs,
                             const unsigned long long *npairs, int64_t cap_pairs, double *const *fluid,
                             uint32_t *mark, Status *st, int grid, cudaStream_t s) {
  k_integrate_fix<true><<<grid, 128, 0, s>>>(insts, pv, pv_alt, pairs, npairs, cap_pairs, fluid, mark, st);
  k_swap_pool<<<1, 1, 0, s>>>(pv, pv_alt, st);
}

}  // namespace gp
