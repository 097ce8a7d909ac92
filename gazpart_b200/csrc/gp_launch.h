// gp_launch.h -- host-side launchers of the device kernels (one per translation unit
// so that the FP64 path can be compiled without FMA contraction).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include "gp_types.h"

namespace gp {

struct TailRec;   // gp_contact.cuh

// --- gp_kernels_fp64.cu (FP64 path, -fmad=false) ---
// ADV_PARTICLE_ELLP: advances particle perm[j] of *pv into slot j of *pv_alt, then swaps
// the two views (so *pv is current afterwards).  With mark non-null, the speculative
// pass: marked particles are left to launch_integrate_fix_*, which also swaps.
void launch_gather_fp64(const InstDev *insts, const PoolView *pv, const int32_t *perm, int64_t n,
                      double *const *fluid, unsigned long long *ticket, Status *st, int grid, cudaStream_t s);
void launch_integrate_fp64(const InstDev *insts, PoolView *pv, PoolView *pv_alt, const int32_t *perm, int64_t n,
                         double *const *fluid, Status *st, int grid, cudaStream_t s, uint32_t *mark = nullptr);
void launch_integrate_fix_fp64(const InstDev *insts, PoolView *pv, PoolView *pv_alt, const PairRec *pairs,
                             const unsigned long long *npairs, int64_t cap_pairs, double *const *fluid,
                             uint32_t *mark, Status *st, int grid, cudaStream_t s);
void launch_interp(const InstDev *inst, int comp, int64_t n, const double *x, const double *y, const double *z,
                   double *out, Status *st, cudaStream_t s);
void launch_frozen_interp(const double *xain, const double *yain, const double *zain, int nx, int ny, int nz,
                          const double *uain, int64_t n, const double *x, const double *y, const double *z,
                          double *out, Status *st, cudaStream_t s);
int contact_grid_blocks();
void launch_contact(const InstDev *insts, const PoolView *pv, const PairRec *pairs, const unsigned long long *npairs,
                    int64_t cap_pairs, const TailRec *in, const unsigned long long *nin, int64_t cap_in,
                    CollRec *coll, unsigned long long *ncoll, int64_t cap_coll, unsigned long long *queue,
                    ContactStatRec *cst, unsigned long long *ncst, int64_t cap_cst, TailRec *out,
                    unsigned long long *nout, int64_t cap_out, int budget, const uint32_t *order,
                    uint32_t *hist, int64_t nhist, Status *st, int grid, cudaStream_t s);
size_t tail_record_bytes();
// The contact queue's order for the candidate pairs (gp_contact.cu): bins holds
// 2 * kQueueBins counters, zero at the launch; key one byte per pair slot.
constexpr int kQueueBins = 256;
void launch_queue_order(const InstDev *insts, const PoolView *pv, const PairRec *pairs,
                        const unsigned long long *npairs, int64_t cap_pairs, const uint32_t *hist, int64_t nhist,
                        uint8_t *key, uint32_t *bins, uint32_t *order, const Status *st, int grid, cudaStream_t s);
void launch_response(const InstDev *insts, const PoolView *pv, const CollRec *coll, const unsigned long long *ncoll,
                     int64_t cap_coll, const int8_t *state, int32_t *acc_list, unsigned long long *nacc, Status *st,
                     int grid, cudaStream_t s);
// per-routine drop-ins (n items; all pointers device)
void launch_force_batch(int64_t n, const double *pcs /*n*10*/, double visc, const double *up,
                        const double *uf, const double *quat, double *fdrag, double *flift, Status *st,
                        cudaStream_t s);
void launch_torque_batch(int64_t n, const double *pcs, double visc, const double *omega, const double *quat,
                         const double *pup, const double *pufap, const double *pvort, double *tp, double *tr,
                         Status *st, cudaStream_t s);
void launch_quat_batch(int64_t n, double *quat, const double *omega, double dt, cudaStream_t s);
void launch_euler_batch(int64_t n, const double *ip /*n*3*/, double dt, double *omega, cudaStream_t s);
void launch_contact_batch(int64_t n, const double *shapes /*n*4: a1 b1 a2 b2*/, const double *centres,
                          const double *quats, int32_t *flag, double *e1, double *e2, double *cn, cudaStream_t s);
void launch_response_batch(int64_t n, double ecp, double mup, const double *ip /*n*3*/, double *p1 /*n*10*/,
                           double *p2, const double *r1, const double *r2, const double *nrm, Status *st,
                           cudaStream_t s);

// --- gp_gather_tma.cu: the FP32 gather with each stencil box staged by the TMA ---
// make_field_map: tensor map over one FP32 field slot ([z][y][x][8], the interior sizes
// given); gather_tma_prepare: the kernel's shared-memory limit, once, outside any stream
// capture; launch_gather_tma: as launch_gather_mixed, for instances that all read the
// mapped field.
int make_field_map(const void *field, int nx, int ny, int nz, CUtensorMap *out);
int gather_tma_prepare();
size_t gather_tma_smem_bytes();
void launch_gather_tma(const CUtensorMap &map, const InstDev *insts, const PoolView *pv, const int32_t *perm,
                       int64_t n, double *const *fluid, unsigned long long *ticket, Status *st, int grid,
                       cudaStream_t s);

// --- gp_stats.cu (-fmad=false) ---
void launch_stat_partfluid(const InstDev *insts, const PoolView *pv, int64_t n, int inst, double *const *fluid,
                           const int32_t *groups, int ngroups, double rhof, double ppi, double *partial,
                           int nblocks, double *out, Status *st, cudaStream_t s);
void launch_collision_stats(const CollRec *coll, const unsigned long long *ncoll, int64_t cap_coll,
                            const int8_t *state, unsigned long long *best1, unsigned long long *best2,
                            const ContactStatRec *rec, const unsigned long long *nrec, int64_t cap_rec,
                            const PoolView *pv, const int32_t *const *group_tab, const int32_t *ngroups, double *acc,
                            unsigned long long *steps, Status *st, cudaStream_t s);

// --- gp_kernels_mixed.cu ---
void launch_gather_mixed(const InstDev *insts, const PoolView *pv, const int32_t *perm, int64_t n,
                      double *const *fluid, unsigned long long *ticket, Status *st, int grid, cudaStream_t s);
void launch_integrate_mixed(const InstDev *insts, PoolView *pv, PoolView *pv_alt, const int32_t *perm, int64_t n,
                         double *const *fluid, Status *st, int grid, cudaStream_t s, uint32_t *mark = nullptr);
void launch_integrate_fix_mixed(const InstDev *insts, PoolView *pv, PoolView *pv_alt, const PairRec *pairs,
                             const unsigned long long *npairs, int64_t cap_pairs, double *const *fluid,
                             uint32_t *mark, Status *st, int grid, cudaStream_t s);
void launch_iota(int32_t *a, int64_t n, cudaStream_t s);

// --- gp_search.cu ---
void launch_bin_count(const InstDev *insts, const PoolView *pv, int64_t n, SearchArrays sa, Status *st, int grid,
                      cudaStream_t s);
void launch_scan(const int32_t *in, int32_t *out, int64_t n, int32_t *block_sums, cudaStream_t s);
int64_t scan_block_sums_size(int64_t n);
void launch_bin_scatter(const InstDev *insts, const PoolView *pv, int64_t n, SearchArrays sa, Status *st, int grid,
                        cudaStream_t s);
void launch_search(const InstDev *insts, int64_t n, SearchArrays sa, PairRec *pairs, unsigned long long *npairs,
                   int64_t cap_pairs, Status *st, int grid, cudaStream_t s);
void launch_match(const CollRec *coll, const unsigned long long *ncoll, int64_t cap_coll, unsigned long long *best1,
                  unsigned long long *best2, int8_t *matched, int8_t *state, Status *st, cudaStream_t s);
void launch_field_layout(void *dst, int prec, int nx, int ny, int nz, int ncomp, int comp, const double *src,
                         int src_layout, int ghost_mode, cudaStream_t s);
// state columns as bits (x y z u v w qa qb qc qd ox oy oz = bits 0..12)
constexpr unsigned kAllStateCols = (1u << kNState) - 1u;
constexpr unsigned kColsPosQuat = 0x3C7u;    // x y z qa qb qc qd: final once the integrate is done
constexpr unsigned kColsVelSpin = 0x1C38u;   // u v w ox oy oz: the response may still change them
constexpr unsigned kColsPos = 0x7u;          // x y z: all the gather reads
void launch_gather_state(const InstDev *insts, const PoolView *pv, int64_t n, int only, double *out,
                         double *const *fluid_cols, double *fluid_out, int64_t count, cudaStream_t s,
                         unsigned cols = kAllStateCols);
void launch_retire(const PoolView *pv, int64_t n, int inst, cudaStream_t s);
void launch_scatter_state(const InstDev *insts, const PoolView *pv, int64_t n, const double *cols,
                          int64_t count, cudaStream_t s, unsigned mask = kAllStateCols);
void launch_init_pool(const PoolView *pv, int64_t begin, int64_t n, int inst, const double *cols,
                      const double *pcs, int64_t ld, int64_t src, cudaStream_t s);
void launch_connectivity(int nxb, int nyb, int nzb, int periodicity, int32_t *ncon, int32_t *con, cudaStream_t s);

}  // namespace gp
