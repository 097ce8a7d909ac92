// gp_types.h -- device-side data structures shared by the kernels and the host API.
#pragma once
#include <cstdint>

#include "../../include/gazpart_gpu.h"

namespace gp {

// Per-ensemble record read by every kernel (one entry per instance; a single-ensemble
// context has one).  Mirrors the module variables the reference routines read.
struct InstDev {
  // particle range in the pool
  int64_t begin, count;
  // field
  const void *field;          // [z: nz+4][y: ny+4][x: nx+3][comp], float or double
  int32_t nx, ny, nz, ncomp;  // interior sizes
  int32_t fprec;              // GP_PREC_FP64 / GP_PREC_MIXED (float storage)
  int32_t periodicity, wall_boundary, store_fluid;
  double dx, dy, dz, lx, ly, lz;
  double visc, dtime, gravity, ecp, mup, ecw, muw;
  // collision box grid (collision_initiation.f90:44-103)
  int32_t nxbox, nybox, nzbox;
  int32_t frozen_flow;         // FROZEN_FLOW: 3 = channel (y and z wrap only)
  double dxbox, dybox, dzbox, xminbox, yminbox, zminbox;
  // search grid (cell edge >= 2 * largest bounding radius)
  int32_t nfx, nfy, nfz, pad1;
  double hfx, hfy, hfz, rmax;
  double rcut;                // particles with a larger bounding radius search a wider stencil
  int64_t cell_begin;         // first cell of this instance in the global cell arrays
};

// Double-buffered structure-of-arrays particle pool.  Column j of buffer b is
// col[b][j]; kernels read the buffer `cur` through perm and write buffer cur^1.
constexpr int kNState = 13;   // x y z u v w qa qb qc qd ox oy oz
constexpr int kNConst = 10;   // a b deq cdrag cpitch crot h5 ipxx ipyy ipzz
constexpr int kNFluid = 6;    // ufap vfap wfap vortx vorty vortz
constexpr int kFieldStride = 8; // field slots per grid point: the six components, padded

struct PoolView {
  double *st[kNState];
  double *pc[kNConst];
  int32_t *id;      // index within the instance (caller order)
  int32_t *inst;    // instance of the particle
};

// Device status word: first error code, the id that raised it, counters.
struct Status {
  int32_t code;
  int32_t first_inst;   // class of the first error + 1 (0: not a particle's error)
  long long first_id;
  unsigned long long n_near;      // candidate pairs within bounding distance
  unsigned long long n_contact;   // pairs in contact
  unsigned long long n_coll;      // colliding pairs (flag && NVREL < ZERO)
  unsigned long long n_accept;    // accepted (responded) pairs
  unsigned long long overflow;    // pairs dropped by a full buffer
  unsigned long long n_solve;     // contact solves run (pairs not proven disjoint)
  unsigned long long n_eval;      // function evaluations of those solves
  unsigned long long max_eval;    // largest evaluation count of one solve
  // A step whose candidate pairs outgrow the pair buffers sets `overflow` at its search;
  // from then on every step kernel returns at entry (step_halted), so that step stops
  // after its advance and later steps of a graph do nothing.  pairs_needed: the largest
  // candidate count such a step reached.  steps_done: steps whose response ran.
  unsigned long long pairs_needed;
  unsigned long long steps_done;
};

__device__ __forceinline__ bool step_halted(const Status *s) {
  return *reinterpret_cast<const volatile unsigned long long *>(&s->overflow) != 0ull;
}

__device__ inline void set_error(Status *s, int code, long long id, int inst = -1) {
  if (atomicCAS(&s->code, 0, code) == 0) {
    s->first_id = id;
    s->first_inst = inst + 1;
  }
}

// A candidate pair in the pool: HOME/NEAR pool slots plus the reference order key
// (IJK of HOME, index of HOME, stencil slot, index of NEAR), compared as (k1, k2).
struct PairRec {
  int32_t home, near;               // pool slots
  unsigned long long k1;            // IJK (1-based box id of HOME)
  unsigned long long k2;            // (id_home << 34) | (slot << 30) | id_near
};
constexpr int64_t kMaxInstanceParticles = (int64_t)1 << 30;
constexpr int kMaxClasses = 1024;   // classes (instances) per context

// A colliding pair with what COLLISION_RESPONSE needs.
struct CollRec {
  int32_t home, near;
  int32_t inst, pad;
  unsigned long long k1, k2;
  double rx1[3], rx2[3], cn[3];
};

// Statistics beside the step (gp_stats.cu).
constexpr int kNStatPartfluid = GP_NSTAT_PARTFLUID;   // MEAN_PARTFLUID(1:36, J, IDP)
constexpr int kNStatCollision = GP_NSTAT_COLLISION;   // MEAN_PART_COL(1:8, IDP1, IDP2)
constexpr int kStatMaxGroups = GP_STAT_MAX_GROUPS;    // polydisperse indices per class

// A pair found in contact, kept for the collision statistics when they are on:
// overlap depth |EPT1 - EPT2|, NVREL and |v_rel| (collision_interaction.f90:253-328).
struct ContactStatRec {
  int32_t home, near;
  int32_t inst, pad;
  unsigned long long k1, k2;
  double depth, nvrel, nrm;
};

// Binned particles of the collision search grid (see gp_search.cu).
struct SearchArrays {
  int32_t *cell_count;   // per search cell (+1 zero sentinel)
  int32_t *cell_start;   // exclusive scan, ncells+1
  int32_t *cell_fill;
  float *cell_rmax;       // per search cell: largest bounding radius of its small particles
  int32_t *cell_of;      // per pool slot
  int32_t *sorted;       // pool slot of each sorted position
  double *sx, *sy, *sz, *sr;
  float4 *spk;           // (x, y, z, r) in float for the conservative first test
  double *sex, *sey, *sez;   // symmetry axis in the lab frame (first column of R(q))
  double *sa2, *sb2;         // squared semi-axes along / across the axis
  long long *sbox;       // packed box coords (I0-1) | (J0-1)<<21 | (K0-1)<<42, -1 if outside
  int32_t *sinst;
  int32_t *sid;          // index of the particle within its instance
  uint32_t *mark;        // per pool slot, non-null when the search flags pair members (speculative integrate)
  int64_t ncells;
};

}  // namespace gp
