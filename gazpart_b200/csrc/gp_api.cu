// gp_api.cu -- host side of the C ABI declared in include/gazpart_gpu.h.
//
// A context owns: one CUDA stream, the interpolation field (device layout, see
// gp_advance.cuh), a structure-of-arrays particle pool, the ensemble table read by the
// kernels, the collision search buffers, a device status word and a captured CUDA
// graph of one step.  Host code here does set-up, bookkeeping and launches only; all
// per-particle and per-pair arithmetic runs in the kernels.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <thread>
#include <utility>
#include <vector>

#include <cuda.h>
#include <cuda_runtime.h>

#include "../../include/gazpart_gpu.h"
#include "gp_launch.h"
#include "gp_types.h"

using namespace gp;

#define GP_CK(call)                                                                               \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess) {                                                                      \
      std::fprintf(stderr, "gazpart_b200: %s failed: %s (%s:%d)\n", #call, cudaGetErrorString(e_), \
                   __FILE__, __LINE__);                                                           \
      return e_ == cudaErrorMemoryAllocation ? GP_ENOMEM : GP_ECUDA;                              \
    }                                                                                             \
  } while (0)

#define GP_TRY(expr)          \
  do {                        \
    int rc_ = (expr);         \
    if (rc_ != GP_OK) return rc_; \
  } while (0)

namespace {

constexpr int kPassCounters = 8;   // first contact-pass counter in gp_ctx::d_counters
constexpr int kMaxPasses = 8;      // contact passes at most (budget 1 takes 7)

template <typename T>
int dalloc(T **p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  GP_CK(cudaMalloc(reinterpret_cast<void **>(p), count * sizeof(T)));
  return GP_OK;
}

template <typename T>
void dfree(T *&p) {
  if (p) cudaFree(p);
  p = nullptr;
}

// Per-particle constants of the force/torque routines, computed with the reference's
// expressions on the host (fluid_force_ellipsoid.f90:59,70,119; fluid_torque_ellipsoid.f90:
// 85,96,147,158).  Order: a b deq cdrag cpitch crot h5 ipxx ipyy ipzz.
void part_const(double emaj, double apr, double rhop, double rhof, double ppi, double ipxx, double ipyy,
                double ipzz, double out[kNConst]) {
  const double pmass = rhop * (4.0 / 3.0) * ppi * std::pow(emaj, 3.0) / (apr * apr);
  const double deq = (2.0 * emaj) / std::pow(apr, 2.0 / 3.0);
  out[0] = emaj;
  out[1] = emaj / apr;
  out[2] = deq;
  out[3] = (1.0 / 2.0) * (rhof / pmass) * (1.0 / 4.0) * (ppi * (deq * deq));
  out[4] = (1.0 / 4.0) * (rhof / pmass) * (1.0 / 4.0) * ppi * (deq * deq * deq);
  out[5] = 0.5 * rhof / pmass;
  const double h = deq / 2.0, h2 = h * h;
  out[6] = h2 * h2 * h;
  out[7] = ipxx;
  out[8] = ipyy;
  out[9] = ipzz;
}

struct ClassProps {
  double emaj, apr, rhop;
};

}  // namespace

struct gp_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  // Second stream of a multi-step graph: the next step's stencil gather runs there
  // while the collision phase finishes on `stream`.
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // gp_step_host's copy/compute hand-offs (created on first use)
  cudaEvent_t ev_host[5] = {};
  // phase begin/end timestamps of the step being captured by gp_step_timed
  // ([2p] begin, [2p+1] end of phase p; null otherwise)
  cudaEvent_t *marks = nullptr;
  gp_params prm{};
  double ppi = 0.0;
  // field
  void *field = nullptr;
  size_t field_bytes = 0;
  double *stage = nullptr;
  size_t stage_count = 0;
  // Classes (the reference's IG = 1..NIG, PART(:, IG)), each an instance with its own
  // particle range, box grid and search-grid cells; `tmpl` holds the shared mesh,
  // physics and field.
  InstDev tmpl{};
  std::vector<InstDev> insts;      // by class slot; a retired slot has count 0
  std::vector<char> live;          // slot in use
  InstDev *d_inst = nullptr;
  // resident fields: slot 0 is the one gp_params describes, more come from gp_add_field
  struct FieldSlot {
    void *ptr = nullptr;
    int nx = 0, ny = 0, nz = 0;
    double lx = 0, ly = 0, lz = 0;
  };
  std::vector<FieldSlot> fields;
  std::vector<int> class_field;    // field slot of each class slot
  int64_t n_slots = 0;             // pool slots holding particles, retired ones included
  bool grid_ready = false;
  // pool
  int64_t cap = 0, n = 0;
  // two buffers: the advance reads one and writes the other in cell order
  double *d_st[2][kNState] = {};
  double *d_pc[2][kNConst] = {};
  double *d_fluid[kNFluid] = {};
  double **d_fluid_cols = nullptr;
  int32_t *d_id[2] = {}, *d_instof[2] = {};
  PoolView *d_pv = nullptr;       // current buffer
  PoolView *d_pv_alt = nullptr;   // the other one
  // search
  SearchArrays sa{};
  int32_t *d_scan_tmp = nullptr;
  int64_t ncells = 0, ncells_cap = 0;
  PairRec *d_pairs = nullptr;
  int64_t cap_pairs = 0;
  CollRec *d_coll = nullptr;
  int64_t cap_coll = 0;
  unsigned long long *d_counters = nullptr;   // [0] npairs [1] ncoll [2] nacc [4] contacts kept for the
                                              // statistics [6] the gather's work ticket [7] collision steps
                                              // in the statistics; from kPassCounters on, per contact pass,
                                              // its queue and the solves it hands over
  unsigned long long *d_best1 = nullptr, *d_best2 = nullptr;
  int8_t *d_matched = nullptr, *d_state = nullptr;
  int32_t *d_acc = nullptr;
  Status *d_status = nullptr;
  // scratch for per-routine calls
  double *d_scratch = nullptr;
  size_t scratch_count = 0;
  std::map<std::pair<int, int>, ClassProps> classes;
  // captured multi-step graphs, by step count
  std::map<int, cudaGraphExec_t> graphs;
  // launch grids (blocks), GP_TUNE_* order; gp_autotune picks them on the live workload
  int tune[GP_NTUNE] = {148 * 8, 148 * 4, 148 * 4, 148 * 4};
  // gather of step s+1 on the side stream, overlapping step s's contact solves; the
  // autotuner keeps it only where it shortens the step
  bool overlap = false;
  // with the overlap, step s+1's integrate also runs on the side stream, speculatively,
  // for the particles in no candidate pair of step s; the rest follow after the response
  // (d_mark: per pool slot, zero between steps; allocated while spec is on)
  bool spec = false;
  uint32_t *d_mark = nullptr;
  int64_t cap_mark = 0;
  int contact_grid = 148 * 4;   // persistent k_contact grid (resident blocks)
  // statistics beside the step: polydisperse index of each particle per class slot
  // (device arrays by particle id, null = all 1), the fluid sample the last step left
  // at each particle, the collision statistics' contact records and sums
  std::vector<int32_t *> group_dev;
  std::vector<int32_t> group_n;
  int32_t **d_group_tab = nullptr;      // [kMaxClasses]
  int32_t *d_group_n = nullptr;         // [kMaxClasses]
  bool fluid_ok = false;
  bool colstats = false;
  ContactStatRec *d_cst = nullptr;
  int64_t cap_cst = 0;
  double *d_colacc = nullptr;           // [kMaxClasses][G][G][GP_NSTAT_COLLISION]
  double *d_stat_partial = nullptr, *d_stat_out = nullptr;
  // contact passes: a solve still running after tail_budget evaluations (0: never) moves
  // to the next pass of the contact kernel, whose budget is three times larger, until a
  // last pass without one; the passes hand over through two alternating buffers
  TailRec *d_tail[2] = {nullptr, nullptr};
  int64_t cap_tail = 0;
  int tail_budget = 0;
  // contact queue order (gp_contact.cu): what each particle's solves took in the last
  // collision phase (d_evhist, by instance begin + id), each candidate pair's bin and the
  // pairs in decreasing predicted length.  Optional: where there is no room it stays off.
  bool qorder_on = true;
  uint32_t *d_evhist = nullptr;
  int64_t cap_evhist = 0;
  uint32_t *d_qorder = nullptr;
  uint8_t *d_qkey = nullptr;
  int64_t cap_qorder = 0;
  uint32_t *d_qbins = nullptr;   // 2 * kQueueBins
  // the mixed gather's staging: 0 stencil rows through L1, 1 each stencil box staged in
  // shared memory by the TMA (gp_gather_tma.cu), over gmap, the tensor map of gmap_field
  int gather_staging = 0;
  CUtensorMap gmap{};
  const void *gmap_field = nullptr;
  int gmap_dims[3] = {0, 0, 0};
};

namespace {

int ensure_scratch(gp_ctx *c, size_t count) {
  if (c->scratch_count >= count) return GP_OK;
  dfree(c->d_scratch);
  c->scratch_count = 0;
  GP_TRY(dalloc(&c->d_scratch, count));
  c->scratch_count = count;
  return GP_OK;
}

void drop_graph(gp_ctx *c) {
  for (auto &g : c->graphs) cudaGraphExecDestroy(g.second);
  c->graphs.clear();
}

int upload_inst(gp_ctx *c) {
  const std::vector<InstDev> &v = c->insts.empty() ? std::vector<InstDev>{c->tmpl} : c->insts;
  GP_CK(cudaMemcpyAsync(c->d_inst, v.data(), v.size() * sizeof(InstDev), cudaMemcpyHostToDevice, c->stream));
  GP_CK(cudaStreamSynchronize(c->stream));
  return GP_OK;
}

int copy_in(gp_ctx *c, double *dst, const double *src, size_t count, int on_device) {
  GP_CK(cudaMemcpyAsync(dst, src, count * sizeof(double), on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                        c->stream));
  return GP_OK;
}

int class_props(gp_ctx *c, int ig, int idp, double pc[kNConst]) {
  auto it = c->classes.find({ig, idp});
  if (it == c->classes.end()) return GP_EBADARG;
  const ClassProps &p = it->second;
  // initiation_particle_position.f90:609-634
  const double a = p.emaj, b = a / p.apr, cc = b;
  const double ipxx = (b * b + cc * cc) / 5.0, ipyy = (a * a + cc * cc) / 5.0, ipzz = (a * a + b * b) / 5.0;
  part_const(p.emaj, p.apr, p.rhop, c->prm.rhof, c->ppi, ipxx, ipyy, ipzz, pc);
  return GP_OK;
}

void free_search(gp_ctx *c) {
  dfree(c->sa.cell_count); dfree(c->sa.cell_start); dfree(c->sa.cell_fill); dfree(c->sa.cell_rmax);
  dfree(c->d_scan_tmp);
  c->ncells_cap = 0;
}

void free_pool(gp_ctx *c) {
  for (int b = 0; b < 2; ++b) {
    for (auto &p : c->d_st[b]) dfree(p);
    for (auto &p : c->d_pc[b]) dfree(p);
    dfree(c->d_id[b]);
    dfree(c->d_instof[b]);
  }
  for (auto &p : c->d_fluid) dfree(p);
  dfree(c->sa.cell_of); dfree(c->sa.sorted); dfree(c->sa.sx); dfree(c->sa.sy); dfree(c->sa.sz); dfree(c->sa.sr);
  dfree(c->sa.sbox); dfree(c->sa.sinst); dfree(c->sa.sid);
  dfree(c->sa.spk); dfree(c->sa.sex); dfree(c->sa.sey); dfree(c->sa.sez); dfree(c->sa.sa2); dfree(c->sa.sb2);
  dfree(c->d_best1); dfree(c->d_best2); dfree(c->d_matched);
  dfree(c->d_pairs); dfree(c->d_coll); dfree(c->d_state); dfree(c->d_acc);
  dfree(c->d_mark);
  c->cap_mark = 0;
  dfree(c->d_evhist); dfree(c->d_qorder); dfree(c->d_qkey);
  c->cap_evhist = 0;
  c->cap_qorder = 0;
  c->cap = 0;
}

// The contact queue's order buffers: the particles' record (zero) for `cap` particles,
// and the order and bin of each of `cap_pairs` pairs.  The order is optional: where
// there is no room it stays off, and a failed allocation's error is cleared so that later
// launch checks do not read it.
void try_qorder(gp_ctx *c) {
  if (c->cap_evhist < c->cap) {
    dfree(c->d_evhist);
    c->cap_evhist = 0;
    if (dalloc(&c->d_evhist, (size_t)c->cap) == GP_OK &&
        cudaMemsetAsync(c->d_evhist, 0, (size_t)c->cap * sizeof(uint32_t), c->stream) == cudaSuccess)
      c->cap_evhist = c->cap;
  }
  if (c->cap_qorder < c->cap_pairs) {
    dfree(c->d_qorder); dfree(c->d_qkey);
    c->cap_qorder = 0;
    if (dalloc(&c->d_qorder, (size_t)c->cap_pairs) == GP_OK && dalloc(&c->d_qkey, (size_t)c->cap_pairs) == GP_OK)
      c->cap_qorder = c->cap_pairs;
  }
  cudaGetLastError();
}

bool qorder_ready(const gp_ctx *c) {
  return c->qorder_on && c->d_qbins && c->cap_evhist >= c->cap && c->cap_evhist >= c->n_slots &&
         c->cap_qorder >= c->cap_pairs;
}

// The speculative integrate's marks, one per pool slot, all zero.
int ensure_mark(gp_ctx *c) {
  if (c->cap_mark >= c->cap) return GP_OK;
  dfree(c->d_mark);
  c->cap_mark = 0;
  GP_TRY(dalloc(&c->d_mark, (size_t)c->cap));
  GP_CK(cudaMemsetAsync(c->d_mark, 0, (size_t)c->cap * sizeof(uint32_t), c->stream));
  c->cap_mark = c->cap;
  return GP_OK;
}

// The marks are optional: where there is no room for them the speculative integrate
// stays off.  A failed allocation also leaves its error as the runtime's last error,
// which later launch checks would read, so it is cleared here.
bool try_mark(gp_ctx *c) {
  if (ensure_mark(c) == GP_OK) return true;
  cudaGetLastError();
  return false;
}

int alloc_pool(gp_ctx *c, int64_t cap) {
  free_pool(c);
  for (int b = 0; b < 2; ++b) {
    for (auto &p : c->d_st[b]) GP_TRY(dalloc(&p, cap));
    for (auto &p : c->d_pc[b]) GP_TRY(dalloc(&p, cap));
    GP_TRY(dalloc(&c->d_id[b], cap));
    GP_TRY(dalloc(&c->d_instof[b], cap));
    GP_CK(cudaMemsetAsync(c->d_instof[b], 0xFF, cap * sizeof(int32_t), c->stream));   // -1: empty slot
  }
  for (auto &p : c->d_fluid) GP_TRY(dalloc(&p, cap));   // interpolated field at each particle
  SearchArrays &sa = c->sa;
  GP_TRY(dalloc(&sa.cell_of, cap)); GP_TRY(dalloc(&sa.sorted, cap));
  GP_TRY(dalloc(&sa.sx, cap)); GP_TRY(dalloc(&sa.sy, cap)); GP_TRY(dalloc(&sa.sz, cap)); GP_TRY(dalloc(&sa.sr, cap));
  GP_TRY(dalloc(&sa.sbox, cap)); GP_TRY(dalloc(&sa.sinst, cap)); GP_TRY(dalloc(&sa.sid, cap));
  GP_TRY(dalloc(&sa.spk, cap)); GP_TRY(dalloc(&sa.sex, cap)); GP_TRY(dalloc(&sa.sey, cap)); GP_TRY(dalloc(&sa.sez, cap));
  GP_TRY(dalloc(&sa.sa2, cap)); GP_TRY(dalloc(&sa.sb2, cap));
  GP_TRY(dalloc(&c->d_best1, cap)); GP_TRY(dalloc(&c->d_best2, cap)); GP_TRY(dalloc(&c->d_matched, cap));
  GP_CK(cudaMemsetAsync(c->d_best1, 0xFF, cap * sizeof(unsigned long long), c->stream));
  GP_CK(cudaMemsetAsync(c->d_best2, 0xFF, cap * sizeof(unsigned long long), c->stream));
  GP_CK(cudaMemsetAsync(c->d_matched, 0, cap, c->stream));
  c->cap_pairs = std::max<int64_t>(int64_t(1) << 20, cap);
  c->cap_coll = std::max<int64_t>(int64_t(1) << 18, cap / 4);
  GP_TRY(dalloc(&c->d_pairs, c->cap_pairs));
  GP_TRY(dalloc(&c->d_coll, c->cap_coll));
  GP_TRY(dalloc(&c->d_state, c->cap_coll));
  GP_TRY(dalloc(&c->d_acc, c->cap_coll));
  c->cap = cap;
  PoolView pv[2];
  for (int b = 0; b < 2; ++b) {
    for (int k = 0; k < kNState; ++k) pv[b].st[k] = c->d_st[b][k];
    for (int k = 0; k < kNConst; ++k) pv[b].pc[k] = c->d_pc[b][k];
    pv[b].id = c->d_id[b];
    pv[b].inst = c->d_instof[b];
  }
  GP_CK(cudaMemcpyAsync(c->d_pv, &pv[0], sizeof(PoolView), cudaMemcpyHostToDevice, c->stream));
  GP_CK(cudaMemcpyAsync(c->d_pv_alt, &pv[1], sizeof(PoolView), cudaMemcpyHostToDevice, c->stream));
  GP_CK(cudaStreamSynchronize(c->stream));
  GP_CK(cudaMemcpyAsync(c->d_fluid_cols, c->d_fluid, sizeof(c->d_fluid), cudaMemcpyHostToDevice, c->stream));
  if (c->colstats && c->cap_cst < c->cap_pairs) {   // every candidate pair may be in contact
    dfree(c->d_cst);
    c->cap_cst = 0;
    GP_TRY(dalloc(&c->d_cst, (size_t)c->cap_pairs));
    c->cap_cst = c->cap_pairs;
  }
  if (c->spec && !try_mark(c)) c->spec = false;
  try_qorder(c);
  return GP_OK;
}

// COLLISION_INITIATION (collision_initiation.f90:44-103, INIT_GRID=2, NPROC=1) and the
// search grid.
int setup_grids(InstDev &I, double max_emaj, double rmax, double rsmall, int64_t cell_begin) {
  const double zero_ref = 1.0e-33;
  const double dpmax = 2.0 * max_emaj;
  double dxbox = 2.0 * dpmax;
  I.nxbox = (int32_t)(I.lx / dxbox);
  if (I.nxbox < 3) return GP_EBADARG;
  I.dxbox = I.lx / (double)I.nxbox;
  I.xminbox = (double)(1 - 1) * I.dx;
  I.yminbox = I.dy * (double)(1 - 1) - zero_ref;
  const double ymaxbox = I.dy * (double)(I.ny - 1) + I.dy + zero_ref;
  I.zminbox = I.dz * (double)(1 - 1) - zero_ref;
  const double zmaxbox = I.dz * (double)(I.nz - 1) + I.dz + zero_ref;
  I.nybox = (int32_t)((ymaxbox - I.yminbox) / I.dxbox);
  I.nzbox = (int32_t)((zmaxbox - I.zminbox) / I.dxbox);
  if (I.nybox < 3 || I.nzbox < 3) return GP_EBADARG;
  if (I.nxbox >= (1 << 21) || I.nybox >= (1 << 21) || I.nzbox >= (1 << 21)) return GP_EBADARG;
  I.dybox = (ymaxbox - I.yminbox) / (double)I.nybox;
  I.dzbox = (zmaxbox - I.zminbox) / (double)I.nzbox;
  // search grid: about two particles per cell, cell edge >= 2 rsmall (1+1e-6) so that
  // all but the largest bounding radii fit the one-cell half stencil
  const double hmin = 2.0 * rsmall * (1.0 + 1.0e-6);
  const int64_t target =
      std::max<int64_t>(3, (int64_t)std::ceil(std::cbrt((double)std::max<int64_t>(I.count, 1) / 2.0)));
  auto nf = [&](double L) {
    int64_t m = (int64_t)std::floor(L / hmin);
    return (int32_t)std::min<int64_t>(m, std::max<int64_t>(target, 3));
  };
  I.nfx = nf(I.lx); I.nfy = nf(I.ly); I.nfz = nf(I.lz);
  if (I.nfx < 3 || I.nfy < 3 || I.nfz < 3) return GP_EBADARG;
  I.hfx = I.lx / I.nfx; I.hfy = I.ly / I.nfy; I.hfz = I.lz / I.nfz;
  I.rmax = rmax;
  I.rcut = 0.5 * std::min(I.hfx, std::min(I.hfy, I.hfz)) / (1.0 + 1.0e-6);
  I.cell_begin = cell_begin;
  const int64_t ncells = (int64_t)I.nfx * I.nfy * I.nfz;
  if (ncells >= (int64_t(1) << 31) - 2) return GP_EBADARG;
  return GP_OK;
}

int alloc_cells(gp_ctx *c, int64_t ncells) {
  if (ncells >= (int64_t(1) << 31) - 2) return GP_EBADARG;
  if (ncells > c->ncells_cap) {
    free_search(c);
    GP_TRY(dalloc(&c->sa.cell_count, ncells + 1));
    GP_TRY(dalloc(&c->sa.cell_start, ncells + 1));
    GP_TRY(dalloc(&c->sa.cell_fill, ncells + 1));
    GP_TRY(dalloc(&c->sa.cell_rmax, ncells + 1));
    GP_TRY(dalloc(&c->d_scan_tmp, (size_t)scan_block_sums_size(ncells)));
    c->ncells_cap = ncells;
  }
  c->ncells = ncells;
  c->sa.ncells = ncells;
  return GP_OK;
}

// Records timestamp `slot` of the step being timed (an external record is a timestamp
// node of the captured graph); a no-op outside gp_step_timed.
int mark(gp_ctx *c, int slot, cudaStream_t s) {
  if (!c->marks) return GP_OK;
  GP_CK(cudaEventRecordWithFlags(c->marks[slot], s, cudaEventRecordExternal));
  return GP_OK;
}

// The one field every live class reads (the TMA-staged gather maps a single field), or
// false when they read several.
bool single_field(const gp_ctx *c, const InstDev **out) {
  const InstDev *f = nullptr;
  if (c->insts.empty()) {
    f = &c->tmpl;
  } else {
    for (size_t k = 0; k < c->insts.size(); ++k) {
      if (!c->live[k]) continue;
      const InstDev &I = c->insts[k];
      if (f && (I.field != f->field || I.nx != f->nx || I.ny != f->ny || I.nz != f->nz)) return false;
      if (!f) f = &I;
    }
  }
  if (!f || !f->field) return false;
  *out = f;
  return true;
}

// The tensor map of the single field, made again when the field or its mesh changed.
int ensure_field_map(gp_ctx *c) {
  const InstDev *f = nullptr;
  if (c->prm.precision != GP_PREC_MIXED || !single_field(c, &f)) return GP_EBADARG;
  if (c->gmap_field == f->field && c->gmap_dims[0] == f->nx && c->gmap_dims[1] == f->ny && c->gmap_dims[2] == f->nz)
    return GP_OK;
  c->gmap_field = nullptr;
  GP_TRY(make_field_map(f->field, f->nx, f->ny, f->nz, &c->gmap));
  c->gmap_field = f->field;
  c->gmap_dims[0] = f->nx; c->gmap_dims[1] = f->ny; c->gmap_dims[2] = f->nz;
  return GP_OK;
}

// Stencil gather at x_n for the particles in the last binning's order, on stream s.
int enqueue_gather(gp_ctx *c, cudaStream_t s) {
  GP_TRY(mark(c, 2 * GP_PHASE_GATHER, s));
  if (c->prm.precision == GP_PREC_MIXED && c->gather_staging == 1 && ensure_field_map(c) == GP_OK)
    // two blocks of four warps per SM are resident; the warps take their runs from the
    // ticket, so more blocks would only wait
    launch_gather_tma(c->gmap, c->d_inst, c->d_pv, c->sa.sorted, c->n, c->d_fluid_cols, c->d_counters + 6,
                      c->d_status, 148 * 2, s);
  else if (c->prm.precision == GP_PREC_MIXED)
    launch_gather_mixed(c->d_inst, c->d_pv, c->sa.sorted, c->n, c->d_fluid_cols, c->d_counters + 6, c->d_status,
                        c->tune[GP_TUNE_GATHER], s);
  else
    launch_gather_fp64(c->d_inst, c->d_pv, c->sa.sorted, c->n, c->d_fluid_cols, c->d_counters + 6, c->d_status,
                       c->tune[GP_TUNE_GATHER], s);
  GP_CK(cudaGetLastError());
  return mark(c, 2 * GP_PHASE_GATHER + 1, s);
}

int enqueue_integrate(gp_ctx *c) {
  GP_TRY(mark(c, 2 * GP_PHASE_INTEGRATE, c->stream));
  if (c->prm.precision == GP_PREC_MIXED)
    launch_integrate_mixed(c->d_inst, c->d_pv, c->d_pv_alt, c->sa.sorted, c->n, c->d_fluid_cols, c->d_status,
                           c->tune[GP_TUNE_INTEGRATE], c->stream);
  else
    launch_integrate_fp64(c->d_inst, c->d_pv, c->d_pv_alt, c->sa.sorted, c->n, c->d_fluid_cols, c->d_status,
                          c->tune[GP_TUNE_INTEGRATE], c->stream);
  GP_CK(cudaGetLastError());
  c->n_slots = c->n;   // the pass writes the active particles, in cell order, to slots [0, n)
  c->fluid_ok = true;  // and the fluid it used, at the same slots
  return mark(c, 2 * GP_PHASE_INTEGRATE + 1, c->stream);
}

// Speculative integrate of the next step on stream s (the side stream): the particles
// the last search did not mark; no swap.
int enqueue_integrate_spec(gp_ctx *c, cudaStream_t s) {
  if (c->prm.precision == GP_PREC_MIXED)
    launch_integrate_mixed(c->d_inst, c->d_pv, c->d_pv_alt, c->sa.sorted, c->n, c->d_fluid_cols, c->d_status,
                           c->tune[GP_TUNE_INTEGRATE], s, c->d_mark);
  else
    launch_integrate_fp64(c->d_inst, c->d_pv, c->d_pv_alt, c->sa.sorted, c->n, c->d_fluid_cols, c->d_status,
                          c->tune[GP_TUNE_INTEGRATE], s, c->d_mark);
  GP_CK(cudaGetLastError());
  return GP_OK;
}

// Its completion after the response: the marked particles, then the swap.  Timed as the
// step's integrate phase.
int enqueue_integrate_fix(gp_ctx *c) {
  GP_TRY(mark(c, 2 * GP_PHASE_INTEGRATE, c->stream));
  if (c->prm.precision == GP_PREC_MIXED)
    launch_integrate_fix_mixed(c->d_inst, c->d_pv, c->d_pv_alt, c->d_pairs, c->d_counters + 0, c->cap_pairs,
                               c->d_fluid_cols, c->d_mark, c->d_status, 148 * 4, c->stream);
  else
    launch_integrate_fix_fp64(c->d_inst, c->d_pv, c->d_pv_alt, c->d_pairs, c->d_counters + 0, c->cap_pairs,
                              c->d_fluid_cols, c->d_mark, c->d_status, 148 * 4, c->stream);
  GP_CK(cudaGetLastError());
  c->n_slots = c->n;
  c->fluid_ok = true;
  return mark(c, 2 * GP_PHASE_INTEGRATE + 1, c->stream);
}

int enqueue_advance(gp_ctx *c) {
  GP_TRY(enqueue_gather(c, c->stream));
  return enqueue_integrate(c);
}

// Binning of the search grid (also the cell order the next advance moves to).
int enqueue_bin(gp_ctx *c) {
  SearchArrays sa = c->sa;
  GP_CK(cudaMemsetAsync(sa.cell_count, 0, (c->ncells + 1) * sizeof(int32_t), c->stream));
  GP_CK(cudaMemsetAsync(sa.cell_fill, 0, (c->ncells + 1) * sizeof(int32_t), c->stream));
  GP_CK(cudaMemsetAsync(sa.cell_rmax, 0, (c->ncells + 1) * sizeof(float), c->stream));
  GP_CK(cudaMemsetAsync(c->d_counters, 0, 6 * sizeof(unsigned long long), c->stream));
  launch_bin_count(c->d_inst, c->d_pv, c->n_slots, sa, c->d_status, c->tune[GP_TUNE_BIN], c->stream);
  launch_scan(sa.cell_count, sa.cell_start, c->ncells, c->d_scan_tmp, c->stream);
  launch_bin_scatter(c->d_inst, c->d_pv, c->n_slots, sa, c->d_status, c->tune[GP_TUNE_BIN], c->stream);
  GP_CK(cudaGetLastError());
  return GP_OK;
}

// Binning and the candidate-pair search; flag: mark the members of the stored pairs.
int enqueue_bin_search(gp_ctx *c, bool flag = false) {
  SearchArrays sa = c->sa;
  sa.mark = flag ? c->d_mark : nullptr;
  GP_TRY(mark(c, 2 * GP_PHASE_BIN, c->stream));
  GP_TRY(enqueue_bin(c));
  GP_TRY(mark(c, 2 * GP_PHASE_BIN + 1, c->stream));
  GP_TRY(mark(c, 2 * GP_PHASE_SEARCH, c->stream));
  // a step with more candidates than either pair buffer holds halts after the search
  launch_search(c->d_inst, c->n, sa, c->d_pairs, c->d_counters + 0, std::min(c->cap_pairs, c->cap_coll),
                c->d_status, c->tune[GP_TUNE_SEARCH], c->stream);
  // The contact queue's order: the pairs in decreasing predicted length, from the
  // particles' record of the last collision phase, which is then cleared for this one.
  // It is formed here, before a multi-step graph forks the next gather onto the side
  // stream, so that the contact kernel is the first work ready after the fork and its
  // persistent grid takes the SMs before the gather's blocks do.
  if (qorder_ready(c)) {
    GP_CK(cudaMemsetAsync(c->d_qbins, 0, 2 * kQueueBins * sizeof(uint32_t), c->stream));
    launch_queue_order(c->d_inst, c->d_pv, c->d_pairs, c->d_counters + 0, c->cap_pairs, c->d_evhist, c->n_slots,
                       c->d_qkey, c->d_qbins, c->d_qorder, c->d_status, 148 * 4, c->stream);
    GP_CK(cudaMemsetAsync(c->d_evhist, 0, (size_t)c->n_slots * sizeof(uint32_t), c->stream));
  }
  GP_CK(cudaGetLastError());
  return mark(c, 2 * GP_PHASE_SEARCH + 1, c->stream);
}

// Contact solves, greedy acceptance and the impulse response.
int enqueue_contact_response(gp_ctx *c) {
  GP_TRY(mark(c, 2 * GP_PHASE_CONTACT, c->stream));
  ContactStatRec *cst = c->colstats ? c->d_cst : nullptr;
  // pass p: budget tail_budget * 3^p while below MINPACK's maxfev (300), then a last
  // pass without one; pass p takes its work from counter kPassCounters + 2p and hands
  // over through counter kPassCounters + 2p + 1
  int budget[kMaxPasses], npass = 0;
  for (int b = c->tail_budget; b > 0 && b < 300 && npass < kMaxPasses - 1; b *= 3) budget[npass++] = b;
  budget[npass++] = 0;
  unsigned long long *pc = c->d_counters + kPassCounters;
  GP_CK(cudaMemsetAsync(pc, 0, 2 * kMaxPasses * sizeof(unsigned long long), c->stream));
  // the first pass takes the pairs in the order enqueue_bin_search formed
  const bool order = qorder_ready(c);
  const int64_t nhist = order ? c->n_slots : 0;
  for (int p = 0; p < npass; ++p) {
    const bool last = p == npass - 1;
    const TailRec *in = p > 0 ? c->d_tail[(p - 1) & 1] : nullptr;
    TailRec *out = last ? nullptr : c->d_tail[p & 1];
    launch_contact(c->d_inst, c->d_pv, c->d_pairs, c->d_counters + 0, c->cap_pairs, in,
                   p > 0 ? pc + 2 * (p - 1) + 1 : nullptr, c->cap_tail, c->d_coll, c->d_counters + 1, c->cap_coll,
                   pc + 2 * p, cst, c->d_counters + 4, c->cap_cst, out, pc + 2 * p + 1, c->cap_tail, budget[p],
                   (order && p == 0) ? c->d_qorder : nullptr, order ? c->d_evhist : nullptr, nhist,
                   c->d_status, c->contact_grid, c->stream);
  }
  GP_TRY(mark(c, 2 * GP_PHASE_CONTACT + 1, c->stream));
  GP_TRY(mark(c, 2 * GP_PHASE_RESPONSE, c->stream));
  launch_match(c->d_coll, c->d_counters + 1, c->cap_coll, c->d_best1, c->d_best2, c->d_matched, c->d_state,
               c->d_status, c->stream);
  launch_response(c->d_inst, c->d_pv, c->d_coll, c->d_counters + 1, c->cap_coll, c->d_state, c->d_acc,
                  c->d_counters + 2, c->d_status, 148 * 4, c->stream);
  if (c->colstats)
    launch_collision_stats(c->d_coll, c->d_counters + 1, c->cap_coll, c->d_state, c->d_best1, c->d_best2, c->d_cst,
                           c->d_counters + 4, c->cap_cst, c->d_pv, c->d_group_tab, c->d_group_n, c->d_colacc,
                           c->d_counters + 7, c->d_status, c->stream);
  GP_CK(cudaGetLastError());
  return mark(c, 2 * GP_PHASE_RESPONSE + 1, c->stream);
}

int enqueue_collision(gp_ctx *c) {
  GP_TRY(enqueue_bin_search(c));
  return enqueue_contact_response(c);
}

// nsteps x (ADV_PARTICLE_ELLP + COLLISION) for capture into one graph.  The response
// changes only velocities and angular velocities, so the gather of step s+1, which
// reads positions and the order of step s's binning, is forked onto the side stream
// right after step s's search and overlaps its contact solves; step s+1's integrate
// joins it.  With spec, step s+1's integrate of every particle outside step s's
// candidate pairs (which the response cannot touch) follows the gather on the side
// stream, and only the pair members are integrated after the join.  marks:
// 2*GP_NPHASE timestamps per step, or null.
int enqueue_steps(gp_ctx *c, int nsteps, cudaEvent_t *marks) {
  auto marks_of = [&](int s) { return marks ? marks + (size_t)s * 2 * GP_NPHASE : nullptr; };
  const bool spec = c->overlap && c->spec && c->d_mark != nullptr && c->cap_mark >= c->cap && nsteps > 1;
  c->marks = marks_of(0);
  int rc = GP_OK;
  if (spec && cudaMemsetAsync(c->d_mark, 0, (size_t)c->cap * sizeof(uint32_t), c->stream) != cudaSuccess)
    rc = GP_ECUDA;
  if (!rc) rc = enqueue_gather(c, c->stream);
  for (int s = 0; s < nsteps && !rc; ++s) {
    c->marks = marks_of(s);
    if (s > 0 && c->overlap && cudaStreamWaitEvent(c->stream, c->ev_join, 0) != cudaSuccess) rc = GP_ECUDA;
    if (s > 0 && !c->overlap && !rc) rc = enqueue_gather(c, c->stream);
    if (!rc) rc = (s > 0 && spec) ? enqueue_integrate_fix(c) : enqueue_integrate(c);
    const bool fork = c->overlap && s + 1 < nsteps;
    if (!rc) rc = enqueue_bin_search(c, spec && fork);
    if (!rc && fork && cudaEventRecord(c->ev_fork, c->stream) != cudaSuccess) rc = GP_ECUDA;
    // the contact kernel is captured first so that its persistent grid is resident
    // before the gather's blocks queue for the SMs it leaves as its queue drains
    if (!rc) rc = enqueue_contact_response(c);
    if (!rc && fork) {
      if (cudaStreamWaitEvent(c->side, c->ev_fork, 0) != cudaSuccess) rc = GP_ECUDA;
      c->marks = marks_of(s + 1);
      if (!rc) rc = enqueue_gather(c, c->side);
      if (!rc && spec) rc = enqueue_integrate_spec(c, c->side);
      c->marks = marks_of(s);
      if (!rc && cudaEventRecord(c->ev_join, c->side) != cudaSuccess) rc = GP_ECUDA;
    }
  }
  c->marks = nullptr;
  return rc;
}

int read_status(gp_ctx *c, Status *h) {
  GP_CK(cudaMemcpyAsync(h, c->d_status, sizeof(Status), cudaMemcpyDeviceToHost, c->stream));
  GP_CK(cudaStreamSynchronize(c->stream));
  return GP_OK;
}

// Pair buffers with room for `pairs` candidate pairs (and as many colliding pairs, so
// that the colliding-pair buffer cannot fill during the contact solves): grown by at
// least a quarter, never shrunk.  Captured graphs hold the old buffers and are dropped.
int size_pairs(gp_ctx *c, int64_t pairs, int64_t coll) {
  const int64_t np = std::max(c->cap_pairs, pairs), nc = std::max(c->cap_coll, coll);
  if (np == c->cap_pairs && nc == c->cap_coll) return GP_OK;
  GP_CK(cudaStreamSynchronize(c->stream));
  GP_CK(cudaStreamSynchronize(c->side));
  drop_graph(c);
  if (np != c->cap_pairs) {
    dfree(c->d_pairs);
    c->cap_pairs = 0;
    GP_TRY(dalloc(&c->d_pairs, np));
    c->cap_pairs = np;
    try_qorder(c);
    if (c->d_cst) {                    // every candidate pair may be in contact
      dfree(c->d_cst);
      c->cap_cst = 0;
      GP_TRY(dalloc(&c->d_cst, (size_t)np));
      c->cap_cst = np;
    }
  }
  if (nc != c->cap_coll) {
    dfree(c->d_coll); dfree(c->d_state); dfree(c->d_acc);
    c->cap_coll = 0;
    GP_TRY(dalloc(&c->d_coll, nc));
    GP_TRY(dalloc(&c->d_state, nc));
    GP_TRY(dalloc(&c->d_acc, nc));
    c->cap_coll = nc;
  }
  return GP_OK;
}

// A step whose candidate pairs outgrew the buffers stopped after its advance (every
// later kernel saw the flag and returned; see Status).  This grows the buffers to the
// count that step reached, clears the flag (and the status code it set, unless another
// error came first) and runs that step's collision phase again; the loop ends once a
// collision phase fits.  *halted: whether h showed a halt.
int resume_after_halt(gp_ctx *c, Status h, bool *halted) {
  *halted = h.overflow != 0;
  for (int attempt = 0; h.overflow; ++attempt) {
    if (attempt >= 4) return GP_EPAIR_OVERFLOW;
    const int64_t need = (int64_t)h.pairs_needed;
    const int64_t grow = std::max<int64_t>(need + need / 4 + 1024, c->cap_pairs + c->cap_pairs / 4);
    GP_TRY(size_pairs(c, grow, grow));
    if (h.code == GP_EPAIR_OVERFLOW) { h.code = 0; h.first_id = 0; h.first_inst = 0; }
    h.overflow = 0;
    h.pairs_needed = 0;
    GP_CK(cudaMemcpyAsync(c->d_status, &h, sizeof(Status), cudaMemcpyHostToDevice, c->stream));
    GP_TRY(enqueue_collision(c));
    GP_TRY(read_status(c, &h));
  }
  return GP_OK;
}

}  // namespace

extern "C" {

int gp_ctx_create(const gp_params *params, gp_ctx **out) {
  if (!params || !out) return GP_EBADARG;
  *out = nullptr;
  const gp_params &p = *params;
  if (p.nx < 4 || p.ny < 4 || p.nz < 4) return GP_EBADARG;
  if (p.interp_scheme != 3) return GP_EBADARG;
  if (p.frozen_flow < 1 || p.frozen_flow > 3) return GP_EBADARG;   // a frozen field; 3 = channel
  if (p.precision != GP_PREC_FP64 && p.precision != GP_PREC_MIXED) return GP_EBADARG;
  if (!(p.lx > 0 && p.ly > 0 && p.lz > 0 && p.dtime > 0 && p.visc > 0)) return GP_EBADARG;
  gp_ctx *c = new gp_ctx();
  c->prm = p;
  c->ppi = 4.0 * std::atan(1.0);   // init_run.f90:123
  // the step's own stream gets the higher priority, so that the collision phase's
  // blocks are scheduled ahead of the overlapped gather
  int prio_low = 0, prio_high = 0;
  if (cudaGetDevice(&c->device) != cudaSuccess ||
      cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high) != cudaSuccess ||
      cudaStreamCreateWithPriority(&c->stream, cudaStreamNonBlocking, prio_high) != cudaSuccess ||
      cudaStreamCreateWithPriority(&c->side, cudaStreamNonBlocking, prio_low) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess) {
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return GP_ECUDA;
  }
  InstDev &I = c->tmpl;
  I.begin = 0;
  I.count = 0;
  I.nx = p.nx; I.ny = p.ny; I.nz = p.nz; I.ncomp = 6;
  I.fprec = p.precision;
  I.periodicity = p.periodicity ? 1 : 0;
  I.wall_boundary = p.wall_boundary ? 1 : 0;
  I.frozen_flow = p.frozen_flow;
  I.store_fluid = p.store_fluid ? 1 : 0;
  I.lx = p.lx; I.ly = p.ly; I.lz = p.lz;
  I.dx = p.lx / (double)(p.nx - 1);   // meshing.f90:43-45
  I.dy = p.ly / (double)(p.ny - 1);
  I.dz = p.lz / (double)(p.nz - 1);
  I.visc = p.visc; I.dtime = p.dtime; I.gravity = p.gravity;
  I.ecp = p.ecp; I.mup = p.mup; I.ecw = p.ecw; I.muw = p.muw;
  const size_t elem = (p.precision == GP_PREC_MIXED) ? sizeof(float) : sizeof(double);
  c->field_bytes = (size_t)(p.nx + 3) * (p.ny + 4) * (p.nz + 4) * kFieldStride * elem;
  int rc = GP_OK;
  if (cudaMalloc(&c->field, c->field_bytes) != cudaSuccess || cudaMemset(c->field, 0, c->field_bytes) != cudaSuccess)
    rc = GP_ENOMEM;
  I.field = c->field;
  c->fields.push_back({c->field, p.nx, p.ny, p.nz, p.lx, p.ly, p.lz});
  if (!rc) rc = dalloc(&c->d_inst, kMaxClasses);
  if (!rc) rc = dalloc(&c->d_pv, 1);
  if (!rc) rc = dalloc(&c->d_pv_alt, 1);
  if (!rc) rc = dalloc(&c->d_fluid_cols, kNFluid);
  if (!rc) rc = dalloc(&c->d_counters, kPassCounters + 2 * kMaxPasses);
  if (!rc && cudaMemset(c->d_counters, 0, (kPassCounters + 2 * kMaxPasses) * sizeof(unsigned long long)) !=
                 cudaSuccess)
    rc = GP_ECUDA;
  if (!rc) {
    // a full buffer only keeps the solve in its lane, so this bounds nothing else
    c->cap_tail = 65536;
    for (int k = 0; k < 2 && !rc; ++k)
      if (cudaMalloc(reinterpret_cast<void **>(&c->d_tail[k]), (size_t)c->cap_tail * tail_record_bytes()) !=
          cudaSuccess)
        rc = GP_ENOMEM;
  }
  if (!rc) rc = dalloc(&c->d_qbins, 2 * kQueueBins);
  if (!rc) rc = dalloc(&c->d_group_tab, kMaxClasses);
  if (!rc) rc = dalloc(&c->d_group_n, kMaxClasses);
  if (!rc) {
    std::vector<int32_t *> tab(kMaxClasses, nullptr);
    std::vector<int32_t> ng(kMaxClasses, 1);
    if (cudaMemcpy(c->d_group_tab, tab.data(), kMaxClasses * sizeof(int32_t *), cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMemcpy(c->d_group_n, ng.data(), kMaxClasses * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess)
      rc = GP_ECUDA;
  }
  if (!rc) rc = dalloc(&c->d_status, 1);
  if (!rc && cudaMemset(c->d_status, 0, sizeof(Status)) != cudaSuccess) rc = GP_ECUDA;
  if (!rc) rc = upload_inst(c);
  if (!rc && cudaStreamSynchronize(c->stream) != cudaSuccess) rc = GP_ECUDA;
  if (!rc) {
    const int cg = contact_grid_blocks();
    if (cg > 0) c->contact_grid = cg;
  }
  if (rc) {
    gp_ctx_destroy(c);
    return rc;
  }
  if (p.max_particles > 0) {
    rc = alloc_pool(c, p.max_particles);
    if (rc) { gp_ctx_destroy(c); return rc; }
  }
  *out = c;
  return GP_OK;
}

int gp_ctx_destroy(gp_ctx *c) {
  if (!c) return GP_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  drop_graph(c);
  free_pool(c);
  free_search(c);
  for (size_t f = 1; f < c->fields.size(); ++f) cudaFree(c->fields[f].ptr);
  if (c->field) cudaFree(c->field);
  dfree(c->stage); dfree(c->d_inst); dfree(c->d_pv); dfree(c->d_pv_alt); dfree(c->d_fluid_cols);
  dfree(c->d_counters);
  for (auto &g : c->group_dev) dfree(g);
  dfree(c->d_group_tab); dfree(c->d_group_n); dfree(c->d_cst); dfree(c->d_colacc);
  dfree(c->d_stat_partial); dfree(c->d_stat_out); dfree(c->d_qbins);
  for (TailRec *t : c->d_tail)
    if (t) cudaFree(t);
  dfree(c->d_status); dfree(c->d_scratch);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  for (auto &e : c->ev_host)
    if (e) cudaEventDestroy(e);
  if (c->side) cudaStreamDestroy(c->side);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return GP_OK;
}

int gp_status(gp_ctx *c, int32_t *code, int64_t *first_id) {
  if (!c) return GP_EBADARG;
  Status h;
  GP_TRY(read_status(c, &h));
  if (code) *code = h.code;
  if (first_id) *first_id = h.first_id;
  return GP_OK;
}

int gp_collision_counters(gp_ctx *c, int64_t *vals) {
  if (!c || !vals) return GP_EBADARG;
  Status h;
  GP_TRY(read_status(c, &h));
  unsigned long long cnt[4];
  GP_CK(cudaMemcpy(cnt, c->d_counters, sizeof(cnt), cudaMemcpyDeviceToHost));
  const unsigned long long v[GP_NCOUNTER] = {h.n_near, cnt[0], h.n_solve, h.n_contact, cnt[1], cnt[2],
                                             h.n_eval, h.max_eval};
  for (int k = 0; k < GP_NCOUNTER; ++k) vals[k] = (int64_t)v[k];
  return GP_OK;
}

int gp_status_class(gp_ctx *c, int32_t *ig) {
  if (!c || !ig) return GP_EBADARG;
  Status h;
  GP_TRY(read_status(c, &h));
  *ig = h.first_inst;
  return GP_OK;
}

int gp_clear_status(gp_ctx *c) {
  if (!c) return GP_EBADARG;
  GP_CK(cudaMemsetAsync(c->d_status, 0, sizeof(Status), c->stream));
  GP_CK(cudaStreamSynchronize(c->stream));
  return GP_OK;
}

int gp_sync(gp_ctx *c) {
  if (!c) return GP_EBADARG;
  GP_CK(cudaStreamSynchronize(c->stream));
  return GP_OK;
}

int gp_set_class(gp_ctx *c, int32_t ig, int32_t idp, double emaj, double apr, double rhop) {
  if (!c || !(emaj > 0) || !(apr > 0) || !(rhop > 0)) return GP_EBADARG;
  c->classes[{ig, idp}] = ClassProps{emaj, apr, rhop};
  return GP_OK;
}

int gp_set_field_slot(gp_ctx *c, int32_t field, int32_t comp, const double *src, int32_t src_layout,
                      int32_t ghost_mode, int32_t on_device) {
  if (!c || !src || comp < 0 || comp > 5 || field < 0 || field >= (int)c->fields.size()) return GP_EBADARG;
  if (src_layout != GP_LAYOUT_INTERIOR && src_layout != GP_LAYOUT_REFERENCE) return GP_EBADARG;
  if (ghost_mode != GP_GHOST_PERIODIC && ghost_mode != GP_GHOST_ZERO) return GP_EBADARG;
  const gp_ctx::FieldSlot &f = c->fields[field];
  const size_t count = (src_layout == GP_LAYOUT_REFERENCE) ? (size_t)f.nx * (f.ny + 4) * (f.nz + 4)
                                                           : (size_t)f.nx * f.ny * f.nz;
  const double *dsrc = src;
  if (!on_device) {
    if (c->stage_count < count) {
      dfree(c->stage);
      c->stage_count = 0;
      GP_TRY(dalloc(&c->stage, count));
      c->stage_count = count;
    }
    GP_CK(cudaMemcpyAsync(c->stage, src, count * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    dsrc = c->stage;
  }
  launch_field_layout(f.ptr, c->prm.precision, f.nx, f.ny, f.nz, kFieldStride, comp, dsrc, src_layout, ghost_mode,
                      c->stream);
  GP_CK(cudaGetLastError());
  GP_CK(cudaStreamSynchronize(c->stream));
  return GP_OK;
}

int gp_set_field(gp_ctx *c, int32_t comp, const double *src, int32_t src_layout, int32_t ghost_mode,
                 int32_t on_device) {
  return gp_set_field_slot(c, 0, comp, src, src_layout, ghost_mode, on_device);
}

int gp_add_field(gp_ctx *c, int32_t nx, int32_t ny, int32_t nz, double lx, double ly, double lz, int32_t *field) {
  if (!c || !field || nx < 4 || ny < 4 || nz < 4 || !(lx > 0 && ly > 0 && lz > 0)) return GP_EBADARG;
  const size_t elem = (c->prm.precision == GP_PREC_MIXED) ? sizeof(float) : sizeof(double);
  const size_t bytes = (size_t)(nx + 3) * (ny + 4) * (nz + 4) * kFieldStride * elem;
  void *ptr = nullptr;
  if (cudaMalloc(&ptr, bytes) != cudaSuccess) return GP_ENOMEM;
  if (cudaMemset(ptr, 0, bytes) != cudaSuccess) { cudaFree(ptr); return GP_ECUDA; }
  c->fields.push_back({ptr, nx, ny, nz, lx, ly, lz});
  *field = (int32_t)c->fields.size() - 1;
  return GP_OK;
}

int gp_field_shape(gp_ctx *c, int32_t field, int32_t dims[3]) {
  if (!c || !dims || field < 0 || field >= (int)c->fields.size()) return GP_EBADARG;
  dims[0] = c->fields[field].nx;
  dims[1] = c->fields[field].ny;
  dims[2] = c->fields[field].nz;
  return GP_OK;
}

}  // extern "C"

namespace {

// A class on field slot f: the context's physics with that field's mesh
// (meshing.f90:43-45).
InstDev class_template(const gp_ctx *c, int f) {
  InstDev I = c->tmpl;
  const gp_ctx::FieldSlot &F = c->fields[f];
  I.field = F.ptr;
  I.nx = F.nx; I.ny = F.ny; I.nz = F.nz;
  I.lx = F.lx; I.ly = F.ly; I.lz = F.lz;
  I.dx = F.lx / (double)(F.nx - 1);
  I.dy = F.ly / (double)(F.ny - 1);
  I.dz = F.lz / (double)(F.nz - 1);
  I.begin = 0;
  I.count = 0;
  return I;
}

// Host copy of the GP_NPROP property columns of n particles.
int read_props(gp_ctx *c, int64_t n, const double *const *props, int32_t on_device, std::vector<double> *hp) {
  for (int k = 0; k < GP_NPROP; ++k) {
    hp[k].resize(n);
    if (on_device) {
      GP_CK(cudaMemcpyAsync(hp[k].data(), props[k], n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    } else {
      std::memcpy(hp[k].data(), props[k], n * sizeof(double));
    }
  }
  GP_CK(cudaStreamSynchronize(c->stream));
  return GP_OK;
}

// Per-particle constants of particles [off, off+cnt) (reference expressions, IEEE
// double) into pcs (kNConst columns of leading dimension ld), and the class's grids.
int class_setup(gp_ctx *c, const std::vector<double> *hp, int64_t off, int64_t cnt, double *pcs, int64_t ld,
                InstDev &I) {
  double max_emaj = 0.0, rmax = 0.0;
  std::vector<double> radii(cnt);
  for (int64_t i = off; i < off + cnt; ++i) {
    double pc[kNConst];
    const double emaj = hp[0][i], apr = hp[1][i], rhop = hp[2][i];
    if (!(emaj > 0) || !(apr > 0) || !(rhop > 0)) return GP_EBADARG;
    part_const(emaj, apr, rhop, c->prm.rhof, c->ppi, hp[3][i], hp[4][i], hp[5][i], pc);
    for (int q = 0; q < kNConst; ++q) pcs[(size_t)q * ld + i] = pc[q];
    max_emaj = std::max(max_emaj, emaj);
    rmax = std::max(rmax, std::max(pc[0], pc[1]));
    radii[i - off] = std::max(pc[0], pc[1]);
  }
  // the search grid is sized for all but the largest 0.1% of bounding radii
  const int64_t qi = std::min<int64_t>(cnt - 1, (int64_t)(0.999 * (double)cnt));
  std::nth_element(radii.begin(), radii.begin() + qi, radii.end());
  I.count = cnt;
  return setup_grids(I, max_emaj, rmax, radii[qi], 0);
}

// After a change of the class table: caller-order offsets and search cells of the live
// classes, the device table, the captured graphs, and (rebin) a binning pass so that
// the next advance moves exactly the live particles.
void size_groups(gp_ctx *c, int slot) {
  if ((int)c->group_dev.size() <= slot) {
    c->group_dev.resize(slot + 1, nullptr);
    c->group_n.resize(slot + 1, 1);
  }
}

// Class slot `slot` goes back to one polydisperse index (all particles IDP = 1).
int clear_groups(gp_ctx *c, int slot) {
  size_groups(c, slot);
  if (!c->group_dev[slot] && c->group_n[slot] == 1) return GP_OK;
  GP_CK(cudaStreamSynchronize(c->stream));
  dfree(c->group_dev[slot]);
  c->group_dev[slot] = nullptr;
  c->group_n[slot] = 1;
  int32_t *null_ptr = nullptr;
  const int32_t one = 1;
  GP_CK(cudaMemcpy(c->d_group_tab + slot, &null_ptr, sizeof(int32_t *), cudaMemcpyHostToDevice));
  GP_CK(cudaMemcpy(c->d_group_n + slot, &one, sizeof(int32_t), cudaMemcpyHostToDevice));
  return GP_OK;
}

int refresh_classes(gp_ctx *c, bool rebin) {
  int64_t begin = 0, cells = 0;
  for (size_t k = 0; k < c->insts.size(); ++k) {
    InstDev &I = c->insts[k];
    if (!c->live[k]) I.count = 0;
    I.begin = begin;
    I.cell_begin = cells;
    begin += I.count;
    if (c->live[k]) cells += (int64_t)I.nfx * I.nfy * I.nfz;
  }
  drop_graph(c);
  c->n = begin;
  c->grid_ready = false;
  if (c->n == 0) {
    c->n_slots = 0;   // every particle left is retired
    return GP_OK;
  }
  GP_TRY(alloc_cells(c, cells));
  GP_TRY(upload_inst(c));
  c->grid_ready = true;
  if (rebin) GP_TRY(enqueue_bin(c));
  return GP_OK;
}

}  // namespace

extern "C" {

int gp_upload_classes(gp_ctx *c, int32_t nclass, const int64_t *counts, const double *const *cols,
                      const double *const *props, int32_t on_device) {
  if (!c || !cols || !props || !counts || nclass <= 0 || nclass > kMaxClasses) return GP_EBADARG;
  int64_t n = 0;
  for (int k = 0; k < nclass; ++k) {
    if (counts[k] <= 0 || counts[k] >= kMaxInstanceParticles) return GP_EBADARG;
    n += counts[k];
  }
  if (n >= (int64_t(1) << 31)) return GP_EBADARG;
  std::vector<double> hp[GP_NPROP];
  GP_TRY(read_props(c, n, props, on_device, hp));
  std::vector<double> pcs((size_t)kNConst * n);
  std::vector<InstDev> insts(nclass, class_template(c, 0));
  int64_t begin = 0;
  for (int k = 0; k < nclass; ++k) {
    GP_TRY(class_setup(c, hp, begin, counts[k], pcs.data(), n, insts[k]));
    begin += counts[k];
  }
  drop_graph(c);
  c->grid_ready = false;
  const int64_t want = std::max<int64_t>(n, c->prm.max_particles);
  if (c->cap < want) GP_TRY(alloc_pool(c, want));
  else
    for (int b = 0; b < 2; ++b) GP_CK(cudaMemsetAsync(c->d_instof[b], 0xFF, c->cap * sizeof(int32_t), c->stream));
  double *stage_cols = nullptr, *stage_pc = nullptr;
  GP_TRY(dalloc(&stage_cols, (size_t)kNState * n));
  GP_TRY(dalloc(&stage_pc, (size_t)kNConst * n));
  for (int k = 0; k < kNState; ++k) GP_TRY(copy_in(c, stage_cols + (size_t)k * n, cols[k], n, on_device));
  GP_CK(cudaMemcpyAsync(stage_pc, pcs.data(), pcs.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  begin = 0;
  for (int k = 0; k < nclass; ++k) {
    launch_init_pool(c->d_pv, begin, counts[k], k, stage_cols, stage_pc, n, begin, c->stream);
    begin += counts[k];
  }
  launch_iota(c->sa.sorted, n, c->stream);   // the first advance keeps the upload order
  GP_CK(cudaGetLastError());
  GP_CK(cudaStreamSynchronize(c->stream));
  cudaFree(stage_cols);
  cudaFree(stage_pc);
  c->insts = insts;
  c->live.assign(nclass, 1);
  c->class_field.assign(nclass, 0);
  c->n_slots = n;
  c->fluid_ok = false;
  for (int k = 0; k < nclass; ++k) GP_TRY(clear_groups(c, k));
  return refresh_classes(c, false);
}

int gp_add_class(gp_ctx *c, int32_t field, int64_t n, const double *const *cols, const double *const *props,
                 int32_t on_device, int32_t *ig) {
  if (!c || !cols || !props || !ig || n <= 0 || n >= kMaxInstanceParticles) return GP_EBADARG;
  if (field < 0 || field >= (int)c->fields.size()) return GP_EBADARG;
  if (c->cap == 0) GP_TRY(alloc_pool(c, std::max<int64_t>(n, c->prm.max_particles)));
  if (c->n_slots + n > c->cap) return GP_ENOMEM;
  size_t slot = 0;
  while (slot < c->live.size() && c->live[slot]) ++slot;
  if (slot >= (size_t)kMaxClasses) return GP_ENOMEM;
  std::vector<double> hp[GP_NPROP];
  GP_TRY(read_props(c, n, props, on_device, hp));
  std::vector<double> pcs((size_t)kNConst * n);
  InstDev I = class_template(c, field);
  GP_TRY(class_setup(c, hp, 0, n, pcs.data(), n, I));
  double *stage_cols = nullptr, *stage_pc = nullptr;
  GP_TRY(dalloc(&stage_cols, (size_t)kNState * n));
  GP_TRY(dalloc(&stage_pc, (size_t)kNConst * n));
  for (int k = 0; k < kNState; ++k) GP_TRY(copy_in(c, stage_cols + (size_t)k * n, cols[k], n, on_device));
  GP_CK(cudaMemcpyAsync(stage_pc, pcs.data(), pcs.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  launch_init_pool(c->d_pv, c->n_slots, n, (int)slot, stage_cols, stage_pc, n, 0, c->stream);
  GP_CK(cudaGetLastError());
  GP_CK(cudaStreamSynchronize(c->stream));
  cudaFree(stage_cols);
  cudaFree(stage_pc);
  c->n_slots += n;
  if (slot == c->live.size()) {
    c->insts.push_back(I);
    c->live.push_back(1);
    c->class_field.push_back(field);
  } else {
    c->insts[slot] = I;
    c->live[slot] = 1;
    c->class_field[slot] = field;
  }
  *ig = (int32_t)slot + 1;
  c->fluid_ok = false;
  GP_TRY(clear_groups(c, (int)slot));
  return refresh_classes(c, true);
}

int gp_download_class(gp_ctx *c, int32_t ig, double *const *cols, int32_t on_device) {
  if (!c || !cols || ig < 1 || ig > (int)c->live.size() || !c->live[ig - 1]) return GP_EBADARG;
  const int64_t n = c->insts[ig - 1].count;
  GP_TRY(ensure_scratch(c, (size_t)kNState * n));
  double *tmp = c->d_scratch;
  launch_gather_state(c->d_inst, c->d_pv, c->n_slots, ig - 1, tmp, c->d_fluid_cols, nullptr, n, c->stream);
  GP_CK(cudaGetLastError());
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  for (int k = 0; k < kNState; ++k)
    GP_CK(cudaMemcpyAsync(cols[k], tmp + (size_t)k * n, n * sizeof(double), kind, c->stream));
  GP_CK(cudaStreamSynchronize(c->stream));
  return GP_OK;
}

int gp_remove_class(gp_ctx *c, int32_t ig, double *const *cols, int32_t on_device) {
  if (!c || ig < 1 || ig > (int)c->live.size() || !c->live[ig - 1]) return GP_EBADARG;
  if (cols) GP_TRY(gp_download_class(c, ig, cols, on_device));
  launch_retire(c->d_pv, c->n_slots, ig - 1, c->stream);
  GP_CK(cudaGetLastError());
  c->live[ig - 1] = 0;
  GP_TRY(clear_groups(c, ig - 1));
  GP_TRY(refresh_classes(c, true));
  GP_CK(cudaStreamSynchronize(c->stream));
  return GP_OK;
}

int gp_class_count(gp_ctx *c, int32_t ig, int64_t *n) {
  if (!c || !n || ig < 1 || ig > (int)c->live.size()) return GP_EBADARG;
  *n = c->live[ig - 1] ? c->insts[ig - 1].count : 0;
  return GP_OK;
}

int gp_set_class_groups(gp_ctx *c, int32_t ig, int32_t ngroups, const int32_t *idp) {
  if (!c || ig < 1 || ig > (int)c->live.size() || !c->live[ig - 1]) return GP_EBADARG;
  if (ngroups < 1 || ngroups > kStatMaxGroups || (!idp && ngroups != 1)) return GP_EBADARG;
  const int slot = ig - 1;
  GP_TRY(clear_groups(c, slot));
  if (!idp) return GP_OK;
  const int64_t n = c->insts[slot].count;
  for (int64_t i = 0; i < n; ++i)
    if (idp[i] < 1 || idp[i] > ngroups) return GP_EBADARG;
  int32_t *d = nullptr;
  GP_TRY(dalloc(&d, n));
  if (cudaMemcpy(d, idp, n * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess) {
    dfree(d);
    return GP_ECUDA;
  }
  c->group_dev[slot] = d;
  c->group_n[slot] = ngroups;
  GP_CK(cudaMemcpy(c->d_group_tab + slot, &d, sizeof(int32_t *), cudaMemcpyHostToDevice));
  GP_CK(cudaMemcpy(c->d_group_n + slot, &ngroups, sizeof(int32_t), cudaMemcpyHostToDevice));
  return GP_OK;
}

int gp_stat_partfluid(gp_ctx *c, int32_t ig, double *out) {
  if (!c || !out || ig < 1 || ig > (int)c->live.size() || !c->live[ig - 1]) return GP_EBADARG;
  if (!c->fluid_ok) return GP_EBADARG;   // no step has sampled the fluid at these particles
  const int slot = ig - 1;
  size_groups(c, slot);
  const int ng = c->group_n[slot];
  constexpr int kBlocks = 148 * 3;
  if (!c->d_stat_partial) {
    GP_TRY(dalloc(&c->d_stat_partial, (size_t)kBlocks * kStatMaxGroups * kNStatPartfluid));
    GP_TRY(dalloc(&c->d_stat_out, (size_t)kStatMaxGroups * kNStatPartfluid));
  }
  launch_stat_partfluid(c->d_inst, c->d_pv, c->n_slots, slot, c->d_fluid_cols, c->group_dev[slot], ng,
                        c->prm.rhof, c->ppi, c->d_stat_partial, kBlocks, c->d_stat_out, c->d_status, c->stream);
  GP_CK(cudaGetLastError());
  GP_CK(cudaMemcpyAsync(out, c->d_stat_out, (size_t)ng * kNStatPartfluid * sizeof(double), cudaMemcpyDeviceToHost,
                        c->stream));
  GP_CK(cudaStreamSynchronize(c->stream));
  return GP_OK;
}

int gp_set_contact_tail(gp_ctx *c, int32_t budget) {
  if (!c || budget < 0 || budget > 300) return GP_EBADARG;
  c->tail_budget = budget;
  drop_graph(c);
  return GP_OK;
}

int gp_get_contact_tail(gp_ctx *c, int32_t *budget) {
  if (!c || !budget) return GP_EBADARG;
  *budget = c->tail_budget;
  return GP_OK;
}

int gp_set_contact_order(gp_ctx *c, int32_t on) {
  if (!c) return GP_EBADARG;
  if ((on != 0) == c->qorder_on) return GP_OK;
  GP_CK(cudaStreamSynchronize(c->stream));
  c->qorder_on = on != 0;
  drop_graph(c);
  if (c->qorder_on && c->d_evhist)   // no record carried over from before it was off
    GP_CK(cudaMemsetAsync(c->d_evhist, 0, (size_t)c->cap_evhist * sizeof(uint32_t), c->stream));
  return GP_OK;
}

int gp_get_contact_order(gp_ctx *c, int32_t *on) {
  if (!c || !on) return GP_EBADARG;
  *on = qorder_ready(c) ? 1 : 0;
  return GP_OK;
}

int gp_set_gather_staging(gp_ctx *c, int32_t mode) {
  if (!c || mode < 0 || mode > 1) return GP_EBADARG;
  if (mode == 1) {
    GP_TRY(ensure_field_map(c));
    GP_TRY(gather_tma_prepare());
  }
  c->gather_staging = mode;
  drop_graph(c);
  return GP_OK;
}

int gp_get_gather_staging(gp_ctx *c, int32_t *mode) {
  if (!c || !mode) return GP_EBADARG;
  const InstDev *f = nullptr;
  *mode = (c->gather_staging == 1 && c->prm.precision == GP_PREC_MIXED && single_field(c, &f)) ? 1 : 0;
  return GP_OK;
}

int gp_collision_stats_enable(gp_ctx *c, int32_t on) {
  if (!c) return GP_EBADARG;
  if ((on != 0) == c->colstats) return GP_OK;
  GP_CK(cudaStreamSynchronize(c->stream));
  if (on && (!c->d_colacc || c->cap_cst < c->cap_pairs)) {
    dfree(c->d_cst);
    c->cap_cst = 0;
    if (!c->d_colacc) {
      GP_TRY(dalloc(&c->d_colacc, (size_t)kMaxClasses * kStatMaxGroups * kStatMaxGroups * kNStatCollision));
      GP_CK(cudaMemset(c->d_colacc, 0,
                       (size_t)kMaxClasses * kStatMaxGroups * kStatMaxGroups * kNStatCollision * sizeof(double)));
    }
    // every candidate pair may be in contact
    GP_TRY(dalloc(&c->d_cst, (size_t)std::max<int64_t>(c->cap_pairs, 1)));
    c->cap_cst = std::max<int64_t>(c->cap_pairs, 1);
  }
  c->colstats = on != 0;
  drop_graph(c);
  return GP_OK;
}

int gp_collision_stats(gp_ctx *c, int32_t ig, double *out, int64_t *steps, int32_t reset) {
  if (!c || !out || ig < 1 || ig > (int)c->live.size()) return GP_EBADARG;
  const int slot = ig - 1;
  size_groups(c, slot);
  const int ng = c->group_n[slot];
  const size_t per_class = (size_t)kStatMaxGroups * kStatMaxGroups * kNStatCollision;
  std::vector<double> acc(per_class, 0.0);
  unsigned long long cnt[8] = {};
  GP_CK(cudaStreamSynchronize(c->stream));
  if (c->d_colacc)
    GP_CK(cudaMemcpy(acc.data(), c->d_colacc + (size_t)slot * per_class, per_class * sizeof(double),
                     cudaMemcpyDeviceToHost));
  GP_CK(cudaMemcpy(cnt, c->d_counters, sizeof(cnt), cudaMemcpyDeviceToHost));
  const double dtime = c->insts.empty() ? c->tmpl.dtime : c->insts[slot].dtime;
  for (int g1 = 0; g1 < ng; ++g1)
    for (int g2 = 0; g2 < ng; ++g2) {
      const double *a = acc.data() + ((size_t)g1 * kStatMaxGroups + g2) * kNStatCollision;
      double *o = out + ((size_t)g1 * ng + g2) * kNStatCollision;
      for (int k = 0; k < kNStatCollision; ++k) o[k] = a[k];
      o[2] = 2.0 * o[1] / dtime;   // collision_interaction.f90:429
      o[4] = o[3] / o[0];          // collision_interaction.f90:430
    }
  if (steps) *steps = (int64_t)cnt[7];
  if (reset) {
    if (c->d_colacc)
      GP_CK(cudaMemsetAsync(c->d_colacc, 0, (size_t)kMaxClasses * per_class * sizeof(double), c->stream));
    GP_CK(cudaMemsetAsync(c->d_counters + 7, 0, sizeof(unsigned long long), c->stream));
    GP_CK(cudaStreamSynchronize(c->stream));
  }
  return GP_OK;
}

int gp_upload_state(gp_ctx *c, int64_t n, const double *const *cols, const double *const *props, int32_t on_device) {
  return gp_upload_classes(c, 1, &n, cols, props, on_device);
}

int gp_download_state(gp_ctx *c, int64_t n, double *const *cols, double *const *fluid, int32_t on_device) {
  if (!c || !cols || n != c->n) return GP_EBADARG;
  if (fluid && !c->prm.store_fluid) return GP_EBADARG;
  // the context's scratch buffer, kept between calls: a fresh allocation and its
  // release (which waits for the device) would cost more than the gather itself
  const size_t per = (size_t)kNState + (fluid ? kNFluid : 0);
  GP_TRY(ensure_scratch(c, per * n));
  double *tmp = c->d_scratch;
  launch_gather_state(c->d_inst, c->d_pv, c->n_slots, -1, tmp, c->d_fluid_cols,
                      fluid ? tmp + (size_t)kNState * n : nullptr, n,
                      c->stream);
  GP_CK(cudaGetLastError());
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  for (int k = 0; k < kNState; ++k)
    GP_CK(cudaMemcpyAsync(cols[k], tmp + (size_t)k * n, n * sizeof(double), kind, c->stream));
  if (fluid)
    for (int k = 0; k < kNFluid; ++k)
      GP_CK(cudaMemcpyAsync(fluid[k], tmp + (size_t)(kNState + k) * n, n * sizeof(double), kind, c->stream));
  GP_CK(cudaStreamSynchronize(c->stream));
  return GP_OK;
}

int gp_put_state(gp_ctx *c, int64_t n, const double *const *cols, int32_t on_device) {
  if (!c || !cols || n != c->n) return GP_EBADARG;
  GP_TRY(ensure_scratch(c, (size_t)kNState * n));
  for (int k = 0; k < kNState; ++k) GP_TRY(copy_in(c, c->d_scratch + (size_t)k * n, cols[k], n, on_device));
  launch_scatter_state(c->d_inst, c->d_pv, c->n_slots, c->d_scratch, n, c->stream);
  GP_CK(cudaGetLastError());
  GP_CK(cudaStreamSynchronize(c->stream));
  c->fluid_ok = false;
  return GP_OK;
}

// One step of an ensemble held in host arrays: put the state, one step (ADV_PARTICLE_ELLP
// + COLLISION, as gp_step(ctx, 1)), download it, with the copies overlapped with the
// step where the data allow.  The gather reads only positions, so it starts once those
// three columns are in; positions and quaternions are final after the integrate (the
// response changes velocities and spins only), so they go out while the collision phase
// runs.  The kernels and their order are those of put, step and download, so the
// results are identical.  in_cols and out_cols may be the same arrays: every column is
// in before any goes out.
int gp_step_host(gp_ctx *c, int64_t n, const double *const *in_cols, double *const *out_cols) {
  if (!c || !in_cols || !out_cols || n <= 0 || n != c->n || !c->grid_ready) return GP_EBADARG;
  for (int k = 0; k < kNState; ++k)
    if (!in_cols[k] || !out_cols[k]) return GP_EBADARG;
  GP_TRY(ensure_scratch(c, (size_t)kNState * n));
  for (auto &e : c->ev_host)
    if (!e) GP_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  double *tmp = c->d_scratch;
  const size_t bytes = (size_t)n * sizeof(double);
  cudaEvent_t *ev = c->ev_host;
  // the copies wait for whatever the stream still does with the scratch buffer
  GP_CK(cudaEventRecord(ev[0], c->stream));
  GP_CK(cudaStreamWaitEvent(c->side, ev[0], 0));
  for (int k = 0; k < kNState; ++k) {
    GP_CK(cudaMemcpyAsync(tmp + (size_t)k * n, in_cols[k], bytes, cudaMemcpyHostToDevice, c->side));
    if (k == 2) GP_CK(cudaEventRecord(ev[1], c->side));   // x, y, z are in
  }
  GP_CK(cudaEventRecord(ev[2], c->side));                 // every column is in
  GP_CK(cudaStreamWaitEvent(c->stream, ev[1], 0));
  launch_scatter_state(c->d_inst, c->d_pv, c->n_slots, tmp, n, c->stream, kColsPos);
  GP_CK(cudaGetLastError());
  GP_TRY(enqueue_gather(c, c->stream));
  GP_CK(cudaStreamWaitEvent(c->stream, ev[2], 0));
  launch_scatter_state(c->d_inst, c->d_pv, c->n_slots, tmp, n, c->stream, kAllStateCols & ~kColsPos);
  GP_CK(cudaGetLastError());
  GP_TRY(enqueue_integrate(c));
  launch_gather_state(c->d_inst, c->d_pv, c->n_slots, -1, tmp, c->d_fluid_cols, nullptr, n, c->stream,
                      kColsPosQuat);
  GP_CK(cudaGetLastError());
  GP_CK(cudaEventRecord(ev[3], c->stream));
  GP_TRY(enqueue_collision(c));
  launch_gather_state(c->d_inst, c->d_pv, c->n_slots, -1, tmp, c->d_fluid_cols, nullptr, n, c->stream,
                      kColsVelSpin);
  GP_CK(cudaGetLastError());
  GP_CK(cudaEventRecord(ev[4], c->stream));
  GP_CK(cudaStreamWaitEvent(c->side, ev[3], 0));
  for (int k = 0; k < kNState; ++k)
    if ((kColsPosQuat >> k) & 1u)
      GP_CK(cudaMemcpyAsync(out_cols[k], tmp + (size_t)k * n, bytes, cudaMemcpyDeviceToHost, c->side));
  GP_CK(cudaStreamWaitEvent(c->side, ev[4], 0));
  for (int k = 0; k < kNState; ++k)
    if ((kColsVelSpin >> k) & 1u)
      GP_CK(cudaMemcpyAsync(out_cols[k], tmp + (size_t)k * n, bytes, cudaMemcpyDeviceToHost, c->side));
  GP_CK(cudaStreamSynchronize(c->side));
  // a collision phase halted by a pair-buffer overflow sent pre-collision velocities:
  // it runs again with larger buffers and its velocities and spins go out again
  Status h;
  bool halted = false;
  GP_TRY(read_status(c, &h));
  GP_TRY(resume_after_halt(c, h, &halted));
  if (halted) {
    launch_gather_state(c->d_inst, c->d_pv, c->n_slots, -1, tmp, c->d_fluid_cols, nullptr, n, c->stream,
                        kColsVelSpin);
    GP_CK(cudaGetLastError());
    for (int k = 0; k < kNState; ++k)
      if ((kColsVelSpin >> k) & 1u)
        GP_CK(cudaMemcpyAsync(out_cols[k], tmp + (size_t)k * n, bytes, cudaMemcpyDeviceToHost, c->stream));
    GP_CK(cudaStreamSynchronize(c->stream));
  }
  return GP_OK;
}

int gp_adv_particle_ellp(gp_ctx *c, int32_t /*ncycle*/) {
  if (!c || c->n <= 0) return GP_EBADARG;
  return enqueue_advance(c);
}

int gp_collision(gp_ctx *c, int32_t /*ncycle*/, double /*time*/, int64_t *n_near, int64_t *n_contact,
                 int64_t *n_coll) {
  if (!c || c->n <= 0 || !c->grid_ready) return GP_EBADARG;
  GP_CK(cudaMemsetAsync(&c->d_status->n_near, 0, 8 * sizeof(unsigned long long), c->stream));
  GP_TRY(enqueue_collision(c));
  Status h;
  GP_TRY(read_status(c, &h));
  bool halted = false;
  GP_TRY(resume_after_halt(c, h, &halted));
  if (n_near || n_contact || n_coll) {
    GP_TRY(read_status(c, &h));
    unsigned long long cnt[4];
    GP_CK(cudaMemcpy(cnt, c->d_counters, sizeof(cnt), cudaMemcpyDeviceToHost));
    if (n_near) *n_near = (int64_t)h.n_near;
    if (n_contact) *n_contact = (int64_t)h.n_contact;
    if (n_coll) *n_coll = (int64_t)cnt[1];
  }
  return GP_OK;
}

// Captures nsteps steps into one graph (the caller ends the capture).
int capture_steps(gp_ctx *c, int nsteps, cudaEvent_t *marks, cudaGraph_t *g) {
  GP_CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  int rc = GP_OK;
  if (marks && cudaEventRecordWithFlags(marks[0], c->stream, cudaEventRecordExternal) != cudaSuccess) rc = GP_ECUDA;
  if (!rc) rc = enqueue_steps(c, nsteps, marks ? marks + 1 : nullptr);
  if (!rc && marks &&
      cudaEventRecordWithFlags(marks[1 + (size_t)nsteps * 2 * GP_NPHASE], c->stream, cudaEventRecordExternal) !=
          cudaSuccess)
    rc = GP_ECUDA;
  const cudaError_t e = cudaStreamEndCapture(c->stream, g);
  if (!rc && e != cudaSuccess) rc = GP_ECUDA;
  if (rc && e == cudaSuccess) cudaGraphDestroy(*g);
  return rc;
}

// Replays `nsteps` steps from the graph cache (one graph per step count in use; the
// cache is bounded).
int replay_steps(gp_ctx *c, int nsteps) {
  auto it = c->graphs.find(nsteps);
  if (it == c->graphs.end()) {
    if (c->graphs.size() >= 8) drop_graph(c);
    cudaGraph_t g;
    GP_TRY(capture_steps(c, nsteps, nullptr, &g));
    cudaGraphExec_t ge = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return GP_ECUDA;
    it = c->graphs.emplace(nsteps, ge).first;
  }
  GP_CK(cudaGraphLaunch(it->second, c->stream));
  c->fluid_ok = true;   // a replay samples the fluid as the capture did
  return GP_OK;
}

int gp_step(gp_ctx *c, int32_t nsteps) {
  if (!c || c->n <= 0 || !c->grid_ready || nsteps < 0) return GP_EBADARG;
  // Steps halted by a pair-buffer overflow: the halted step is finished with larger
  // buffers (resume_after_halt) and the steps after it are replayed.
  int remaining = nsteps;
  for (int attempt = 0; remaining > 0; ++attempt) {
    if (attempt > 32) return GP_EPAIR_OVERFLOW;
    GP_CK(cudaMemsetAsync(&c->d_status->steps_done, 0, sizeof(unsigned long long), c->stream));
    GP_TRY(replay_steps(c, remaining));
    Status h;
    GP_TRY(read_status(c, &h));
    bool halted = false;
    const int64_t done = (int64_t)h.steps_done;
    GP_TRY(resume_after_halt(c, h, &halted));
    if (!halted) break;
    remaining -= (int)done + 1;
  }
  return GP_OK;
}

int gp_step_timed(gp_ctx *c, int32_t nsteps, float *total_ms, float *phase_ms_avg, int32_t *kernels_per_step) {
  if (!c || c->n <= 0 || !c->grid_ready || nsteps <= 0) return GP_EBADARG;
  // [0] start, then 2*GP_NPHASE per step (begin/end of each phase), then the end
  std::vector<cudaEvent_t> ev(2 + (size_t)nsteps * 2 * GP_NPHASE);
  for (auto &e : ev) GP_CK(cudaEventCreate(&e));
  cudaGraph_t g;
  cudaGraphExec_t ge = nullptr;
  int rc = capture_steps(c, nsteps, ev.data(), &g);
  if (!rc && kernels_per_step) {
    size_t nn = 0;
    cudaGraphGetNodes(g, nullptr, &nn);
    std::vector<cudaGraphNode_t> nodes(nn);
    cudaGraphGetNodes(g, nodes.data(), &nn);
    int nk = 0;
    for (auto nd : nodes) {
      cudaGraphNodeType t;
      if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++nk;
    }
    *kernels_per_step = nk / nsteps;
  }
  if (!rc) {
    if (cudaGraphInstantiate(&ge, g, 0) != cudaSuccess) rc = GP_ECUDA;
    cudaGraphDestroy(g);
  }
  if (!rc && cudaGraphLaunch(ge, c->stream) != cudaSuccess) rc = GP_ECUDA;
  if (!rc && cudaStreamSynchronize(c->stream) != cudaSuccess) rc = GP_ECUDA;
  if (!rc) {
    // a graph halted by a pair-buffer overflow timed a short step; its halted step is
    // finished with larger buffers and the whole measurement is taken again
    Status h;
    bool halted = false;
    rc = read_status(c, &h);
    if (!rc) rc = resume_after_halt(c, h, &halted);
    if (!rc && halted) {
      if (ge) cudaGraphExecDestroy(ge);
      for (auto &x : ev) cudaEventDestroy(x);
      return gp_step_timed(c, nsteps, total_ms, phase_ms_avg, kernels_per_step);
    }
  }
  if (!rc) {
    double acc[GP_NPHASE] = {};
    float t = 0.f;
    for (int s = 0; s < nsteps && !rc; ++s)
      for (int p = 0; p < GP_NPHASE && !rc; ++p) {
        const size_t k = 1 + ((size_t)s * GP_NPHASE + p) * 2;
        if (cudaEventElapsedTime(&t, ev[k], ev[k + 1]) != cudaSuccess) rc = GP_ECUDA;
        acc[p] += t;
      }
    if (!rc && cudaEventElapsedTime(&t, ev[0], ev.back()) != cudaSuccess) rc = GP_ECUDA;
    if (!rc && total_ms) *total_ms = t;
    if (!rc && phase_ms_avg)
      for (int p = 0; p < GP_NPHASE; ++p) phase_ms_avg[p] = (float)(acc[p] / nsteps);
  }
  if (ge) cudaGraphExecDestroy(ge);
  for (auto &x : ev) cudaEventDestroy(x);
  return rc;
}

int gp_collision_pairs(gp_ctx *c, int64_t cap, int32_t *home, int32_t *near, int64_t *count) {
  if (!c) return GP_EBADARG;
  unsigned long long cnt[4];
  GP_CK(cudaStreamSynchronize(c->stream));
  GP_CK(cudaMemcpy(cnt, c->d_counters, sizeof(cnt), cudaMemcpyDeviceToHost));
  const int64_t nc = (int64_t)std::min<unsigned long long>(cnt[1], (unsigned long long)c->cap_coll);
  std::vector<CollRec> recs(nc);
  std::vector<int8_t> st(nc);
  if (nc > 0) {
    GP_CK(cudaMemcpy(recs.data(), c->d_coll, nc * sizeof(CollRec), cudaMemcpyDeviceToHost));
    GP_CK(cudaMemcpy(st.data(), c->d_state, nc, cudaMemcpyDeviceToHost));
  }
  // class by class, each in the reference's list order
  std::vector<std::pair<std::array<unsigned long long, 3>, int64_t>> acc;
  for (int64_t e = 0; e < nc; ++e)
    if (st[e] == 1) acc.push_back({{(unsigned long long)recs[e].inst, recs[e].k1, recs[e].k2}, e});
  std::sort(acc.begin(), acc.end());
  if (count) *count = (int64_t)acc.size();
  for (int64_t k = 0; k < (int64_t)acc.size() && k < cap; ++k) {
    const unsigned long long k2 = acc[k].first[2];
    const int64_t base = c->insts[acc[k].first[0]].begin;
    if (home) home[k] = (int32_t)(base + (int64_t)(k2 >> 34));
    if (near) near[k] = (int32_t)(base + (int64_t)(k2 & ((1ull << 30) - 1)));
  }
  return GP_OK;
}

int gp_collision_box_connectivity(gp_ctx *c, int32_t *nbox, int32_t *ncon, int32_t *con, int32_t *grid_dims,
                                  double *grid_geom) {
  if (!c || !c->grid_ready) return GP_EBADARG;
  const InstDev &I = c->insts[0];   // the first class's grid
  const int64_t nb = (int64_t)I.nxbox * I.nybox * I.nzbox;
  if (nbox) *nbox = (int32_t)nb;
  if (grid_dims) { grid_dims[0] = I.nxbox; grid_dims[1] = I.nybox; grid_dims[2] = I.nzbox; }
  if (grid_geom) {
    grid_geom[0] = I.dxbox; grid_geom[1] = I.dybox; grid_geom[2] = I.dzbox;
    grid_geom[3] = I.xminbox; grid_geom[4] = I.yminbox; grid_geom[5] = I.zminbox;
  }
  if (!ncon && !con) return GP_OK;
  int32_t *dn = nullptr, *dc = nullptr;
  GP_TRY(dalloc(&dn, nb));
  GP_TRY(dalloc(&dc, nb * 27));
  launch_connectivity(I.nxbox, I.nybox, I.nzbox, I.periodicity, dn, dc, c->stream);
  GP_CK(cudaGetLastError());
  if (ncon) GP_CK(cudaMemcpyAsync(ncon, dn, nb * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  if (con) GP_CK(cudaMemcpyAsync(con, dc, nb * 27 * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  GP_CK(cudaStreamSynchronize(c->stream));
  cudaFree(dn);
  cudaFree(dc);
  return GP_OK;
}

// ---------------------------------------------------------------- drop-ins ----
int gp_interp_lag3(gp_ctx *c, int32_t comp, int64_t nint, const double *xint, const double *yint, const double *zint,
                   double *uint, int32_t on_device) {
  if (!c || comp < 0 || comp > 5 || nint < 0) return GP_EBADARG;
  if (nint == 0) return GP_OK;
  const double *dx = xint, *dy = yint, *dz = zint;
  double *dout = uint;
  if (!on_device) {
    GP_TRY(ensure_scratch(c, 4 * (size_t)nint));
    double *s = c->d_scratch;
    GP_TRY(copy_in(c, s, xint, nint, 0));
    GP_TRY(copy_in(c, s + nint, yint, nint, 0));
    GP_TRY(copy_in(c, s + 2 * nint, zint, nint, 0));
    dx = s; dy = s + nint; dz = s + 2 * nint; dout = s + 3 * nint;
  }
  launch_interp(c->d_inst, comp, nint, dx, dy, dz, dout, c->d_status, c->stream);
  GP_CK(cudaGetLastError());
  if (!on_device) GP_CK(cudaMemcpyAsync(uint, dout, nint * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  GP_CK(cudaStreamSynchronize(c->stream));
  return GP_OK;
}

int gp_frozen_interp_lag3(gp_ctx *c, const double *xain, const double *yain, const double *zain, int32_t nx,
                          int32_t ny, int32_t nz, const double *uain, int64_t nint, const double *xint,
                          const double *yint, const double *zint, double *uint) {
  if (!c || nx < 3 || ny < 3 || nz < 3 || nint < 0) return GP_EBADARG;
  if (nint == 0) return GP_OK;
  const size_t nf = (size_t)nx * ny * nz;
  GP_TRY(ensure_scratch(c, (size_t)nx + ny + nz + nf + 4 * (size_t)nint));
  double *s = c->d_scratch;
  double *dxa = s, *dya = dxa + nx, *dza = dya + ny, *du = dza + nz, *dxi = du + nf, *dyi = dxi + nint,
         *dzi = dyi + nint, *dout = dzi + nint;
  GP_TRY(copy_in(c, dxa, xain, nx, 0));
  GP_TRY(copy_in(c, dya, yain, ny, 0));
  GP_TRY(copy_in(c, dza, zain, nz, 0));
  GP_TRY(copy_in(c, du, uain, nf, 0));
  GP_TRY(copy_in(c, dxi, xint, nint, 0));
  GP_TRY(copy_in(c, dyi, yint, nint, 0));
  GP_TRY(copy_in(c, dzi, zint, nint, 0));
  launch_frozen_interp(dxa, dya, dza, nx, ny, nz, du, nint, dxi, dyi, dzi, dout, c->d_status, c->stream);
  GP_CK(cudaGetLastError());
  GP_CK(cudaMemcpyAsync(uint, dout, nint * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  GP_CK(cudaStreamSynchronize(c->stream));
  return GP_OK;
}

int gp_fluid_force_ellipsoid_batch(gp_ctx *c, int64_t n, const int32_t *ig, const int32_t *idp, const double *up,
                                   const double *uf, const double *quat, double *fdrag, double *flift,
                                   int32_t on_device) {
  if (!c || n < 0 || !ig || !idp) return GP_EBADARG;
  if (n == 0) return GP_OK;
  std::vector<int32_t> hig(n), hidp(n);
  if (on_device) {
    GP_CK(cudaMemcpy(hig.data(), ig, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
    GP_CK(cudaMemcpy(hidp.data(), idp, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
  } else {
    std::memcpy(hig.data(), ig, n * sizeof(int32_t));
    std::memcpy(hidp.data(), idp, n * sizeof(int32_t));
  }
  std::vector<double> pcs((size_t)kNConst * n);
  for (int64_t i = 0; i < n; ++i) GP_TRY(class_props(c, hig[i], hidp[i], &pcs[(size_t)kNConst * i]));
  GP_TRY(ensure_scratch(c, (size_t)n * (kNConst + 3 + 3 + 4 + 3 + 3)));
  double *dpc = c->d_scratch, *dup = dpc + kNConst * n, *duf = dup + 3 * n, *dq = duf + 3 * n, *dfd = dq + 4 * n,
         *dfl = dfd + 3 * n;
  GP_CK(cudaMemcpyAsync(dpc, pcs.data(), pcs.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  GP_TRY(copy_in(c, dup, up, 3 * n, on_device));
  GP_TRY(copy_in(c, duf, uf, 3 * n, on_device));
  GP_TRY(copy_in(c, dq, quat, 4 * n, on_device));
  launch_force_batch(n, dpc, c->prm.visc, dup, duf, dq, dfd, dfl, c->d_status, c->stream);
  GP_CK(cudaGetLastError());
  const cudaMemcpyKind k = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  GP_CK(cudaMemcpyAsync(fdrag, dfd, 3 * n * sizeof(double), k, c->stream));
  GP_CK(cudaMemcpyAsync(flift, dfl, 3 * n * sizeof(double), k, c->stream));
  GP_CK(cudaStreamSynchronize(c->stream));
  return GP_OK;
}

int gp_fluid_force_ellipsoid(gp_ctx *c, int32_t ig, int32_t idp, double upart, double vpart, double wpart,
                             double ufluid, double vfluid, double wfluid, const double quat[4], double fdrag[3],
                             double flift[3]) {
  const double up[3] = {upart, vpart, wpart}, uf[3] = {ufluid, vfluid, wfluid};
  return gp_fluid_force_ellipsoid_batch(c, 1, &ig, &idp, up, uf, quat, fdrag, flift, 0);
}

int gp_fluid_torque_ellipsoid_batch(gp_ctx *c, int64_t n, const int32_t *ig, const int32_t *idp, const double *omega,
                                    const double *quat, const double *part_up, const double *part_ufap,
                                    const double *part_vort, double *tpitch, double *trot, int32_t on_device) {
  if (!c || n < 0 || !ig || !idp) return GP_EBADARG;
  if (n == 0) return GP_OK;
  std::vector<int32_t> hig(n), hidp(n);
  if (on_device) {
    GP_CK(cudaMemcpy(hig.data(), ig, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
    GP_CK(cudaMemcpy(hidp.data(), idp, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
  } else {
    std::memcpy(hig.data(), ig, n * sizeof(int32_t));
    std::memcpy(hidp.data(), idp, n * sizeof(int32_t));
  }
  std::vector<double> pcs((size_t)kNConst * n);
  for (int64_t i = 0; i < n; ++i) GP_TRY(class_props(c, hig[i], hidp[i], &pcs[(size_t)kNConst * i]));
  GP_TRY(ensure_scratch(c, (size_t)n * (kNConst + 3 + 4 + 3 + 3 + 3 + 3 + 3)));
  double *dpc = c->d_scratch, *dom = dpc + kNConst * n, *dq = dom + 3 * n, *dup = dq + 4 * n, *duf = dup + 3 * n,
         *dvo = duf + 3 * n, *dtp = dvo + 3 * n, *dtr = dtp + 3 * n;
  GP_CK(cudaMemcpyAsync(dpc, pcs.data(), pcs.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  GP_TRY(copy_in(c, dom, omega, 3 * n, on_device));
  GP_TRY(copy_in(c, dq, quat, 4 * n, on_device));
  GP_TRY(copy_in(c, dup, part_up, 3 * n, on_device));
  GP_TRY(copy_in(c, duf, part_ufap, 3 * n, on_device));
  GP_TRY(copy_in(c, dvo, part_vort, 3 * n, on_device));
  launch_torque_batch(n, dpc, c->prm.visc, dom, dq, dup, duf, dvo, dtp, dtr, c->d_status, c->stream);
  GP_CK(cudaGetLastError());
  const cudaMemcpyKind k = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  GP_CK(cudaMemcpyAsync(tpitch, dtp, 3 * n * sizeof(double), k, c->stream));
  GP_CK(cudaMemcpyAsync(trot, dtr, 3 * n * sizeof(double), k, c->stream));
  GP_CK(cudaStreamSynchronize(c->stream));
  return GP_OK;
}

int gp_fluid_torque_ellipsoid(gp_ctx *c, int32_t ig, int32_t idp, double ox, double oy, double oz,
                              const double quat[4], const double part_up[3], const double part_ufap[3],
                              const double part_vort[3], double tpitch[3], double trot[3]) {
  const double om[3] = {ox, oy, oz};
  return gp_fluid_torque_ellipsoid_batch(c, 1, &ig, &idp, om, quat, part_up, part_ufap, part_vort, tpitch, trot, 0);
}

int gp_quaternion_integration_batch(gp_ctx *c, int64_t n, double *quat, const double *omega, double dt,
                                    int32_t on_device) {
  if (!c || n < 0) return GP_EBADARG;
  if (n == 0) return GP_OK;
  GP_TRY(ensure_scratch(c, (size_t)7 * n));
  double *dq = c->d_scratch, *dom = dq + 4 * n;
  GP_TRY(copy_in(c, dq, quat, 4 * n, on_device));
  GP_TRY(copy_in(c, dom, omega, 3 * n, on_device));
  launch_quat_batch(n, dq, dom, dt, c->stream);
  GP_CK(cudaGetLastError());
  GP_CK(cudaMemcpyAsync(quat, dq, 4 * n * sizeof(double), on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                        c->stream));
  GP_CK(cudaStreamSynchronize(c->stream));
  return GP_OK;
}

int gp_quaternion_integration(gp_ctx *c, double quat[4], double omgx, double omgy, double omgz, double dt) {
  const double om[3] = {omgx, omgy, omgz};
  return gp_quaternion_integration_batch(c, 1, quat, om, dt, 0);
}

int gp_euler_integration(gp_ctx *c, int32_t ig, int32_t idp, double *omgx, double *omgy, double *omgz) {
  if (!c || !omgx || !omgy || !omgz) return GP_EBADARG;
  double pc[kNConst];
  GP_TRY(class_props(c, ig, idp, pc));
  GP_TRY(ensure_scratch(c, 6));
  const double h[6] = {pc[7], pc[8], pc[9], *omgx, *omgy, *omgz};
  GP_CK(cudaMemcpyAsync(c->d_scratch, h, sizeof(h), cudaMemcpyHostToDevice, c->stream));
  launch_euler_batch(1, c->d_scratch, c->prm.dtime, c->d_scratch + 3, c->stream);
  GP_CK(cudaGetLastError());
  double o[3];
  GP_CK(cudaMemcpyAsync(o, c->d_scratch + 3, sizeof(o), cudaMemcpyDeviceToHost, c->stream));
  GP_CK(cudaStreamSynchronize(c->stream));
  *omgx = o[0]; *omgy = o[1]; *omgz = o[2];
  return GP_OK;
}

int gp_ellipsoid_contact_detection_batch(gp_ctx *c, int64_t n, const double *shapes, const double *centres,
                                         const double *quats, int32_t *flag, double *ept1, double *ept2,
                                         double *cnormal, int32_t on_device) {
  if (!c || n < 0) return GP_EBADARG;
  if (n == 0) return GP_OK;
  // shapes come in as (emaj1, apr1, emaj2, apr2); the kernel takes semi-axes (a, a/apr)
  std::vector<double> hs(4 * (size_t)n);
  if (on_device) GP_CK(cudaMemcpy(hs.data(), shapes, hs.size() * sizeof(double), cudaMemcpyDeviceToHost));
  else std::memcpy(hs.data(), shapes, hs.size() * sizeof(double));
  for (int64_t i = 0; i < n; ++i) {
    hs[4 * i + 1] = hs[4 * i] / hs[4 * i + 1];
    hs[4 * i + 3] = hs[4 * i + 2] / hs[4 * i + 3];
  }
  GP_TRY(ensure_scratch(c, (size_t)n * (4 + 6 + 8 + 9) + (size_t)n));
  double *ds = c->d_scratch, *dc = ds + 4 * n, *dq = dc + 6 * n, *de1 = dq + 8 * n, *de2 = de1 + 3 * n,
         *dcn = de2 + 3 * n;
  int32_t *dflag = reinterpret_cast<int32_t *>(dcn + 3 * n);
  GP_CK(cudaMemcpyAsync(ds, hs.data(), hs.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  GP_TRY(copy_in(c, dc, centres, 6 * n, on_device));
  GP_TRY(copy_in(c, dq, quats, 8 * n, on_device));
  launch_contact_batch(n, ds, dc, dq, dflag, de1, de2, dcn, c->stream);
  GP_CK(cudaGetLastError());
  const cudaMemcpyKind k = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  GP_CK(cudaMemcpyAsync(flag, dflag, n * sizeof(int32_t), k, c->stream));
  GP_CK(cudaMemcpyAsync(ept1, de1, 3 * n * sizeof(double), k, c->stream));
  GP_CK(cudaMemcpyAsync(ept2, de2, 3 * n * sizeof(double), k, c->stream));
  GP_CK(cudaMemcpyAsync(cnormal, dcn, 3 * n * sizeof(double), k, c->stream));
  GP_CK(cudaStreamSynchronize(c->stream));
  return GP_OK;
}

int gp_ellipsoid_contact_detection(gp_ctx *c, int32_t ig, int32_t idp1, int32_t idp2, double ixp, double iyp,
                                   double izp, const double iquat[4], double jxp, double jyp, double jzp,
                                   const double jquat[4], int32_t *flag, double ept1[3], double ept2[3],
                                   double cnormal[3]) {
  if (!c) return GP_EBADARG;
  auto a = c->classes.find({ig, idp1}), b = c->classes.find({ig, idp2});
  if (a == c->classes.end() || b == c->classes.end()) return GP_EBADARG;
  const double shapes[4] = {a->second.emaj, a->second.apr, b->second.emaj, b->second.apr};
  const double centres[6] = {ixp, iyp, izp, jxp, jyp, jzp};
  const double quats[8] = {iquat[0], iquat[1], iquat[2], iquat[3], jquat[0], jquat[1], jquat[2], jquat[3]};
  return gp_ellipsoid_contact_detection_batch(c, 1, shapes, centres, quats, flag, ept1, ept2, cnormal, 0);
}

int gp_collision_response(gp_ctx *c, int32_t ig, int32_t idp, double part1[10], double part2[10],
                          const double r_impact1[3], const double r_impact2[3], const double normal[3]) {
  if (!c || !part1 || !part2) return GP_EBADARG;
  double pc[kNConst];
  GP_TRY(class_props(c, ig, idp, pc));
  GP_TRY(ensure_scratch(c, 3 + 10 + 10 + 9));
  double h[32];
  h[0] = pc[7]; h[1] = pc[8]; h[2] = pc[9];
  std::memcpy(h + 3, part1, 10 * sizeof(double));
  std::memcpy(h + 13, part2, 10 * sizeof(double));
  std::memcpy(h + 23, r_impact1, 3 * sizeof(double));
  std::memcpy(h + 26, r_impact2, 3 * sizeof(double));
  std::memcpy(h + 29, normal, 3 * sizeof(double));
  double *d = c->d_scratch;
  GP_CK(cudaMemcpyAsync(d, h, sizeof(h), cudaMemcpyHostToDevice, c->stream));
  GP_CK(cudaMemsetAsync(c->d_status, 0, sizeof(Status), c->stream));
  launch_response_batch(1, c->prm.ecp, c->prm.mup, d, d + 3, d + 13, d + 23, d + 26, d + 29, c->d_status, c->stream);
  GP_CK(cudaGetLastError());
  GP_CK(cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  Status s;
  GP_TRY(read_status(c, &s));
  std::memcpy(part1, h + 3, 10 * sizeof(double));
  std::memcpy(part2, h + 13, 10 * sizeof(double));
  return s.code;
}

// Serving loop.  Jobs arrive at their times (seconds after the call starts, wall clock);
// in arrival order, each is admitted as soon as its footprint fits the HBM budget
// beside the running jobs and its particles fit the pool; every loop iteration steps
// all running jobs together (one advance and one collision phase for all of them) and
// retires the jobs that have run their steps, writing their final state back.  A job
// whose particle raises an error is retired at once with that status; the others go on.
int gp_serve(gp_ctx *c, gp_job *jobs, int32_t njobs, double hbm_budget, double bytes_per_particle,
             int64_t *particle_steps) {
  if (!c || (!jobs && njobs > 0) || njobs < 0 || !(bytes_per_particle > 0)) return GP_EBADARG;
  using clock = std::chrono::steady_clock;
  const auto t0 = clock::now();
  auto now = [&] { return std::chrono::duration<double>(clock::now() - t0).count(); };
  std::vector<int> order(njobs);
  for (int j = 0; j < njobs; ++j) {
    order[j] = j;
    jobs[j].admitted_s = jobs[j].done_s = -1.0;
    jobs[j].status = GP_OK;
    if (jobs[j].n <= 0 || jobs[j].steps < 0 || !jobs[j].cols || !jobs[j].props) return GP_EBADARG;
  }
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return jobs[a].arrival_s < jobs[b].arrival_s; });
  std::vector<int> ig_of(njobs, 0), left(njobs, 0);
  std::vector<int> running;
  size_t next = 0;
  double used = 0.0;
  int64_t done_work = 0;
  int rc = GP_OK;
  auto retire = [&](int j, int status) -> int {
    int r = gp_remove_class(c, ig_of[j], jobs[j].cols, 0);
    jobs[j].done_s = now();
    jobs[j].status = status;
    used -= (double)jobs[j].n * bytes_per_particle;
    running.erase(std::find(running.begin(), running.end(), j));
    return r;
  };
  while (!rc && (next < order.size() || !running.empty())) {
    // admission, first come first served
    while (next < order.size()) {
      gp_job &J = jobs[order[next]];
      if (J.arrival_s > now()) break;
      const double need = (double)J.n * bytes_per_particle;
      if ((c->cap > 0 && J.n > c->cap) || (need > hbm_budget)) {   // can never run here
        J.admitted_s = J.done_s = now();
        J.status = GP_ENOMEM;
        ++next;
        continue;
      }
      if (used + need > hbm_budget) break;
      if (c->cap > 0 && c->n_slots + J.n > c->cap) break;   // room after the next compaction
      int32_t ig = 0;
      rc = gp_add_class(c, J.field, J.n, J.cols, J.props, 0, &ig);
      if (rc) break;
      ig_of[order[next]] = ig;
      left[order[next]] = J.steps;
      J.admitted_s = now();
      used += need;
      running.push_back(order[next]);
      ++next;
    }
    if (rc) break;
    // jobs with no steps to run leave at once
    for (size_t k = 0; k < running.size() && !rc;) {
      const int j = running[k];
      if (left[j] == 0) rc = retire(j, GP_OK); else ++k;
    }
    if (rc) break;
    if (running.empty()) {
      if (next < order.size()) {
        const double wait = jobs[order[next]].arrival_s - now();
        if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 0.01)));
      }
      continue;
    }
    // one step of every running job
    GP_CK(cudaMemsetAsync(&c->d_status->n_near, 0, 8 * sizeof(unsigned long long), c->stream));
    rc = enqueue_advance(c);
    if (!rc) rc = enqueue_collision(c);
    if (rc) break;
    Status h;
    rc = read_status(c, &h);
    if (rc) break;
    if (h.overflow) {
      bool halted = false;
      rc = resume_after_halt(c, h, &halted);
      if (!rc) rc = read_status(c, &h);
      if (rc) break;
    }
    for (int j : running) {
      --left[j];
      done_work += jobs[j].n;
    }
    if (h.code) {
      const int bad_ig = h.first_inst;
      int bad = -1;
      for (int j : running)
        if (ig_of[j] == bad_ig) bad = j;
      if (bad < 0) { rc = h.code; break; }   // not attributable to one job
      rc = retire(bad, h.code);
      if (!rc) rc = gp_clear_status(c);
    }
    for (size_t k = 0; k < running.size() && !rc;) {
      const int j = running[k];
      if (left[j] <= 0) rc = retire(j, GP_OK); else ++k;
    }
  }
  if (particle_steps) *particle_steps = done_work;
  return rc;
}

int gp_set_pair_capacity(gp_ctx *c, int64_t cap_pairs, int64_t cap_coll) {
  if (!c || cap_pairs < 1 || cap_coll < 1 || !c->d_pairs) return GP_EBADARG;
  GP_CK(cudaStreamSynchronize(c->stream));
  GP_CK(cudaStreamSynchronize(c->side));
  // drop to one slot first so that size_pairs reallocates at exactly these sizes
  drop_graph(c);
  dfree(c->d_pairs); dfree(c->d_coll); dfree(c->d_state); dfree(c->d_acc);
  c->cap_pairs = c->cap_coll = 0;
  GP_TRY(dalloc(&c->d_pairs, cap_pairs));
  c->cap_pairs = cap_pairs;
  GP_TRY(dalloc(&c->d_coll, cap_coll));
  GP_TRY(dalloc(&c->d_state, cap_coll));
  GP_TRY(dalloc(&c->d_acc, cap_coll));
  c->cap_coll = cap_coll;
  if (c->d_cst) {
    dfree(c->d_cst);
    c->cap_cst = 0;
    GP_TRY(dalloc(&c->d_cst, (size_t)cap_pairs));
    c->cap_cst = cap_pairs;
  }
  return GP_OK;
}

int gp_pair_capacity(gp_ctx *c, int64_t *cap_pairs, int64_t *cap_coll) {
  if (!c) return GP_EBADARG;
  if (cap_pairs) *cap_pairs = c->cap_pairs;
  if (cap_coll) *cap_coll = c->cap_coll;
  return GP_OK;
}

int gp_set_launch(gp_ctx *c, const int32_t *grids) {
  if (!c || !grids) return GP_EBADARG;
  for (int t = 0; t < GP_NTUNE; ++t)
    if (grids[t] < 1 || grids[t] > 148 * 64) return GP_EBADARG;
  if (grids[GP_NTUNE] < 0 || grids[GP_NTUNE] > 2) return GP_EBADARG;
  if (grids[GP_NTUNE] == 2 && !try_mark(c)) return GP_ENOMEM;
  for (int t = 0; t < GP_NTUNE; ++t) c->tune[t] = grids[t];
  c->overlap = grids[GP_NTUNE] != 0;
  c->spec = grids[GP_NTUNE] == 2;
  drop_graph(c);
  return GP_OK;
}

// Coordinate descent over the launch grids: each tunable in turn, each candidate timed
// by one-step graphs on the live ensemble (median of three), the fastest kept.  The
// state is saved before and restored after, so the ensemble does not move; the pool
// order and the last binning may change, which no result depends on.
int gp_autotune(gp_ctx *c, int32_t *grids_out) {
  if (!c || c->n <= 0 || !c->grid_ready) return GP_EBADARG;
  const int64_t n = c->n;
  double *save = nullptr;
  GP_TRY(dalloc(&save, (size_t)kNState * n));
  const bool colstats = c->colstats;   // the trials add nothing to the statistics
  c->colstats = false;
  launch_gather_state(c->d_inst, c->d_pv, c->n_slots, -1, save, c->d_fluid_cols, nullptr, n, c->stream);
  GP_CK(cudaGetLastError());
  static const int kMult[] = {1, 2, 4, 8, 16};
  static const int kPhase[GP_NTUNE] = {GP_PHASE_GATHER, GP_PHASE_INTEGRATE, GP_PHASE_BIN, GP_PHASE_SEARCH};
  int rc = GP_OK;
  for (int t = 0; t < GP_NTUNE && !rc; ++t) {
    int best = c->tune[t];
    float best_ms = 1e30f;
    for (int m : kMult) {
      c->tune[t] = 148 * m;
      drop_graph(c);
      float ph[GP_NPHASE], trial[3];
      for (int r = 0; r < 3 && !rc; ++r) {
        rc = gp_step_timed(c, 1, nullptr, ph, nullptr);
        trial[r] = ph[kPhase[t]];
      }
      if (rc) break;
      std::sort(trial, trial + 3);
      if (trial[1] < best_ms) { best_ms = trial[1]; best = c->tune[t]; }
    }
    c->tune[t] = best;
  }
  // The mixed gather's staging (stencil rows through L1, or each stencil box staged by
  // the TMA), by the gather's one-step time, where the classes read one field.
  if (!rc && c->prm.precision == GP_PREC_MIXED && ensure_field_map(c) == GP_OK && gather_tma_prepare() == GP_OK) {
    int best = c->gather_staging;
    float best_ms = 1e30f;
    for (int m = 0; m < 2 && !rc; ++m) {
      c->gather_staging = m;
      drop_graph(c);
      float ph[GP_NPHASE], trial[3];
      for (int r = 0; r < 3 && !rc; ++r) {
        rc = gp_step_timed(c, 1, nullptr, ph, nullptr);
        trial[r] = ph[GP_PHASE_GATHER];
      }
      if (rc) break;
      std::sort(trial, trial + 3);
      if (trial[1] < best_ms) { best_ms = trial[1]; best = m; }
    }
    c->gather_staging = best;
  }
  cudaGetLastError();
  // Overlapped gather (and speculative integrate) or not, timed as eight-step graphs
  // (median of three), closer to the steady state than shorter graphs.  Overlapped work
  // only gets the SMs the contact solves leave, so it is also tried with the gather at
  // the widest grid, whatever the one-step trials chose.
  const bool can_spec = !rc && try_mark(c);
  if (!rc) {
    const int tuned = c->tune[GP_TUNE_GATHER];
    const int gath[5] = {tuned, tuned, 148 * 16, tuned, 148 * 16};
    const bool over[5] = {false, true, true, true, true};
    const bool spec[5] = {false, false, false, true, true};
    float best = 1e30f;
    int pick = 0;
    for (int k = 0; k < 5 && !rc; ++k) {
      if ((k == 2 || k == 4) && tuned == 148 * 16) continue;
      if (spec[k] && !can_spec) continue;
      c->overlap = over[k];
      c->spec = spec[k];
      c->tune[GP_TUNE_GATHER] = gath[k];
      drop_graph(c);
      float trial[3];
      for (int r = 0; r < 3 && !rc; ++r) rc = gp_step_timed(c, 8, &trial[r], nullptr, nullptr);
      std::sort(trial, trial + 3);
      if (trial[1] < best) { best = trial[1]; pick = k; }
    }
    c->overlap = over[pick];
    c->spec = spec[pick];
    c->tune[GP_TUNE_GATHER] = gath[pick];
  }
  drop_graph(c);
  if (!rc) {
    launch_scatter_state(c->d_inst, c->d_pv, c->n_slots, save, n, c->stream);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(c->stream) != cudaSuccess) rc = GP_ECUDA;
  }
  cudaFree(save);
  c->colstats = colstats;
  c->fluid_ok = false;
  if (!rc && grids_out) {
    for (int t = 0; t < GP_NTUNE; ++t) grids_out[t] = c->tune[t];
    grids_out[GP_NTUNE] = c->overlap ? (c->spec ? 2 : 1) : 0;
  }
  return rc;
}

}  // extern "C"
