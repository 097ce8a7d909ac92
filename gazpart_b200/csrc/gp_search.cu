// gp_search.cu -- binning, neighbour search, greedy matching and the data-movement
// kernels of the collision step.
#include <cooperative_groups.h>

#include "gp_types.h"
#include "gp_launch.h"

namespace cg = cooperative_groups;

namespace gp {

// COLLISION on the device (collision.f90:7-200 with NPROC=1).
//
// The reference lists candidate pairs box by box (collision_detection_connectivity.f90:
// 145-207): for each box IJK, for each particle NP1 of the box in ascending index,
// first the later particles of the same box, then every particle of the 13 forward
// neighbour boxes COLBOX(IJK)%CON(1..NCON) in order.  It then walks that list and lets
// a pair collide only if neither particle has collided yet this step
// (collision_interaction.f90:190-419).
//
// Device formulation (same result):
//  1. particles are binned into a search grid whose cell edge is at least twice the
//     largest bounding radius max(EMAJ, EMAJ/APR); a pair can only be in contact if
//     its bounding spheres overlap (each contact point must lie inside the other body,
//     ellipsoid_contact_detection.f90:125), so a half-stencil sweep over that grid
//     finds every pair that could collide;
//  2. for each such pair the reference's box ids decide whether the reference lists it
//     at all and in which orientation, and give its position in the reference list as
//     the key (IJK of HOME, index of HOME, stencil slot, index of NEAR);
//  3. contacts and NVREL are evaluated for all of them on the pre-collision state (a
//     pair is only ever evaluated while both its particles are unmodified);
//  4. the lexicographically-first maximal matching of the colliding pairs under that key
//     -- which is what the sequential COLOR walk produces -- is computed in parallel
//     rounds (a pair is accepted when it holds the smallest key at both endpoints);
//  5. COLLISION_RESPONSE is applied to the accepted pairs (disjoint, so race free).

// Canonical slot of the 13 forward neighbour offsets in COLBOX order
// (collision_box_connectivity.f90:127-312: boxes 9,12,15,17,18,20,21,22,23,24,25,26,27),
// indexed by (dI+1)*9 + (dJ+1)*3 + (dK+1); 0 = not a forward offset.
__constant__ int8_t c_fwd_slot[27] = {
    // dI = -1: (dJ,dK) = (-1,-1) (-1,0) (-1,1) (0,-1) (0,0) (0,1) (1,-1) (1,0) (1,1)
    0, 0, 0, 0, 0, 8, 0, 0, 11,
    // dI = 0
    0, 0, 6, 0, 0, 9, 0, 4, 12,
    // dI = +1
    0, 2, 7, 0, 3, 10, 1, 5, 13};

__device__ __forceinline__ int wrap_delta(int d, int n, bool periodic) {
  if (periodic) {
    if (d == n - 1) return -1;
    if (d == -(n - 1)) return 1;
  }
  return d;
}


// ---------------------------------------------------------------------------
// 1. search-grid cell of every particle (counting pass)
// ---------------------------------------------------------------------------
__device__ __forceinline__ int cell_coord(double v, double h, int n) {
  const double f = v / h;
  int c = (f >= 0.0) ? (f < (double)n ? (int)f : n - 1) : 0;
  return c;
}

__global__ void k_bin_count(const InstDev *__restrict__ insts, const PoolView *__restrict__ pv, int64_t n,
                            SearchArrays sa, const Status *st) {
  if (step_halted(st)) return;
  const PoolView P = *pv;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t nround = (n + stride - 1) / stride * stride;   // whole warps stay in the loop
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nround; i += stride) {
    int32_t c = -1;
    if (i < n) {
      const int inst = P.inst[i];
      if (inst >= 0) {
        const InstDev &I = insts[inst];
        const int cx = cell_coord(P.st[0][i], I.hfx, I.nfx);
        const int cy = cell_coord(P.st[1][i], I.hfy, I.nfy);
        const int cz = cell_coord(P.st[2][i], I.hfz, I.nfz);
        c = (int32_t)(I.cell_begin + ((int64_t)cz * I.nfy + cy) * I.nfx + cx);
      }
      sa.cell_of[i] = c;
    }
    // particles are kept in cell order, so neighbouring lanes usually share a cell:
    // one atomic per cell per warp
    const unsigned peers = __match_any_sync(0xffffffffu, c);
    const int leader = __ffs(peers) - 1;
    if (c >= 0 && (int)(threadIdx.x & 31) == leader) atomicAdd(&sa.cell_count[c], __popc(peers));
  }
}

void launch_bin_count(const InstDev *insts, const PoolView *pv, int64_t n, SearchArrays sa, Status *st,
                      int grid, cudaStream_t s) {
  k_bin_count<<<grid, 256, 0, s>>>(insts, pv, n, sa, st);
}

// ---------------------------------------------------------------------------
// 2. exclusive scan (three-level, 2048 elements per block)
// ---------------------------------------------------------------------------
constexpr int kScanThreads = 512, kScanPer = 4, kScanBlock = kScanThreads * kScanPer;

__global__ void k_scan_block(const int32_t *__restrict__ in, int32_t *__restrict__ out, int64_t n,
                             int32_t *__restrict__ sums) {
  __shared__ int32_t warp_tot[kScanThreads / 32];
  const int64_t base = (int64_t)blockIdx.x * kScanBlock + (int64_t)threadIdx.x * kScanPer;
  int32_t v[kScanPer];
  int32_t run = 0;
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    const int64_t idx = base + k;
    v[k] = (idx < n) ? in[idx] : 0;
    const int32_t t = v[k];
    v[k] = run;
    run += t;
  }
  // inclusive warp scan of per-thread totals
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int32_t x = run;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int32_t w = (lane < kScanThreads / 32) ? warp_tot[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kScanThreads / 32) warp_tot[lane] = w;
  }
  __syncthreads();
  const int32_t excl = x - run + (wid > 0 ? warp_tot[wid - 1] : 0);
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    const int64_t idx = base + k;
    if (idx < n) out[idx] = v[k] + excl;
  }
  if (threadIdx.x == kScanThreads - 1 && sums != nullptr) sums[blockIdx.x] = excl + run;
}

__global__ void k_scan_add(int32_t *__restrict__ out, int64_t n, const int32_t *__restrict__ offs) {
  const int64_t base = (int64_t)blockIdx.x * kScanBlock;
  const int32_t o = offs[blockIdx.x];
  for (int k = threadIdx.x; k < kScanBlock; k += blockDim.x) {
    const int64_t idx = base + k;
    if (idx < n) out[idx] += o;
  }
}

static int64_t nblocks(int64_t n) { return (n + kScanBlock - 1) / kScanBlock; }

int64_t scan_block_sums_size(int64_t n) {
  // level-1 sums, level-2 sums (and their scans)
  const int64_t b1 = nblocks(n + 1), b2 = nblocks(b1), b3 = nblocks(b2);
  return 2 * (b1 + b2 + b3) + 16;
}

// out[0..n] = exclusive scan of in[0..n-1], out[n] = total.  in[n] must be readable
// as zero (the caller allocates n+1 counters).
void launch_scan(const int32_t *in, int32_t *out, int64_t n, int32_t *tmp, cudaStream_t s) {
  const int64_t m = n + 1;
  const int64_t b1 = nblocks(m), b2 = nblocks(b1), b3 = nblocks(b2);
  int32_t *s1 = tmp, *s1x = s1 + b1, *s2 = s1x + b1, *s2x = s2 + b2, *s3 = s2x + b2;
  k_scan_block<<<(unsigned)b1, kScanThreads, 0, s>>>(in, out, m, s1);
  if (b1 > 1) {
    k_scan_block<<<(unsigned)b2, kScanThreads, 0, s>>>(s1, s1x, b1, s2);
    if (b2 > 1) {
      k_scan_block<<<(unsigned)b3, kScanThreads, 0, s>>>(s2, s2x, b2, s3);   // b3 == 1 for n < 8.6e9
      k_scan_add<<<(unsigned)b2, kScanThreads, 0, s>>>(s1x, b1, s2x);
    }
    k_scan_add<<<(unsigned)b1, kScanThreads, 0, s>>>(out, m, s1x);
  }
}

// ---------------------------------------------------------------------------
// 3. scatter into cell order + reference box ids (collision_detection_connectivity.f90:74-89)
// ---------------------------------------------------------------------------
__global__ void k_bin_scatter(const InstDev *__restrict__ insts, const PoolView *__restrict__ pv, int64_t n,
                              SearchArrays sa, Status *st) {
  if (step_halted(st)) return;
  const PoolView P = *pv;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t nround = (n + stride - 1) / stride * stride;
  const int lane = threadIdx.x & 31;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nround; i += stride) {
    const int32_t c = (i < n) ? sa.cell_of[i] : -1;
    const unsigned peers = __match_any_sync(0xffffffffu, c);
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (c >= 0 && lane == leader) base = atomicAdd(&sa.cell_fill[c], __popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (c < 0) continue;
    const int pos = sa.cell_start[c] + base + __popc(peers & ((1u << lane) - 1u));
    const int inst = P.inst[i];
    const InstDev &I = insts[inst];
    const double x = P.st[0][i], y = P.st[1][i], z = P.st[2][i];
    sa.sorted[pos] = (int32_t)i;
    sa.sx[pos] = x;
    sa.sy[pos] = y;
    sa.sz[pos] = z;
    const double ea = P.pc[0][i], eb = P.pc[1][i];
    sa.sr[pos] = fmax(ea, eb);
    // w carries the bounding radius, negated for particles above the small-particle cut
    const double rb = fmax(ea, eb);
    sa.spk[pos] = make_float4((float)x, (float)y, (float)z, rb > I.rcut ? -(float)rb : (float)rb);
    // a float rounded up bounds the radius; non-negative floats order like their bits
    if (rb <= I.rcut) atomicMax(reinterpret_cast<int *>(sa.cell_rmax) + c, __float_as_int(__double2float_ru(rb)));
    sa.sa2[pos] = ea * ea;
    sa.sb2[pos] = eb * eb;
    {
      const double q0 = P.st[6][i], q1 = P.st[7][i], q2 = P.st[8][i], q3 = P.st[9][i];
      sa.sex[pos] = 1.0 - 2.0 * (q2 * q2 + q3 * q3);
      sa.sey[pos] = 2.0 * (q1 * q2 + q0 * q3);
      sa.sez[pos] = 2.0 * (q1 * q3 - q0 * q2);
    }
    sa.sinst[pos] = inst;
    sa.sid[pos] = P.id[i];
    const double fx = (x - I.xminbox) / I.dxbox, fy = (y - I.yminbox) / I.dybox, fz = (z - I.zminbox) / I.dzbox;
    long long box = -1;
    if (fx > -1.0 && fx < 2.0e9 && fy > -1.0 && fy < 2.0e9 && fz > -1.0 && fz < 2.0e9) {
      const int i0 = (int)fx + 1, j0 = (int)fy + 1, k0 = (int)fz + 1;
      if (i0 >= 1 && i0 <= I.nxbox && j0 >= 1 && j0 <= I.nybox && k0 >= 1 && k0 <= I.nzbox)
        box = (long long)(i0 - 1) | ((long long)(j0 - 1) << 21) | ((long long)(k0 - 1) << 42);
    }
    if (box < 0) set_error(st, GP_EOUT_OF_GRID, (long long)P.id[i], P.inst[i]);
    sa.sbox[pos] = box;
  }
}

void launch_bin_scatter(const InstDev *insts, const PoolView *pv, int64_t n, SearchArrays sa, Status *st, int grid,
                        cudaStream_t s) {
  k_bin_scatter<<<grid, 256, 0, s>>>(insts, pv, n, sa, st);
}

// ---------------------------------------------------------------------------
// 4. half-stencil sweep of the search grid, reference adjacency and order key
// ---------------------------------------------------------------------------
// mark (non-null when the next step's integrate runs speculatively): both particles of
// a stored pair are flagged, since the response may change their velocities.
__device__ __forceinline__ void emit_pair(PairRec *pairs, unsigned long long *npairs, int64_t cap, const PairRec &r,
                                          uint32_t *mark, Status *st) {
  cg::coalesced_group g = cg::coalesced_threads();
  unsigned long long base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(npairs, (unsigned long long)g.size());
  base = g.shfl(base, 0);
  const unsigned long long slot = base + g.thread_rank();
  if ((int64_t)slot < cap) {
    pairs[slot] = r;
    if (mark != nullptr) {
      mark[r.home] = 1u;
      mark[r.near] = 1u;
    }
  } else {
    atomicAdd(&st->overflow, 1ull);
    atomicMax(&st->pairs_needed, slot + 1ull);
    set_error(st, GP_EPAIR_OVERFLOW, (long long)r.home);
  }
}

// A home particle as the conservative float test of its candidates reads it: position,
// bounding radius, its instance's box lengths and x periodicity (32 bytes).
struct HomeF {
  float x, y, z, r, lx, ly, lz;
  int perx;
};

__device__ __forceinline__ HomeF home_f(const InstDev &I, double x, double y, double z, double r) {
  return {(float)x, (float)y, (float)z, (float)r, (float)I.lx, (float)I.ly, (float)I.lz, I.periodicity != 0};
}

// The conservative float test of candidate qs (sorted position) against a home at sorted
// position s: |float - double| distance error < 2e-6, slack 1e-5.  Nearly every
// candidate of the sweep fails it, so it reads only the candidate's float record.
// kLarge: the home particle is above the cut and sweeps a full stencil; it takes every
// small candidate and the large ones that follow it in sorted order.  Otherwise the home
// particle is small, sweeps the half stencil and leaves large candidates to them.
template <bool kLarge>
__device__ __forceinline__ bool near_float(const float4 c, int32_t qs, int32_t s, const HomeF &h) {
  if (c.w < 0.f && (!kLarge || qs <= s)) return false;
  float fx = c.x - h.x, fy = c.y - h.y, fz = c.z - h.z;
  if (h.perx && fabsf(fx) > 0.5f * h.lx) fx = fx - copysignf(h.lx, fx);
  if (fabsf(fy) > 0.5f * h.ly) fy = fy - copysignf(h.ly, fy);
  if (fabsf(fz) > 0.5f * h.lz) fz = fz - copysignf(h.lz, fz);
  const float rf = h.r + fabsf(c.w) + 1.0e-5f;
  return fx * fx + fy * fy + fz * fz <= rf * rf;
}

// One candidate (s, qs) of the sweep that passed near_float: FP64 bounding-sphere test,
// centre-line separation test, reference box adjacency, then emission with the
// reference's ordering keys.
struct SearchHome {
  double xp, yp, zp, rp;
  long long bp;
  int32_t s, pslot, idp;
  bool perx;
};

__device__ __forceinline__ void search_candidate(const InstDev &I, const SearchArrays &sa, const SearchHome &h,
                                                 int32_t qs, PairRec *pairs, unsigned long long *npairs,
                                                 int64_t cap, Status *st) {
  double dx = sa.sx[qs] - h.xp, dy = sa.sy[qs] - h.yp, dz = sa.sz[qs] - h.zp;
  if (h.perx && fabs(dx) > I.lx / 2) dx = dx - copysign(I.lx, dx);
  if (fabs(dy) > I.ly / 2.) dy = dy - copysign(I.ly, dy);
  if (fabs(dz) > I.lz / 2.) dz = dz - copysign(I.lz, dz);
  const double rr = (h.rp + sa.sr[qs]) * (1.0 + 1e-9);
  const double d2 = dx * dx + dy * dy + dz * dz;
  if (d2 > rr * rr) return;
  // Support-function test along the centre line: for unit d, the extent of a
  // spheroid is h(d) = sqrt(b^2 + (a^2-b^2)(e.d)^2).  If h_p + h_q < |d| the two
  // bodies are disjoint, so no contact point can lie inside the other body
  // (ellipsoid_contact_detection.f90:125) and the reference cannot flag the pair.
  if (d2 > 0.0) {
    const double dist = sqrt(d2), inv = 1.0 / dist;
    const double ux = dx * inv, uy = dy * inv, uz = dz * inv;
    const double cp = sa.sex[h.s] * ux + sa.sey[h.s] * uy + sa.sez[h.s] * uz;
    const double cq = sa.sex[qs] * ux + sa.sey[qs] * uy + sa.sez[qs] * uz;
    const double hp = sqrt(fmax(sa.sb2[h.s] + (sa.sa2[h.s] - sa.sb2[h.s]) * cp * cp, 0.0));
    const double hq = sqrt(fmax(sa.sb2[qs] + (sa.sa2[qs] - sa.sb2[qs]) * cq * cq, 0.0));
    if (hp + hq < dist * (1.0 - 1e-9)) return;
  }
  atomicAdd(&st->n_near, 1ull);
  // reference adjacency of the two boxes (collision_box_connectivity.f90)
  const long long bp = h.bp, bq = sa.sbox[qs];
  if (bp < 0 || bq < 0) return;   // already reported as out of grid
  const int pi = (int)(bp & 0x1FFFFF), pj = (int)((bp >> 21) & 0x1FFFFF), pk = (int)(bp >> 42);
  const int qi = (int)(bq & 0x1FFFFF), qj = (int)((bq >> 21) & 0x1FFFFF), qk = (int)(bq >> 42);
  const int di = wrap_delta(qi - pi, I.nxbox, h.perx);
  const int dj = wrap_delta(qj - pj, I.nybox, true);
  const int dk = wrap_delta(qk - pk, I.nzbox, true);
  if (di < -1 || di > 1 || dj < -1 || dj > 1 || dk < -1 || dk > 1) return;
  const int32_t idq = sa.sid[qs];
  PairRec r;
  int slot;
  long long hb;
  bool home_is_p;
  if (di == 0 && dj == 0 && dk == 0) {
    slot = 0;
    home_is_p = h.idp < idq;
    hb = bp;
  } else {
    const int idx = (di + 1) * 9 + (dj + 1) * 3 + (dk + 1);
    slot = c_fwd_slot[idx];
    if (slot > 0) {
      home_is_p = true;
      hb = bp;
    } else {
      slot = c_fwd_slot[26 - idx];
      home_is_p = false;
      hb = bq;
    }
  }
  const int hi = (int)(hb & 0x1FFFFF), hj = (int)((hb >> 21) & 0x1FFFFF), hk = (int)(hb >> 42);
  const unsigned long long ijk =
      (unsigned long long)(hi + 1) + (unsigned long long)hj * I.nxbox + (unsigned long long)hk * I.nxbox * I.nybox;
  const int32_t idh = home_is_p ? h.idp : idq, idn = home_is_p ? idq : h.idp;
  r.home = home_is_p ? h.pslot : sa.sorted[qs];
  r.near = home_is_p ? sa.sorted[qs] : h.pslot;
  r.k1 = ijk;
  r.k2 = ((unsigned long long)idh << 34) | ((unsigned long long)slot << 30) | (unsigned long long)idn;
  emit_pair(pairs, npairs, cap, r, sa.mark, st);
}

__device__ __forceinline__ int wrap_cell(int c, int n) { return c < 0 ? c + n : (c >= n ? c - n : c); }

// Cells [lo, hi] of one x-row as at most two contiguous ranges of sorted particles
// (periodic x wraps, otherwise the row is clipped).  lo >= -nfx and hi < 2 nfx.
struct RowRanges {
  int32_t a0, a1, b0, b1;
};
__device__ __forceinline__ RowRanges row_ranges(const SearchArrays &sa, int64_t base, int nfx, int lo, int hi,
                                                bool perx) {
  RowRanges r = {0, 0, 0, 0};
  if (hi - lo + 1 >= nfx && perx) {
    r.a0 = sa.cell_start[base];
    r.a1 = sa.cell_start[base + nfx];
    return r;
  }
  if (lo < 0) {
    if (perx) { r.b0 = sa.cell_start[base + nfx + lo]; r.b1 = sa.cell_start[base + nfx]; }
    lo = 0;
  }
  if (hi >= nfx) {
    if (perx) { r.b0 = sa.cell_start[base]; r.b1 = sa.cell_start[base + hi - nfx + 1]; }
    hi = nfx - 1;
  }
  if (lo <= hi) {
    r.a0 = sa.cell_start[base + lo];
    r.a1 = sa.cell_start[base + hi + 1];
  }
  return r;
}

// Pair search over the search grid.  The cell edge is at least twice the cut radius,
// so two small particles (bounding radius <= cut) can only meet in the same or an
// adjacent cell; a small particle sweeps the half stencil of its cell: the 13 forward
// neighbours that follow it in (z, y, x) order, (cx+1, cy, cz), the three cells
// cx-1..cx+1 of row (cy+1, cz) and the nine of layer cz+1.  Cells are numbered
// x-fastest, so these are five x-rows, each one or two contiguous ranges of sorted
// particles; the home cell is swept from the next sorted particle on.  A large particle
// (radius above the cut, rare) sweeps every cell within its radius plus the largest
// radius.  Every pair is visited exactly once.
#ifndef GP_SEARCH_MIN_BLOCKS
#define GP_SEARCH_MIN_BLOCKS 4
#endif

// A home particle's data, kept in shared memory for the lanes that test its candidates.
struct HomeRec {
  double xp, yp, zp, rp;
  long long bp;
  int32_t s, pslot, idp, inst;
};
constexpr int kSearchThreads = 256;
constexpr int kMaxRanges = 10;   // 5 rows, each at most two contiguous ranges

// Each lane takes one home particle (32 consecutive sorted particles per warp) and works
// out the ranges of sorted particles its half stencil must test: the five forward rows
// of cells, trimmed to the cells within reach.  The warp then tests all its homes'
// candidates together, 32 at a time: candidate idx of the warp's concatenated lists goes
// to lane idx mod 32, which looks up the owning home and range in shared memory.  Lanes
// stay busy however unevenly the candidates fall among the homes.  Homes above the cut
// radius sweep their wide stencil afterwards, each on its own lane.
__global__ void __launch_bounds__(kSearchThreads, GP_SEARCH_MIN_BLOCKS) k_search(
    const InstDev *__restrict__ insts, int64_t n, SearchArrays sa, PairRec *__restrict__ pairs,
    unsigned long long *npairs, int64_t cap, Status *st) {
  // no halt test here: this kernel is what raises the flag, and a later block must not
  // skip its pairs because an earlier one overflowed (the count it leaves in
  // pairs_needed sizes the buffers).  In a step after a halted one the binning did not
  // run and every cell is empty (its counts were cleared), so the sweep finds nothing.
  __shared__ HomeRec homes[kSearchThreads];
  __shared__ HomeF homesf[kSearchThreads];
  __shared__ int32_t rstart[kSearchThreads][kMaxRanges];   // first sorted particle of a range
  __shared__ int32_t rcum[kSearchThreads][kMaxRanges];     // candidates of the home before it
  __shared__ int8_t rnum[kSearchThreads];
  constexpr unsigned kFull = 0xffffffffu;
  const int t = threadIdx.x, lane = t & 31, wbase = t & ~31;
  const int64_t nact = sa.cell_start[sa.ncells];
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t s0 = (int64_t)blockIdx.x * blockDim.x + wbase; s0 < nact; s0 += stride) {
    const int64_t s = s0 + lane;
    int nr = 0;
    int32_t c = 0;
    bool large = false;
    int cx = 0, cy = 0, cz = 0;
    HomeRec hr;
    if (s < nact) {
      hr.inst = sa.sinst[s];
      const InstDev &I = insts[hr.inst];
      hr.s = (int32_t)s;
      hr.xp = sa.sx[s]; hr.yp = sa.sy[s]; hr.zp = sa.sz[s]; hr.rp = sa.sr[s];
      hr.bp = sa.sbox[s];
      hr.pslot = sa.sorted[s];
      hr.idp = sa.sid[s];
      homes[t] = hr;
      homesf[t] = home_f(I, hr.xp, hr.yp, hr.zp, hr.rp);
      const int nfx = I.nfx, nfy = I.nfy, nfz = I.nfz;
      const bool perx = I.periodicity != 0;
      // the binning pass's own cell of this particle (same inputs, same function)
      cx = cell_coord(hr.xp, I.hfx, nfx); cy = cell_coord(hr.yp, I.hfy, nfy); cz = cell_coord(hr.zp, I.hfz, nfz);
      const int64_t lc = ((int64_t)cz * nfy + cy) * nfx + cx;
      large = sa.spk[s].w < 0.f;
      if (!large) {
        // Small candidates have radius <= rcut, so only cells whose box comes within
        // R = rp + rcut of this particle can hold a partner: rows and end cells farther
        // away are skipped (distances to the neighbour boxes from the offsets inside the
        // home cell, shortened by 1e-9 of the cell edge against rounding).
        const double R = (hr.rp + I.rcut) * (1.0 + 1e-9), R2 = R * R;
        const double fx = hr.xp - cx * I.hfx, fy = hr.yp - cy * I.hfy, fz = hr.zp - cz * I.hfz;
        const double ex = 1e-9 * I.hfx, ey = 1e-9 * I.hfy, ez = 1e-9 * I.hfz;
        const double dxl = fmax(fx - ex, 0.0), dxh = fmax(I.hfx - fx - ex, 0.0);
        const double dyl = fmax(fy - ey, 0.0), dyh = fmax(I.hfy - fy - ey, 0.0);
        const double dzh = fmax(I.hfz - fz - ez, 0.0);
        auto add = [&](int32_t a0, int32_t a1) {
          if (a1 > a0) {
            rstart[t][nr] = a0;
            rcum[t][nr] = c;
            c += a1 - a0;
            ++nr;
          }
        };
        for (int r = 0; r < 5; ++r) {
          int ry = cy, rz = cz, lo = cx - 1, hi = cx + 1;
          double dyz2 = 0.0;
          if (r == 0) {
            lo = hi = cx + 1;                    // the rest of the home cell is taken below
          } else if (r == 1) {
            ry = wrap_cell(cy + 1, nfy);
            dyz2 = dyh * dyh;
          } else {
            rz = wrap_cell(cz + 1, nfz);
            ry = wrap_cell(cy + (r - 3), nfy);
            const double dyb = (r == 2) ? dyl : (r == 4 ? dyh : 0.0);
            dyz2 = dyb * dyb + dzh * dzh;
          }
          if (r > 0 && dyz2 > R2) continue;
          const int64_t base = I.cell_begin + ((int64_t)rz * nfy + ry) * nfx;
          // each end cell within reach of its own largest radius
          auto reach2 = [&](int cell) {
            const int w = cell < 0 ? cell + nfx : (cell >= nfx ? cell - nfx : cell);
            const double rr_ = (hr.rp + (double)sa.cell_rmax[base + w]) * (1.0 + 1e-9);
            return rr_ * rr_;
          };
          const bool left_ok = (cx - 1 >= 0 || perx);
          const bool right_ok = (cx + 1 < nfx || perx);
          if (r > 0 && (!left_ok || dxl * dxl + dyz2 > R2 || dxl * dxl + dyz2 > reach2(cx - 1))) lo = cx;
          const bool right = right_ok && dxh * dxh + dyz2 <= R2 && dxh * dxh + dyz2 <= reach2(cx + 1);
          if (r > 0 && !right) hi = cx;
          if (r > 0 && lo == cx && hi == cx && dyz2 > reach2(cx)) continue;
          RowRanges rr = {0, 0, 0, 0};
          if (r > 0 || right) rr = row_ranges(sa, base, nfx, lo, hi, perx);
          if (r == 0) {
            // home cell from s+1, contiguous with cell cx+1 when that is not wrapped
            if (rr.a1 == 0 && rr.a0 == 0) rr.a1 = sa.cell_start[I.cell_begin + lc + 1];
            rr.a0 = (int32_t)s + 1;
          }
          add(rr.a0, rr.a1);
          add(rr.b0, rr.b1);
        }
      }
    }
    rnum[t] = (int8_t)nr;
    __syncwarp();
    // the warp's candidate lists, concatenated in lane order
    int32_t incl = c;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int32_t v = __shfl_up_sync(kFull, incl, d);
      if (lane >= d) incl += v;
    }
    const int32_t total = __shfl_sync(kFull, incl, 31);
    const int32_t excl = incl - c;
    for (int32_t base = 0; base < total; base += 32) {
      const int32_t idx = base + lane;
      // the last lane o whose list starts at or before idx owns it
      int o = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const int32_t e = __shfl_sync(kFull, excl, (o + step) & 31);
        if (o + step < 32 && e <= idx) o += step;
      }
      const int32_t eo = __shfl_sync(kFull, excl, o);
      if (idx < total) {
        const int to = wbase + o;
        const int32_t k = idx - eo;
        int j = 0;
        const int no = rnum[to];
        while (j + 1 < no && rcum[to][j + 1] <= k) ++j;
        const int32_t q = rstart[to][j] + (k - rcum[to][j]);
        if (near_float<false>(sa.spk[q], q, 0, homesf[to])) {
          const HomeRec ho = homes[to];
          const InstDev &I = insts[ho.inst];
          SearchHome h;
          h.s = ho.s; h.xp = ho.xp; h.yp = ho.yp; h.zp = ho.zp; h.rp = ho.rp;
          h.bp = ho.bp; h.pslot = ho.pslot; h.idp = ho.idp;
          h.perx = I.periodicity != 0;
          search_candidate(I, sa, h, q, pairs, npairs, cap, st);
        }
      }
    }
    if (large) {
      // a particle above the cut: every cell within its radius plus the largest radius
      const InstDev &I = insts[hr.inst];
      const int nfx = I.nfx, nfy = I.nfy, nfz = I.nfz;
      SearchHome h;
      h.s = hr.s; h.xp = hr.xp; h.yp = hr.yp; h.zp = hr.zp; h.rp = hr.rp;
      h.bp = hr.bp; h.pslot = hr.pslot; h.idp = hr.idp;
      h.perx = I.periodicity != 0;
      const HomeF hf = home_f(I, h.xp, h.yp, h.zp, h.rp);
      const double reach = (h.rp + I.rmax) * (1.0 + 1.0e-6);
      const int rx = (int)ceil(reach / I.hfx), ry = (int)ceil(reach / I.hfy), rz = (int)ceil(reach / I.hfz);
      const bool ally = 2 * ry + 1 >= nfy, allz = 2 * rz + 1 >= nfz;
      const int y0 = ally ? 0 : cy - ry, y1 = ally ? nfy - 1 : cy + ry;
      const int z0 = allz ? 0 : cz - rz, z1 = allz ? nfz - 1 : cz + rz;
      const int lo = (2 * rx + 1 >= nfx) ? 0 : cx - rx, hi = (2 * rx + 1 >= nfx) ? nfx - 1 : cx + rx;
      for (int zz = z0; zz <= z1; ++zz) {
        const int wz = wrap_cell(zz, nfz);
        for (int yy = y0; yy <= y1; ++yy) {
          const int wy = wrap_cell(yy, nfy);
          const int64_t base = I.cell_begin + ((int64_t)wz * nfy + wy) * nfx;
          const RowRanges rr = row_ranges(sa, base, nfx, lo, hi, h.perx || (2 * rx + 1 >= nfx));
          for (int32_t qs = rr.a0; qs < rr.a1; ++qs)
            if (qs != s && near_float<true>(sa.spk[qs], qs, h.s, hf))
              search_candidate(I, sa, h, qs, pairs, npairs, cap, st);
          for (int32_t qs = rr.b0; qs < rr.b1; ++qs)
            if (qs != s && near_float<true>(sa.spk[qs], qs, h.s, hf))
              search_candidate(I, sa, h, qs, pairs, npairs, cap, st);
        }
      }
    }
    __syncwarp();   // the records are rewritten by the warp's next 32 homes
  }
}

void launch_search(const InstDev *insts, int64_t n, SearchArrays sa, PairRec *pairs, unsigned long long *npairs,
                   int64_t cap_pairs, Status *st, int grid, cudaStream_t s) {
  k_search<<<grid, 256, 0, s>>>(insts, n, sa, pairs, npairs, cap_pairs, st);
}

// ---------------------------------------------------------------------------
// 5. lexicographically-first maximal matching of the colliding pairs
//    (the outcome of the COLOR walk, collision_interaction.f90:190-207,397-398)
// ---------------------------------------------------------------------------
constexpr int kMatchThreads = 1024;

__global__ void __launch_bounds__(kMatchThreads) k_match(const CollRec *__restrict__ coll,
                                                         const unsigned long long *__restrict__ ncoll, int64_t cap,
                                                         unsigned long long *best1, unsigned long long *best2,
                                                         int8_t *matched, int8_t *state, Status *st) {
  if (step_halted(st)) return;
  __shared__ int remaining_s[kMatchThreads / 32];
  __shared__ int remaining;
  const int64_t nc = (int64_t)min(*ncoll, (unsigned long long)cap);
  const unsigned long long kMax = ~0ull;
  for (int64_t e = threadIdx.x; e < nc; e += kMatchThreads) state[e] = 0;
  __syncthreads();
  bool done = (nc == 0);
  int64_t pass = 0;
  while (!done) {
    for (int64_t e = threadIdx.x; e < nc; e += kMatchThreads) {
      if (state[e] != 0) continue;
      const CollRec &r = coll[e];
      atomicMin(&best1[r.home], r.k1);
      atomicMin(&best1[r.near], r.k1);
    }
    __syncthreads();
    for (int64_t e = threadIdx.x; e < nc; e += kMatchThreads) {
      if (state[e] != 0) continue;
      const CollRec &r = coll[e];
      if (best1[r.home] == r.k1) atomicMin(&best2[r.home], r.k2);
      if (best1[r.near] == r.k1) atomicMin(&best2[r.near], r.k2);
    }
    __syncthreads();
    for (int64_t e = threadIdx.x; e < nc; e += kMatchThreads) {
      if (state[e] != 0) continue;
      const CollRec &r = coll[e];
      if (best1[r.home] == r.k1 && best2[r.home] == r.k2 && best1[r.near] == r.k1 && best2[r.near] == r.k2) {
        state[e] = 3;   // accepted in this pass
        matched[r.home] = 1;
        matched[r.near] = 1;
      }
    }
    __syncthreads();
    for (int64_t e = threadIdx.x; e < nc; e += kMatchThreads) {
      const int8_t sv = state[e];
      if (sv != 0 && sv != 3) continue;
      const CollRec &r = coll[e];
      best1[r.home] = kMax; best1[r.near] = kMax;
      best2[r.home] = kMax; best2[r.near] = kMax;
    }
    __syncthreads();
    int cnt = 0;
    for (int64_t e = threadIdx.x; e < nc; e += kMatchThreads) {
      const int8_t sv = state[e];
      if (sv == 3) { state[e] = 1; continue; }
      if (sv != 0) continue;
      const CollRec &r = coll[e];
      if (matched[r.home] || matched[r.near]) state[e] = 2; else ++cnt;
    }
    cnt = __reduce_add_sync(0xffffffffu, cnt);
    if ((threadIdx.x & 31) == 0) remaining_s[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
      int t = 0;
      for (int w = 0; w < kMatchThreads / 32; ++w) t += remaining_s[w];
      remaining = t;
    }
    __syncthreads();
    ++pass;
    done = (remaining == 0);
    if (!done && pass > nc + 1) {   // every pass accepts at least one pair; cannot happen
      if (threadIdx.x == 0) set_error(st, GP_ETIMEOUT, pass);
      done = true;
    }
  }
  __syncthreads();
  for (int64_t e = threadIdx.x; e < nc; e += kMatchThreads) {
    const CollRec &r = coll[e];
    matched[r.home] = 0;
    matched[r.near] = 0;
  }
}

void launch_match(const CollRec *coll, const unsigned long long *ncoll, int64_t cap_coll, unsigned long long *best1,
                  unsigned long long *best2, int8_t *matched, int8_t *state, Status *st, cudaStream_t s) {
  k_match<<<1, kMatchThreads, 0, s>>>(coll, ncoll, cap_coll, best1, best2, matched, state, st);
}

// ---------------------------------------------------------------------------
// Data movement
// ---------------------------------------------------------------------------
// Internal field layout from a reference-layout or interior source (one component).
template <typename T>
__global__ void k_field_layout(T *__restrict__ dst, int nx, int ny, int nz, int ncomp, int comp,
                               const double *__restrict__ src, int src_layout, int ghost_mode) {
  const int64_t sx = nx + 3, sy = ny + 4, sz = nz + 4;
  const int64_t total = sx * sy * sz;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int ix = (int)(t % sx), jy = (int)((t / sx) % sy), kz = (int)(t / (sx * sy));
    int i = ix;
    if (ix == 0) i = nx;
    else if (ix == nx + 1) i = 1;
    else if (ix == nx + 2) i = 2;
    const int j = jy - 1, k = kz - 1;   // reference indices, -1..N+2
    double v;
    if (src_layout == GP_LAYOUT_REFERENCE) {
      v = src[(int64_t)(i - 1) + (int64_t)nx * ((int64_t)(j + 1) + (int64_t)(ny + 4) * (int64_t)(k + 1))];
    } else {
      const bool inside = (j >= 1 && j <= ny && k >= 1 && k <= nz);
      if (!inside && ghost_mode == GP_GHOST_ZERO) {
        v = 0.0;
      } else {
        const int jj = (j < 1) ? j + ny : (j > ny ? j - ny : j);
        const int kk = (k < 1) ? k + nz : (k > nz ? k - nz : k);
        v = src[(int64_t)(i - 1) + (int64_t)nx * ((int64_t)(jj - 1) + (int64_t)ny * (int64_t)(kk - 1))];
      }
    }
    dst[t * ncomp + comp] = (T)v;
  }
}

void launch_field_layout(void *dst, int prec, int nx, int ny, int nz, int ncomp, int comp, const double *src,
                         int src_layout, int ghost_mode, cudaStream_t s) {
  const int grid = 148 * 8;
  if (prec == GP_PREC_MIXED)
    k_field_layout<float><<<grid, 256, 0, s>>>(static_cast<float *>(dst), nx, ny, nz, ncomp, comp, src, src_layout,
                                                ghost_mode);
  else
    k_field_layout<double><<<grid, 256, 0, s>>>(static_cast<double *>(dst), nx, ny, nz, ncomp, comp, src,
                                                 src_layout, ghost_mode);
}

// Pool -> caller order: out[c*count + begin(class) + id] = state column c, where the
// caller's arrays hold the classes one after another; with only >= 0, class `only`
// alone at offset 0.  Only the columns whose bit is set in `cols` are written.
__global__ void k_gather_state(const InstDev *__restrict__ insts, const PoolView *__restrict__ pv, int64_t n,
                               int only, double *__restrict__ out, double *const *fluid, double *__restrict__ fout,
                               int64_t count, unsigned cols) {
  const PoolView P = *pv;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int inst = P.inst[i];
    if (inst < 0 || (only >= 0 && inst != only)) continue;
    const int64_t id = (only >= 0 ? 0 : insts[inst].begin) + P.id[i];
    if (id < 0 || id >= count) continue;
#pragma unroll
    for (int c = 0; c < kNState; ++c)
      if ((cols >> c) & 1u) out[c * count + id] = P.st[c][i];
    if (fout != nullptr && fluid != nullptr) {
#pragma unroll
      for (int c = 0; c < kNFluid; ++c) fout[c * count + id] = fluid[c][i];
    }
  }
}

void launch_gather_state(const InstDev *insts, const PoolView *pv, int64_t n, int only, double *out,
                         double *const *fluid_cols, double *fluid_out, int64_t count, cudaStream_t s,
                         unsigned cols) {
  const int grid = 148 * 8;
  k_gather_state<<<grid, 256, 0, s>>>(insts, pv, n, only, out, fluid_cols, fluid_out, count, cols);
}

// Retires class `inst`: its particles leave the binning, and the next advance drops them.
__global__ void k_retire(const PoolView *__restrict__ pv, int64_t n, int inst) {
  const PoolView P = *pv;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (P.inst[i] == inst) P.inst[i] = -1;
}

void launch_retire(const PoolView *pv, int64_t n, int inst, cudaStream_t s) {
  if (n > 0) k_retire<<<148 * 8, 256, 0, s>>>(pv, n, inst);
}

// caller order -> pool (state columns only; those whose bit is set in `mask`)
__global__ void k_scatter_state(const InstDev *__restrict__ insts, const PoolView *__restrict__ pv, int64_t n,
                                const double *__restrict__ cols, int64_t count, unsigned mask) {
  const PoolView P = *pv;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int inst = P.inst[i];
    if (inst < 0) continue;
    const int64_t id = insts[inst].begin + P.id[i];
    if (id < 0 || id >= count) continue;
#pragma unroll
    for (int c = 0; c < kNState; ++c)
      if ((mask >> c) & 1u) P.st[c][i] = cols[c * count + id];
  }
}

void launch_scatter_state(const InstDev *insts, const PoolView *pv, int64_t n, const double *cols, int64_t count,
                          cudaStream_t s, unsigned mask) {
  k_scatter_state<<<148 * 8, 256, 0, s>>>(insts, pv, n, cols, count, mask);
}

// One class into pool slots [begin, begin+n): particle k of the class is column entry
// src + k of the staged arrays (leading dimension ld); ids are 0-based within the class.
__global__ void k_init_pool(const PoolView *__restrict__ pv, int64_t begin, int64_t n, int inst,
                            const double *__restrict__ cols, const double *__restrict__ pcs, int64_t ld,
                            int64_t src) {
  const PoolView P = *pv;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = begin + k, e = src + k;
#pragma unroll
    for (int c = 0; c < kNState; ++c) P.st[c][i] = cols[c * ld + e];
#pragma unroll
    for (int c = 0; c < kNConst; ++c) P.pc[c][i] = pcs[c * ld + e];
    P.id[i] = (int32_t)k;
    P.inst[i] = inst;
  }
}

void launch_init_pool(const PoolView *pv, int64_t begin, int64_t n, int inst, const double *cols, const double *pcs,
                      int64_t ld, int64_t src, cudaStream_t s) {
  if (n <= 0) return;
  k_init_pool<<<148 * 8, 256, 0, s>>>(pv, begin, n, inst, cols, pcs, ld, src);
}

__global__ void k_iota(int32_t *a, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    a[i] = (int32_t)i;
}

void launch_iota(int32_t *a, int64_t n, cudaStream_t s) {
  if (n > 0) k_iota<<<148 * 8, 256, 0, s>>>(a, n);
}

// COLLISION_BOX_CONNECTIVITY (collision_box_connectivity.f90:42-322), NPROC=1.
__global__ void k_connectivity(int NXB, int NYB, int NZB, int periodicity, int32_t *ncon, int32_t *con) {
  const int64_t nbox = (int64_t)NXB * NYB * NZB;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nbox; t += (int64_t)gridDim.x * blockDim.x) {
    const int i0 = (int)(t % NXB) + 1, j0 = (int)((t / NXB) % NYB) + 1, k0 = (int)(t / ((int64_t)NXB * NYB)) + 1;
    auto BOX = [&](int i, int j, int k) { return (int32_t)(i + (j - 1) * NXB + (k - 1) * NXB * NYB); };
    int im1 = i0 - 1, ip1 = i0 + 1, jm1 = j0 - 1, jp1 = j0 + 1, km1 = k0 - 1, kp1 = k0 + 1;
    if (im1 < 1 && periodicity) im1 = NXB;
    if (ip1 > NXB && periodicity) ip1 = 1;
    if (jm1 < 1) jm1 = NYB;
    if (jp1 > NYB) jp1 = 1;
    if (km1 < 1) km1 = NZB;
    if (kp1 > NZB) kp1 = 1;
    int32_t c[27];
    int nn = 0;
    if (km1 >= 1 && jp1 <= NYB && ip1 <= NXB) c[nn++] = BOX(ip1, jp1, km1);   // box 9
    if (jm1 >= 1 && ip1 <= NXB) c[nn++] = BOX(ip1, jm1, k0);                  // box 12
    if (ip1 <= NXB) c[nn++] = BOX(ip1, j0, k0);                                // box 15
    if (jp1 <= NYB) {
      c[nn++] = BOX(i0, jp1, k0);                                               // box 17
      if (ip1 <= NXB) c[nn++] = BOX(ip1, jp1, k0);                             // box 18
    }
    if (kp1 <= NZB) {
      if (jm1 >= 1) {
        c[nn++] = BOX(i0, jm1, kp1);                                            // box 20
        if (ip1 <= NXB) c[nn++] = BOX(ip1, jm1, kp1);                          // box 21
      }
      if (im1 >= 1) c[nn++] = BOX(im1, j0, kp1);                               // box 22
      c[nn++] = BOX(i0, j0, kp1);                                               // box 23
      if (ip1 <= NXB) c[nn++] = BOX(ip1, j0, kp1);                             // box 24
      if (jp1 <= NYB) {
        if (im1 >= 1) c[nn++] = BOX(im1, jp1, kp1);                            // box 25
        c[nn++] = BOX(i0, jp1, kp1);                                            // box 26
        if (ip1 <= NXB) c[nn++] = BOX(ip1, jp1, kp1);                          // box 27
      }
    }
    const int64_t ijk = (i0 - 1) + (int64_t)(j0 - 1) * NXB + (int64_t)(k0 - 1) * NXB * NYB;
    ncon[ijk] = nn;
    for (int q = 0; q < 27; ++q) con[ijk * 27 + q] = (q < nn) ? c[q] : 0;
  }
}

void launch_connectivity(int nxb, int nyb, int nzb, int periodicity, int32_t *ncon, int32_t *con, cudaStream_t s) {
  k_connectivity<<<148 * 8, 128, 0, s>>>(nxb, nyb, nzb, periodicity, ncon, con);
}

}  // namespace gp
