// gp_gather_tma.cu -- the FP32 stencil gather (interp_lag3.f90:124-288 for the six
// field components) with each particle's stencil box staged in shared memory by the
// tensor-memory accelerator.
//
// The field is [z][y][x][8] FP32 (six components padded to eight, so a point is 32
// bytes).  A particle's 4 x 4 x 4-point stencil is one box of that array, {8, 4, 4, 4}
// elements, 2 KB: one cp.async.bulk.tensor request brings it into shared memory.  Each
// warp takes runs of 32 slots of the cell order from a counter (as k_gather does) and
// works through a run in eight groups of four particles; the boxes of the next groups
// are in flight while a group is summed, in kTmaStages buffers of four boxes, each
// completed on its own mbarrier.  The sums read the boxes from shared memory in the
// order and with the roundings of gather_warp_fp32 (gp_advance.cuh), so the two paths
// give the same values bit for bit.  Stencils that are not four contiguous points in x
// (the channel's mirrored walls) are gathered per lane, as in k_gather.
//
// The tensor map covers this GPU's own field only and the loads are not multicast.  The
// box origin's innermost coordinate is the component index 0, so every request starts
// on a 32-byte boundary.  A wait that runs past its limit records GP_ETIMEOUT, waits
// (again bounded) for the warp's loads still in flight and ends the kernel.
#include <cuda.h>
#include <cuda_runtime.h>
#include <math_constants.h>

#include "gp_advance.cuh"
#include "gp_launch.h"

namespace gp {
namespace {

constexpr int kTmaThreads = 128;                                 // four warps a block
constexpr int kTmaWarps = kTmaThreads / 32;
constexpr int kTmaStages = 3;                                    // groups of four boxes per warp
constexpr int kBoxFloats = 4 * 4 * 4 * kFieldStride;             // 512 floats, 2 KB
constexpr int kGroupFloats = 4 * kBoxFloats;                     // 8 KB
constexpr int kWarpFloats = kTmaStages * kGroupFloats;           // 24 KB
constexpr size_t kTmaSmemBytes = (size_t)kTmaWarps * kWarpFloats * sizeof(float) +
                                 (size_t)kTmaWarps * kTmaStages * sizeof(uint64_t);
constexpr long long kWaitLimit = 1ll << 20;                       // polls of one phase

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// true once the barrier's phase of this parity has completed
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  uint32_t done;
  asm volatile(
      "{\n"
      "  .reg .pred p;\n"
      "  mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      "  selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Waits for the phase, at most kWaitLimit polls; false if it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
  for (long long tries = 0; tries < kWaitLimit; ++tries)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// One stencil box {c 0..7, x0..x0+3, y0..y0+3, z0..z0+3} of the field into dst.
__device__ __forceinline__ void tma_load_box(float* dst, const CUtensorMap* map, int x0, int y0, int z0,
                                             uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(x0), "r"(y0), "r"(z0), "r"(smem_u32(bar))
      : "memory");
}

__global__ void __launch_bounds__(kTmaThreads, 2)
    k_gather_tma(const __grid_constant__ CUtensorMap map, const InstDev* __restrict__ insts,
                 const PoolView* __restrict__ src_pv, const int32_t* __restrict__ perm, int64_t n,
                 double* const* __restrict__ fluid, unsigned long long* __restrict__ ticket, Status* st) {
  extern __shared__ __align__(128) float smem[];
  if (step_halted(st)) return;
  constexpr unsigned kFull = 0xffffffffu;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float* const buf = smem + warp * kWarpFloats;
  uint64_t* const bar = reinterpret_cast<uint64_t*>(smem + kTmaWarps * kWarpFloats) + warp * kTmaStages;
  if (lane == 0)
    for (int s = 0; s < kTmaStages; ++s) mbar_init(&bar[s], 1);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  __syncwarp();
  unsigned parity = 0;      // bit s: parity of stage s's next phase
  unsigned pending = 0;     // bit s: a phase of stage s issued and not yet waited for
  const int t = lane & 7, k = t >> 1, half = t & 1;
  for (;;) {
    unsigned long long wt = 0;
    if (lane == 0) wt = atomicAdd(ticket, 1ull);
    const int64_t w = (int64_t)__shfl_sync(kFull, wt, 0);
    if (w * 32 >= n) break;
    const int64_t j = w * 32 + lane;
    int inst = -1;
    int64_t i = 0;
    if (j < n) {
      i = perm[j];
      inst = src_pv->inst[i];
    }
    int mode = 0;
    Stencil s;
    if (inst >= 0) {
      if (stencil(insts[inst], src_pv->st[0][i], src_pv->st[1][i], src_pv->st[2][i], s))
        mode = s.contiguous ? 1 : 2;
      else
        set_error(st, GP_EOUT_OF_GRID, (long long)src_pv->id[i], inst);
    }
    if (j < n && mode == 0) {
#pragma unroll
      for (int c = 0; c < 6; ++c) fluid[c][j] = CUDART_NAN;
    }
    // box origin in the field array: point (ix[0], j0 - 1, k0 - 1) of field_point
    const int x0 = (mode == 1) ? s.ix[0] : 0, y0 = (mode == 1) ? s.j0 : 0, z0 = (mode == 1) ? s.k0 : 0;
    const unsigned boxed = __ballot_sync(kFull, mode == 1);
    // Group g (particles 4g .. 4g+3 of the run) into stage g % kTmaStages: lane 4g arms the
    // barrier with the group's bytes, then each of the four lanes requests its own box.
    auto issue = [&](int g) {
      const int sg = g % kTmaStages;
      const unsigned mine = (boxed >> (4 * g)) & 0xFu;
      __syncwarp();
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // earlier reads of the buffer
      if (lane == 4 * g) mbar_arrive_expect_tx(&bar[sg], (unsigned)__popc(mine) * kBoxFloats * 4u);
      __syncwarp();
      if ((lane >> 2) == g && mode == 1)
        tma_load_box(buf + sg * kGroupFloats + (lane & 3) * kBoxFloats, &map, x0, y0, z0, &bar[sg]);
      pending |= 1u << sg;
    };
#pragma unroll 1
    for (int g = 0; g < kTmaStages; ++g) issue(g);
    bool ok = true;
#pragma unroll 1
    for (int g = 0; g < 8; ++g) {
      const int sg = g % kTmaStages;
      const int o = g * 4 + (lane >> 3);
      const int mo = __shfl_sync(kFull, mode, o);
      const float alo = __shfl_sync(kFull, (float)s.alfa, o), beo = __shfl_sync(kFull, (float)s.beta, o);
      const float gao = __shfl_sync(kFull, (float)s.gama, o);
      if (!__all_sync(kFull, mbar_wait(&bar[sg], (parity >> sg) & 1u))) {
        ok = false;
        break;
      }
      parity ^= 1u << sg;
      pending &= ~(1u << sg);
      float4 zs = make_float4(0.f, 0.f, 0.f, 0.f);
      float wxl = 0.f;
      if (mo == 1) {
        float fx[4], fy[4], fz[4];
        lag3_wf(alo, fx);
        lag3_wf(beo, fy);
        lag3_wf(gao, fz);
        const float wx = pick4(fx, k);
        const float* p = buf + sg * kGroupFloats + (lane >> 3) * kBoxFloats + k * kFieldStride + 4 * half;
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
          float4 ys = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
          for (int jj = 0; jj < 4; ++jj) {
            const float4 v = *reinterpret_cast<const float4*>(p + (kk * 4 + jj) * 4 * kFieldStride);
            ys.x = __fmaf_rn(fy[jj], v.x, ys.x);
            ys.y = __fmaf_rn(fy[jj], v.y, ys.y);
            ys.z = __fmaf_rn(fy[jj], v.z, ys.z);
            ys.w = __fmaf_rn(fy[jj], v.w, ys.w);
          }
          zs.x = __fmaf_rn(fz[kk], ys.x, zs.x);
          zs.y = __fmaf_rn(fz[kk], ys.y, zs.y);
          zs.z = __fmaf_rn(fz[kk], ys.z, zs.z);
          zs.w = __fmaf_rn(fz[kk], ys.w, zs.w);
        }
        wxl = wx;
      }
      const double wd = (double)wxl;
      double d0 = (double)zs.x * wd, d1 = (double)zs.y * wd;
      double d2 = (double)zs.z * wd, d3 = (double)zs.w * wd;
#pragma unroll
      for (int m = 2; m <= 4; m <<= 1) {
        d0 += __shfl_xor_sync(kFull, d0, m);
        d1 += __shfl_xor_sync(kFull, d1, m);
        d2 += __shfl_xor_sync(kFull, d2, m);
        d3 += __shfl_xor_sync(kFull, d3, m);
      }
      if (mo == 1 && t < 2) {
        const int64_t jo = w * 32 + o;
        if (half == 0) {
          fluid[0][jo] = d0; fluid[1][jo] = d1; fluid[2][jo] = d2; fluid[3][jo] = d3;
        } else {
          fluid[4][jo] = d0; fluid[5][jo] = d1;
        }
      }
      if (g + kTmaStages < 8) issue(g + kTmaStages);
    }
    if (!ok) {
      // a box that never arrived: report it, let the warp's other requests land, stop
      if (lane == 0) set_error(st, GP_ETIMEOUT, -1);
      for (int sg = 0; sg < kTmaStages; ++sg)
        if (pending & (1u << sg)) mbar_wait(&bar[sg], (parity >> sg) & 1u);
      return;
    }
    if (mode == 2) {
      double g6[6];
      gather6_fp32(insts[inst], s, g6);
#pragma unroll
      for (int c = 0; c < 6; ++c) fluid[c][j] = g6[c];
    }
  }
}

}  // namespace

size_t gather_tma_smem_bytes() { return kTmaSmemBytes; }

int gather_tma_prepare() {
  return cudaFuncSetAttribute(k_gather_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTmaSmemBytes) ==
                 cudaSuccess
             ? GP_OK
             : GP_ECUDA;
}

// Tensor map over an FP32 field slot laid out [z: nz+4][y: ny+4][x: nx+3][8]: boxes of
// {8, 4, 4, 4} elements.  cuTensorMapEncodeTiled is reached through the runtime's driver
// entry points, so that the library needs no link to the driver library.
int make_field_map(const void* field, int nx, int ny, int nz, CUtensorMap* out) {
  using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  // looked up once (a thread-safe static initialisation); null if the driver lacks it
  static const Encode encode = []() -> Encode {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    return reinterpret_cast<Encode>(f);
  }();
  if (!encode) return GP_ECUDA;
  if (!field || (reinterpret_cast<uintptr_t>(field) & 15u) != 0) return GP_EBADARG;
  const cuuint64_t row = (cuuint64_t)kFieldStride * sizeof(float);
  const cuuint64_t dims[4] = {(cuuint64_t)kFieldStride, (cuuint64_t)nx + 3, (cuuint64_t)ny + 4, (cuuint64_t)nz + 4};
  const cuuint64_t strides[3] = {row, row * ((cuuint64_t)nx + 3), row * ((cuuint64_t)nx + 3) * ((cuuint64_t)ny + 4)};
  const cuuint32_t box[4] = {(cuuint32_t)kFieldStride, 4, 4, 4};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUresult r = encode(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<void*>(field), dims, strides, box,
                            estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? GP_OK : GP_ECUDA;
}

void launch_gather_tma(const CUtensorMap& map, const InstDev* insts, const PoolView* pv, const int32_t* perm,
                       int64_t n, double* const* fluid, unsigned long long* ticket, Status* st, int grid,
                       cudaStream_t s) {
  cudaMemsetAsync(ticket, 0, sizeof(unsigned long long), s);
  k_gather_tma<<<grid, kTmaThreads, kTmaSmemBytes, s>>>(map, insts, pv, perm, n, fluid, ticket, st);
}

}  // namespace gp
