// gp_noalloc.cu -- batched ellipsoid contact detection that allocates no memory.
//
// Some callers of this library cannot allocate device memory at the point where they
// need a contact solve: a solver that has already filled HBM with its particle pool
// (an allocation would fail), a real-time loop that cannot afford the device-wide
// synchronisation that cudaFree implies, or a host program whose memory plan is fixed
// at start-up and forbids allocation afterwards.  The context-based
// gp_ellipsoid_contact_detection_batch grows a per-context device buffer on demand, so
// it is closed to them.  gp_ellipsoid_contact_detection_batch_noalloc serves them
// instead: it needs no context, and it stages inputs and results through one
// fixed-size array placed in device memory when the library is loaded.
//
// Limits and sharing rules
//  - At most GP_NOALLOC_MAX_PAIRS pairs per call; larger calls return GP_EBADARG and do
//    no work.  The staging array costs GP_NOALLOC_MAX_PAIRS * 220 bytes (7.2 MB) of
//    device memory on every device that loads the library.
//  - The array is shared by every call on a device and keeps the previous call's
//    contents.  The kernel overwrites every output slot of the pairs it is given before
//    the results are copied out, so nothing in the array has to start at zero.
//  - Calls that may overlap on the GPU (different streams or host threads on one
//    device) race on the array; callers must order them, for instance by using one
//    stream.
//  - The call waits for its stream before it returns.  A stream that is being captured
//    (or the legacy default stream while another stream captures) is refused with
//    GP_EBADARG before anything is enqueued, so the caller's capture is left intact.
//  - The first call on each device (and again after the device's context has been
//    replaced, e.g. by cudaDeviceReset) looks up the array's device address with that
//    device current.  That call may make the CUDA runtime load this library's device
//    code.
//
// This file is compiled without FMA contraction (-fmad=false), as the FP64 kernels are,
// so its results equal those of gp_ellipsoid_contact_detection_batch bit for bit.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/gazpart_gpu.h"
#include "gp_lm.cuh"

namespace gp {
namespace {

// per pair: shapes 4, centres 6, quaternions 8, ept1 3, ept2 3, cnormal 3 doubles,
// then one int32 flag (stored two to a double slot)
constexpr int64_t kMaxPairs = GP_NOALLOC_MAX_PAIRS;
constexpr int64_t kDoublesPerPair = 4 + 6 + 8 + 3 + 3 + 3;
constexpr int64_t kScratchDoubles = kDoublesPerPair * kMaxPairs + kMaxPairs / 2;

static __device__ __align__(256) double g_contact_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
// Per device: the context the address was looked up in, and the address.
unsigned long long g_scratch_ctx[kMaxDevices] = {};
double *g_scratch_ptr[kMaxDevices] = {};

struct Regions {
  double *shapes, *centres, *quats, *e1, *e2, *cn;
  int32_t *flag;
};

// Regions are laid out for the maximum size, so they do not depend on n.
__host__ __device__ Regions regions(double *base) {
  Regions r;
  r.shapes = base;
  r.centres = r.shapes + 4 * kMaxPairs;
  r.quats = r.centres + 6 * kMaxPairs;
  r.e1 = r.quats + 8 * kMaxPairs;
  r.e2 = r.e1 + 3 * kMaxPairs;
  r.cn = r.e2 + 3 * kMaxPairs;
  r.flag = reinterpret_cast<int32_t *>(r.cn + 3 * kMaxPairs);
  return r;
}

// ellipsoid_contact_detection.f90:1-187 for n pairs held in the staging array.  Shapes
// arrive as (emaj1, apr1, emaj2, apr2); the minor semi-axis emaj/apr is formed here with
// the same correctly rounded division the context-based entry point does on the host.
__global__ void __launch_bounds__(128, 4) k_contact_batch_staged(int64_t n, double *base) {
  const Regions r = regions(base);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double *s = r.shapes + 4 * i, *c = r.centres + 6 * i, *q = r.quats + 8 * i;
    const Quat q1 = {q[0], q[1], q[2], q[3]}, q2 = {q[4], q[5], q[6], q[7]};
    double a[3], b[3], nn[3];
    r.flag[i] = contact_detection(s[0], s[0] / s[1], s[2], s[2] / s[3], c, q1, c + 3, q2, a, b, nn) ? 1 : 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      r.e1[3 * i + k] = a[k];
      r.e2[3 * i + k] = b[k];
      r.cn[3 * i + k] = nn[k];
    }
  }
}

// Unique id of the current CUDA context (cuCtxGetId), through the runtime's driver
// entry points so that the library needs no link to the driver library.  0 if the
// runtime has not made a context current yet.
int current_context_id(unsigned long long *id) {
  using GetCurrent = CUresult (*)(CUcontext *);
  using GetId = CUresult (*)(CUcontext, unsigned long long *);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  if (!get_current || !get_id) {
    void *f1 = nullptr, *f2 = nullptr;
    cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = q1;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
        cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) != cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f1 || !f2)
      return GP_ECUDA;
    get_current = reinterpret_cast<GetCurrent>(f1);
    get_id = reinterpret_cast<GetId>(f2);
  }
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS) return GP_ECUDA;
  *id = 0;
  if (ctx && get_id(ctx, id) != CUDA_SUCCESS) return GP_ECUDA;
  return GP_OK;
}

// Device address of the staging array on the current device.  Looked up once per device
// and context: a new context (after cudaDeviceReset) may load the module at another
// address, so the lookup is repeated when the context id changes.
int scratch_for_current_device(double **out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return GP_ECUDA;
  if (dev < 0 || dev >= kMaxDevices) return GP_EBADARG;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  unsigned long long ctx = 0;
  int rc = current_context_id(&ctx);
  if (rc) return rc;
  if (!g_scratch_ptr[dev] || ctx == 0 || ctx != g_scratch_ctx[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_contact_scratch) != cudaSuccess || !p) return GP_ECUDA;
    // the lookup makes the runtime's context current if it was not yet
    rc = current_context_id(&ctx);
    if (rc) return rc;
    if (ctx == 0) return GP_ECUDA;
    g_scratch_ptr[dev] = static_cast<double *>(p);
    g_scratch_ctx[dev] = ctx;
  }
  *out = g_scratch_ptr[dev];
  return GP_OK;
}

}  // namespace
}  // namespace gp

extern "C" int gp_ellipsoid_contact_detection_batch_noalloc(int64_t n, const double *shapes,
                                                            const double *centres, const double *quats,
                                                            int32_t *flag, double *ept1, double *ept2,
                                                            double *cnormal, int32_t on_device,
                                                            void *stream) {
  using namespace gp;
  if (n < 0 || n > kMaxPairs) return GP_EBADARG;
  if (n == 0) return GP_OK;
  if (!shapes || !centres || !quats || !flag || !ept1 || !ept2 || !cnormal) return GP_EBADARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the call ends by waiting for the stream, which a stream under capture cannot do
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) {
    (void)cudaGetLastError();
    return GP_EBADARG;
  }
  if (cs != cudaStreamCaptureStatusNone) return GP_EBADARG;
  double *base = nullptr;
  const int rc = scratch_for_current_device(&base);
  if (rc) return rc;
  const Regions r = regions(base);
  const cudaMemcpyKind kin = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  const cudaMemcpyKind kout = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  const size_t nd = (size_t)n * sizeof(double);
  if (cudaMemcpyAsync(r.shapes, shapes, 4 * nd, kin, s) != cudaSuccess ||
      cudaMemcpyAsync(r.centres, centres, 6 * nd, kin, s) != cudaSuccess ||
      cudaMemcpyAsync(r.quats, quats, 8 * nd, kin, s) != cudaSuccess)
    return GP_ECUDA;
  const int64_t blocks = (n + 127) / 128;
  k_contact_batch_staged<<<(int)(blocks < 148 * 8 ? blocks : 148 * 8), 128, 0, s>>>(n, base);
  if (cudaGetLastError() != cudaSuccess) return GP_ECUDA;
  if (cudaMemcpyAsync(flag, r.flag, (size_t)n * sizeof(int32_t), kout, s) != cudaSuccess ||
      cudaMemcpyAsync(ept1, r.e1, 3 * nd, kout, s) != cudaSuccess ||
      cudaMemcpyAsync(ept2, r.e2, 3 * nd, kout, s) != cudaSuccess ||
      cudaMemcpyAsync(cnormal, r.cn, 3 * nd, kout, s) != cudaSuccess)
    return GP_ECUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return GP_ECUDA;
  return GP_OK;
}
