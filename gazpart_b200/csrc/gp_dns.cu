// gp_dns.cu -- the pseudo-spectral fluid solver of the reference's DNS mode, on the device.
//
// ADV_FLUID (adv_fluid.f90:1-271) advances the periodic velocity field one step:
//   1. u -> û = FFT(u) * FACTOR                                  (:47-60)
//   2. RHS1 = NONLINEAR_TERMS(u, û): the projection of FFT(u x ω) onto the
//      divergence-free plane, ω = IFFT(i k x û) (nonlinear_terms.f90:81-160)
//   3. û_{n+1}^* = (û + dt/2 RHS1) e^{-ν k² dt};  û = (û + dt RHS1) e^{-ν k² dt}   (:95-110)
//   4. u = IFFT(û); RHS2 = NONLINEAR_TERMS(u, û)                  (:117-140)
//   5. û = û_{n+1}^* + dt/2 RHS2; PROJ_DIVFREE; û *= FILTER        (:145-170, proj_divfree.f90)
//   6. u = IFFT(û)                                                (:178-187)
// The transforms are cuFFT's (D2Z forward, Z2D backward, both unnormalised as P3DFFT's
// are), the three components of a vector field in one batched call; every step between
// them is one element-wise kernel per stage, in FP64 and without FMA contraction, in the
// reference's evaluation order.  A step makes 7 batched calls (21 transforms).  Wavenumbers follow
// meshing.f90:96-140 (KX = (I-1) KFIRST on the half-spectrum, KY and KZ signed), and the
// aliasing filter meshing.f90:144-180 (sharp or smooth, RTRUNC), computed per mode.
// The stochastic forcing of STEADY runs (ADV_FORCING, ADD_FORCING3) is not part of it.
#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>

#include "../../include/gazpart_gpu.h"
#include "gp_types.h"

struct gp_dns {
  int nx = 0, ny = 0, nz = 0, nxh = 0;
  double kfirst = 0, klast = 0, visc = 0, dtime = 0, factor = 0, rtrunc = 0;
  int aliascontrol = 0;
  cudaStream_t stream = nullptr;
  cufftHandle fwd = 0, bwd = 0;   // three transforms per call
  bool plans = false;
  // each a block of three components back to back: physical [3][z][y][x], spectral
  // [3][z][y][x/2+1]
  double *u = nullptr;            // velocity
  double *t = nullptr;            // vorticity, then u x ω
  cufftDoubleComplex *uh = nullptr, *unp1 = nullptr, *w = nullptr, *tmp = nullptr;
  size_t np = 0, nh = 0;          // points of one component
};

namespace gp {
namespace {

constexpr double kZero = 1.0e-33;       // ZERO, mod_dns_dim.f90:136
constexpr double kInfinity = 1.0e33;   // INFINITY, mod_dns_dim.f90:137

#define GP_DTRY(x)          \
  do {                      \
    const int rc__ = (x);   \
    if (rc__) return rc__;  \
  } while (0)

struct Spec {
  int nxh, ny, nz;
  double kfirst;
};

__device__ __forceinline__ void wavenumbers(const Spec &s, int64_t e, double &kx, double &ky, double &kz) {
  const int i = (int)(e % s.nxh), j = (int)((e / s.nxh) % s.ny), k = (int)(e / ((int64_t)s.nxh * s.ny));
  kx = (double)i * s.kfirst;                                     // (I-1)*KFIRST
  ky = (j + 1 <= s.ny / 2 + 1) ? (double)j * s.kfirst : (double)(j - s.ny) * s.kfirst;
  kz = (k + 1 <= s.nz / 2 + 1) ? (double)k * s.kfirst : (double)(k - s.nz) * s.kfirst;
}

// (ICMPL * a) * r: i a = (-Im a, Re a), then each part times the real r
__device__ __forceinline__ cufftDoubleComplex cmul_i_real(cufftDoubleComplex a, double r) {
  return make_cuDoubleComplex(-a.y * r, a.x * r);
}

// VORTX..Z = i k x û (nonlinear_terms.f90:81-92); the outputs are copies the backward
// transform may overwrite.
__global__ void k_vorticity_hat(Spec s, const cufftDoubleComplex *__restrict__ in, cufftDoubleComplex *out) {
  const int64_t n = (int64_t)s.nxh * s.ny * s.nz;
  const cufftDoubleComplex *uh = in, *vh = in + n, *wh = in + 2 * n;
  cufftDoubleComplex *ox = out, *oy = out + n, *oz = out + 2 * n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    double kx, ky, kz;
    wavenumbers(s, e, kx, ky, kz);
    const cufftDoubleComplex U = uh[e], V = vh[e], W = wh[e];
    const cufftDoubleComplex a = cmul_i_real(W, ky), b = cmul_i_real(V, kz);
    const cufftDoubleComplex c = cmul_i_real(U, kz), d = cmul_i_real(W, kx);
    const cufftDoubleComplex f = cmul_i_real(V, kx), g = cmul_i_real(U, ky);
    ox[e] = make_cuDoubleComplex(a.x - b.x, a.y - b.y);
    oy[e] = make_cuDoubleComplex(c.x - d.x, c.y - d.y);
    oz[e] = make_cuDoubleComplex(f.x - g.x, f.y - g.y);
  }
}

// TX..TZ = u x ζ in physical space (nonlinear_terms.f90:105-113), in place over ζ.
__global__ void k_cross(int64_t n, const double *__restrict__ vel, double *z) {
  const double *u = vel, *v = vel + n, *w = vel + 2 * n;
  double *zx = z, *zy = z + n, *zz = z + 2 * n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const double a = zx[e], b = zy[e], c = zz[e];
    zx[e] = v[e] * c - w[e] * b;
    zy[e] = w[e] * a - u[e] * c;
    zz[e] = u[e] * b - v[e] * a;
  }
}

__device__ __forceinline__ cufftDoubleComplex scale(cufftDoubleComplex a, double r) {
  return make_cuDoubleComplex(a.x * r, a.y * r);
}
__device__ __forceinline__ cufftDoubleComplex add(cufftDoubleComplex a, cufftDoubleComplex b) {
  return make_cuDoubleComplex(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ cufftDoubleComplex sub(cufftDoubleComplex a, cufftDoubleComplex b) {
  return make_cuDoubleComplex(a.x - b.x, a.y - b.y);
}

// The projected nonlinear term of nonlinear_terms.f90:119-160 from the transformed
// u x ζ (scaled by FACTOR first, :114-117), added to the RHS that ADV_FLUID clears to
// cmplx(ZERO, ZERO) = (1e-33, 1e-33) (adv_fluid.f90:73-75, :122-124).
__device__ __forceinline__ void rhs_of(double kx, double ky, double kz, double factor, cufftDoubleComplex tx,
                                      cufftDoubleComplex ty, cufftDoubleComplex tz, cufftDoubleComplex r[3]) {
  tx = scale(tx, factor);
  ty = scale(ty, factor);
  tz = scale(tz, factor);
  double k2 = kx * kx + ky * ky + kz * kz;
  if (k2 <= kZero) k2 = kInfinity;
  const cufftDoubleComplex zero = make_cuDoubleComplex(kZero, kZero);
  r[0] = sub(sub(add(zero, scale(tx, (ky * ky + kz * kz) / k2)), scale(ty, kx * ky / k2)), scale(tz, kx * kz / k2));
  r[1] = sub(add(sub(zero, scale(tx, ky * kx / k2)), scale(ty, (kx * kx + kz * kz) / k2)), scale(tz, ky * kz / k2));
  r[2] = add(sub(sub(zero, scale(tx, kz * kx / k2)), scale(ty, kz * ky / k2)), scale(tz, (kx * kx + ky * ky) / k2));
}

// adv_fluid.f90:95-110: the first stage with the integrating factor.
__global__ void k_stage1(Spec s, double factor, double visc, double dtime, cufftDoubleComplex *hat,
                         cufftDoubleComplex *np1, const cufftDoubleComplex *__restrict__ t3) {
  const int64_t n = (int64_t)s.nxh * s.ny * s.nz;
  cufftDoubleComplex *uh = hat, *vh = hat + n, *wh = hat + 2 * n;
  cufftDoubleComplex *unp1 = np1, *vnp1 = np1 + n, *wnp1 = np1 + 2 * n;
  const cufftDoubleComplex *tx = t3, *ty = t3 + n, *tz = t3 + 2 * n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    double kx, ky, kz;
    wavenumbers(s, e, kx, ky, kz);
    cufftDoubleComplex r[3];
    rhs_of(kx, ky, kz, factor, tx[e], ty[e], tz[e], r);
    const double kappa2 = kx * kx + ky * ky + kz * kz;
    const double ef = exp(-visc * kappa2 * dtime);
    cufftDoubleComplex *out_np1[3] = {unp1, vnp1, wnp1};
    cufftDoubleComplex *io[3] = {uh, vh, wh};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const cufftDoubleComplex a = io[c][e];
      out_np1[c][e] = scale(add(a, scale(r[c], dtime / 2)), ef);
      io[c][e] = scale(add(a, scale(r[c], dtime)), ef);
    }
  }
}

// adv_fluid.f90:145-170 with PROJ_DIVFREE (proj_divfree.f90:28-44) and the aliasing
// filter (meshing.f90:144-180) applied per mode.
__global__ void k_stage2(Spec s, double factor, double dtime, double klast, int aliascontrol, double rtrunc,
                         double ppi, cufftDoubleComplex *hat, const cufftDoubleComplex *__restrict__ np1,
                         const cufftDoubleComplex *__restrict__ t3) {
  const int64_t n = (int64_t)s.nxh * s.ny * s.nz;
  cufftDoubleComplex *uh = hat, *vh = hat + n, *wh = hat + 2 * n;
  const cufftDoubleComplex *unp1 = np1, *vnp1 = np1 + n, *wnp1 = np1 + 2 * n;
  const cufftDoubleComplex *tx = t3, *ty = t3 + n, *tz = t3 + 2 * n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    double kx, ky, kz;
    wavenumbers(s, e, kx, ky, kz);
    cufftDoubleComplex r[3];
    rhs_of(kx, ky, kz, factor, tx[e], ty[e], tz[e], r);
    cufftDoubleComplex U = add(unp1[e], scale(r[0], dtime / 2));
    cufftDoubleComplex V = add(vnp1[e], scale(r[1], dtime / 2));
    cufftDoubleComplex W = add(wnp1[e], scale(r[2], dtime / 2));
    double k2 = kx * kx + ky * ky + kz * kz;
    if (k2 <= kZero) k2 = kInfinity;
    const cufftDoubleComplex divc = add(add(scale(U, kx), scale(V, ky)), scale(W, kz));
    U = sub(U, scale(divc, kx / k2));
    V = sub(V, scale(divc, ky / k2));
    W = sub(W, scale(divc, kz / k2));
    const double qx = kx / klast, qy = ky / klast, qz = kz / klast;
    const double k2scl = qx * qx + qy * qy + qz * qz;
    double filt = 1.0;
    if (aliascontrol == 1) {
      if (k2scl > rtrunc * rtrunc) filt = 0.0;
    } else if (aliascontrol == 2) {
      if (k2scl > rtrunc * rtrunc && k2scl <= 1.0) {
        const double cc = cos((ppi / 2.0) * (sqrt(k2scl) - rtrunc) / (1.0 - rtrunc));
        const double c2 = cc * cc;
        filt = c2 * c2;
      } else if (k2scl > 1.0) {
        filt = 0.0;
      }
    }
    uh[e] = scale(U, filt);
    vh[e] = scale(V, filt);
    wh[e] = scale(W, filt);
  }
}

__global__ void k_scale_spec(int64_t n, double factor, cufftDoubleComplex *a) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
    a[e] = scale(a[e], factor);
}

int grid_of(int64_t n) { return (int)std::min<int64_t>((n + 255) / 256, 148 * 16); }

// NONLINEAR_TERMS: leaves FFT(u x ζ) (unscaled) in d->w.
int nonlinear(gp_dns *d, const Spec &s) {
  const int64_t nh = (int64_t)d->nh, np = (int64_t)d->np;
  k_vorticity_hat<<<grid_of(nh), 256, 0, d->stream>>>(s, d->uh, d->w);
  if (cufftExecZ2D(d->bwd, d->w, d->t) != CUFFT_SUCCESS) return GP_ECUDA;
  k_cross<<<grid_of(np), 256, 0, d->stream>>>(np, d->u, d->t);
  if (cufftExecD2Z(d->fwd, d->t, d->w) != CUFFT_SUCCESS) return GP_ECUDA;
  return cudaGetLastError() == cudaSuccess ? GP_OK : GP_ECUDA;
}

template <typename T>
int alloc(T **p, size_t count) {
  return cudaMalloc(reinterpret_cast<void **>(p), count * sizeof(T)) == cudaSuccess ? GP_OK : GP_ENOMEM;
}

}  // namespace
}  // namespace gp

extern "C" {

int gp_dns_create(const gp_params *p, int32_t aliascontrol, double rtrunc, gp_dns **out) {
  using namespace gp;
  if (!p || !out) return GP_EBADARG;
  *out = nullptr;
  if (p->nx < 4 || p->ny < 4 || p->nz < 4 || (p->nx % 2) || (p->ny % 2) || (p->nz % 2)) return GP_EBADARG;
  if (!(p->lx > 0 && p->visc > 0 && p->dtime > 0) || aliascontrol < 0 || aliascontrol > 2) return GP_EBADARG;
  if (aliascontrol > 0 && !(rtrunc > 0.0 && rtrunc < 1.0)) return GP_EBADARG;
  gp_dns *d = new gp_dns;
  d->nx = p->nx; d->ny = p->ny; d->nz = p->nz; d->nxh = p->nx / 2 + 1;
  const double ppi = 4.0 * std::atan(1.0);
  d->kfirst = 2.0 * ppi / p->lx;             // KFIRST = TWOPI/LXMAX   (init_run.f90:128)
  d->klast = ppi / (p->lx / p->nx);          // KLAST = PPI/(LXMAX/NX)  (init_run.f90:129)
  d->visc = p->visc;
  d->dtime = p->dtime;
  d->factor = 1.0 / (double)((int64_t)p->nx * p->ny * p->nz);   // FACTOR = 1/NGLOB (main.f90:213)
  d->aliascontrol = aliascontrol;
  d->rtrunc = rtrunc;
  d->nh = (size_t)d->nxh * d->ny * d->nz;
  d->np = (size_t)d->nx * d->ny * d->nz;
  int rc = cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking) == cudaSuccess ? GP_OK : GP_ECUDA;
  if (!rc) rc = alloc(&d->u, 3 * d->np);
  if (!rc) rc = alloc(&d->t, 3 * d->np);
  if (!rc) rc = alloc(&d->uh, 3 * d->nh);
  if (!rc) rc = alloc(&d->unp1, 3 * d->nh);
  if (!rc) rc = alloc(&d->w, 3 * d->nh);
  if (!rc) rc = alloc(&d->tmp, 3 * d->nh);
  if (!rc) {
    long long dims[3] = {d->nz, d->ny, d->nx};
    size_t ws = 0;
    // three components back to back: the basic layout with batch 3 (64-bit sizes)
    if (cufftCreate(&d->fwd) != CUFFT_SUCCESS || cufftCreate(&d->bwd) != CUFFT_SUCCESS) {
      rc = GP_ECUDA;
    } else {
      d->plans = true;
      if (cufftMakePlanMany64(d->fwd, 3, dims, nullptr, 1, (long long)d->np, nullptr, 1, (long long)d->nh, CUFFT_D2Z,
                              3, &ws) != CUFFT_SUCCESS ||
          cufftMakePlanMany64(d->bwd, 3, dims, nullptr, 1, (long long)d->nh, nullptr, 1, (long long)d->np, CUFFT_Z2D,
                              3, &ws) != CUFFT_SUCCESS ||
          cufftSetStream(d->fwd, d->stream) != CUFFT_SUCCESS || cufftSetStream(d->bwd, d->stream) != CUFFT_SUCCESS)
        rc = GP_ECUDA;
    }
  }
  if (!rc && cudaMemsetAsync(d->u, 0, 3 * d->np * sizeof(double), d->stream) != cudaSuccess) rc = GP_ECUDA;
  if (!rc && cudaStreamSynchronize(d->stream) != cudaSuccess) rc = GP_ECUDA;
  if (rc) {
    gp_dns_destroy(d);
    return rc;
  }
  *out = d;
  return GP_OK;
}

int gp_dns_destroy(gp_dns *d) {
  if (!d) return GP_OK;
  if (d->stream) cudaStreamSynchronize(d->stream);
  if (d->plans) {
    cufftDestroy(d->fwd);
    cufftDestroy(d->bwd);
  }
  cudaFree(d->u); cudaFree(d->t); cudaFree(d->uh); cudaFree(d->unp1); cudaFree(d->w); cudaFree(d->tmp);
  if (d->stream) cudaStreamDestroy(d->stream);
  delete d;
  return GP_OK;
}

int gp_dns_set_velocity(gp_dns *d, const double *u, const double *v, const double *w, int32_t on_device) {
  if (!d || !u || !v || !w) return GP_EBADARG;
  const double *src[3] = {u, v, w};
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  for (int c = 0; c < 3; ++c)
    if (cudaMemcpyAsync(d->u + c * d->np, src[c], d->np * sizeof(double), kind, d->stream) != cudaSuccess)
      return GP_ECUDA;
  return cudaStreamSynchronize(d->stream) == cudaSuccess ? GP_OK : GP_ECUDA;
}

int gp_dns_get_velocity(gp_dns *d, double *u, double *v, double *w, int32_t on_device) {
  if (!d || !u || !v || !w) return GP_EBADARG;
  double *dst[3] = {u, v, w};
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  for (int c = 0; c < 3; ++c)
    if (cudaMemcpyAsync(dst[c], d->u + c * d->np, d->np * sizeof(double), kind, d->stream) != cudaSuccess)
      return GP_ECUDA;
  return cudaStreamSynchronize(d->stream) == cudaSuccess ? GP_OK : GP_ECUDA;
}

int gp_adv_fluid(gp_dns *d, int32_t /*ncycle*/) {
  using namespace gp;
  if (!d) return GP_EBADARG;
  const Spec s = {d->nxh, d->ny, d->nz, d->kfirst};
  const int64_t n3 = 3 * (int64_t)d->nh;
  const int g = grid_of((int64_t)d->nh);
  // 1. û = FFT(u) * FACTOR (the forward transform leaves u as it is)
  if (cufftExecD2Z(d->fwd, d->u, d->uh) != CUFFT_SUCCESS) return GP_ECUDA;
  k_scale_spec<<<grid_of(n3), 256, 0, d->stream>>>(n3, d->factor, d->uh);
  // 2-3. first stage
  int rc = nonlinear(d, s);
  if (rc) return rc;
  k_stage1<<<g, 256, 0, d->stream>>>(s, d->factor, d->visc, d->dtime, d->uh, d->unp1, d->w);
  // 4. the predictor in physical space (from a copy: the backward transform overwrites
  //    its input, and û is still needed), then the second nonlinear term
  if (cudaMemcpyAsync(d->tmp, d->uh, n3 * sizeof(cufftDoubleComplex), cudaMemcpyDeviceToDevice, d->stream) !=
      cudaSuccess)
    return GP_ECUDA;
  if (cufftExecZ2D(d->bwd, d->tmp, d->u) != CUFFT_SUCCESS) return GP_ECUDA;
  rc = nonlinear(d, s);
  if (rc) return rc;
  // 5. corrector, projection, filter
  k_stage2<<<g, 256, 0, d->stream>>>(s, d->factor, d->dtime, d->klast, d->aliascontrol, d->rtrunc,
                                     4.0 * std::atan(1.0), d->uh, d->unp1, d->w);
  // 6. back to physical space (û is not needed after this)
  if (cufftExecZ2D(d->bwd, d->uh, d->u) != CUFFT_SUCCESS) return GP_ECUDA;
  if (cudaGetLastError() != cudaSuccess) return GP_ECUDA;
  return cudaStreamSynchronize(d->stream) == cudaSuccess ? GP_OK : GP_ECUDA;
}

// Spectral vorticity of the current velocity into d->t (three components).
static int vorticity_to_t(gp_dns *d) {
  using namespace gp;
  const Spec s = {d->nxh, d->ny, d->nz, d->kfirst};
  const int64_t n3 = 3 * (int64_t)d->nh;
  if (cufftExecD2Z(d->fwd, d->u, d->w) != CUFFT_SUCCESS) return GP_ECUDA;
  k_scale_spec<<<grid_of(n3), 256, 0, d->stream>>>(n3, d->factor, d->w);
  k_vorticity_hat<<<grid_of((int64_t)d->nh), 256, 0, d->stream>>>(s, d->w, d->unp1);
  if (cufftExecZ2D(d->bwd, d->unp1, d->t) != CUFFT_SUCCESS) return GP_ECUDA;
  return cudaGetLastError() == cudaSuccess ? GP_OK : GP_ECUDA;
}

int gp_dns_vorticity(gp_dns *d, double *ox, double *oy, double *oz, int32_t on_device) {
  if (!d || !ox || !oy || !oz) return GP_EBADARG;
  const int rc = vorticity_to_t(d);
  if (rc) return rc;
  double *dst[3] = {ox, oy, oz};
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  for (int c = 0; c < 3; ++c)
    if (cudaMemcpyAsync(dst[c], d->t + c * d->np, d->np * sizeof(double), kind, d->stream) != cudaSuccess)
      return GP_ECUDA;
  return cudaStreamSynchronize(d->stream) == cudaSuccess ? GP_OK : GP_ECUDA;
}

int gp_dns_couple(gp_dns *d, gp_ctx *ctx, int32_t field, int32_t with_vorticity) {
  if (!d || !ctx) return GP_EBADARG;
  int32_t dims[3];
  const int rs = gp_field_shape(ctx, field, dims);
  if (rs) return rs;
  if (dims[0] != d->nx || dims[1] != d->ny || dims[2] != d->nz) return GP_EBADARG;   // other meshes
  if (cudaStreamSynchronize(d->stream) != cudaSuccess) return GP_ECUDA;
  // FLUIDCOMM (main.f90:499-505): the velocity's y and z ghosts are periodic copies
  for (int c = 0; c < 3; ++c) {
    const int rc = gp_set_field_slot(ctx, field, c, d->u + c * d->np, GP_LAYOUT_INTERIOR, GP_GHOST_PERIODIC, 1);
    if (rc) return rc;
  }
  if (with_vorticity) {
    // vorticity of the current field, with zero ghosts as the reference's arrays have
    int rc = vorticity_to_t(d);
    if (!rc && cudaStreamSynchronize(d->stream) != cudaSuccess) rc = GP_ECUDA;
    for (int c = 0; c < 3 && !rc; ++c)
      rc = gp_set_field_slot(ctx, field, 3 + c, d->t + c * d->np, GP_LAYOUT_INTERIOR, GP_GHOST_ZERO, 1);
    if (rc) return rc;
  }
  return GP_OK;
}

}  // extern "C"
