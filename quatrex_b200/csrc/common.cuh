// Shared device helpers of libqtxrgf: complex double arithmetic on double2,
// status codes and launch bookkeeping.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/qtx_rgf.h"

typedef double2 cplx;

__host__ __device__ __forceinline__ cplx cmk(double r, double i) { return make_double2(r, i); }
__host__ __device__ __forceinline__ cplx cadd(cplx a, cplx b) { return cmk(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ cplx csub(cplx a, cplx b) { return cmk(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ cplx cmul(cplx a, cplx b) {
  return cmk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ cplx cconj(cplx a) { return cmk(a.x, -a.y); }
__host__ __device__ __forceinline__ cplx cscale(cplx a, double s) { return cmk(a.x * s, a.y * s); }
// a + b*c
__host__ __device__ __forceinline__ cplx cfma(cplx b, cplx c, cplx a) {
  return cmk(fma(b.x, c.x, fma(-b.y, c.y, a.x)), fma(b.x, c.y, fma(b.y, c.x, a.y)));
}
// a - b*c
__host__ __device__ __forceinline__ cplx cfms(cplx b, cplx c, cplx a) {
  return cmk(fma(-b.x, c.x, fma(b.y, c.y, a.x)), fma(-b.x, c.y, fma(-b.y, c.x, a.y)));
}
// 1 / z by Smith's scaled division (R. L. Smith, CACM 5(8), 1962), which avoids
// overflow of |z|^2 for large or small components.
__host__ __device__ __forceinline__ cplx crecip(cplx z) {
  if (fabs(z.x) >= fabs(z.y)) {
    double r = z.y / z.x;
    double den = z.x + z.y * r;
    return cmk(1.0 / den, -r / den);
  } else {
    double r = z.x / z.y;
    double den = z.x * r + z.y;
    return cmk(r / den, -1.0 / den);
  }
}
// 1 / z of a pivot, Smith's scaling with one reciprocal and one quotient (the
// Gauss-Jordan inverses share it, so they agree on every pivot).
__host__ __device__ __forceinline__ cplx crecip_pivot(cplx z) {
  if (fabs(z.x) >= fabs(z.y)) {
    const double r = z.y / z.x;
    const double t = 1.0 / (z.x + z.y * r);
    return cmk(t, -r * t);
  }
  const double r = z.x / z.y;
  const double t = 1.0 / (z.x * r + z.y);
  return cmk(r * t, -t);
}
__host__ __device__ __forceinline__ double cabs1(cplx z) { return fabs(z.x) + fabs(z.y); }
// a xl + b xr for real a, b: the lesser / greater Green's function block from
// the responses to the two contact sources (G^< = f_L X_L + f_R X_R,
// G^> = (f_L - 1) X_L + (f_R - 1) X_R).  Every path that forms these blocks
// uses this one expression.
__host__ __device__ __forceinline__ cplx keldysh_mix(double a, cplx xl, double b, cplx xr) {
  return cmk(fma(a, xl.x, b * xr.x), fma(a, xl.y, b * xr.y));
}

// Per-context launch counter (host side), incremented by every launch helper.
extern thread_local int64_t* g_qtx_launch_counter;
inline void qtx_count_launch() {
  if (g_qtx_launch_counter) ++*g_qtx_launch_counter;
}

#define QTX_CUDA_TRY(expr)                                           \
  do {                                                               \
    cudaError_t _e = (expr);                                         \
    if (_e != cudaSuccess) {                                         \
      throw QtxError(QTX_E_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
    }                                                                \
  } while (0)

struct QtxError {
  qtx_status code;
  std::string msg;
  QtxError(qtx_status c, std::string m) : code(c), msg(std::move(m)) {}
};

inline void qtx_check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw QtxError(QTX_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  qtx_count_launch();
}

inline unsigned ceil_div_u(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

// Opt kernel `func` in to `bytes` of dynamic shared memory on the CURRENT
// device.  The attribute is per device, so the library remembers the largest
// value set for each (kernel, device) pair and sets it again on a device that
// has not seen it.  Thread safe; throws QTX_E_CUDA when the runtime refuses.
void qtx_opt_in_smem(const void* func, size_t bytes);

// Stream-ordered allocation from the device's default pool.  The pool keeps
// freed memory for reuse (release threshold unlimited); when a request does
// not fit, the memory the pool holds unused is returned to the driver and the
// request is tried once more (no device-wide synchronisation: only blocks
// whose stream-ordered free has completed are released).  Returns nullptr on
// failure, with the CUDA error cleared.
inline void* qtx_malloc_async(size_t bytes, cudaStream_t s) {
  void* p = nullptr;
  if (cudaMallocAsync(&p, bytes, s) == cudaSuccess) return p;
  cudaGetLastError();
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    return nullptr;
  }
  int dev = 0;
  cudaMemPool_t pool;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess ||
      cudaMemPoolTrimTo(pool, 0) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  p = nullptr;
  if (cudaMallocAsync(&p, bytes, s) == cudaSuccess) return p;
  cudaGetLastError();
  return nullptr;
}
