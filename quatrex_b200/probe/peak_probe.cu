// FP64 peak probe (measurement tool, not part of libqtxrgf.so): the
// issue-rate ceiling of the FP64 tensor path (DMMA, mma.sync m8n8k4 f64) and of
// scalar DFMA on this GPU, used as the roofline denominator of the FP64
// kernels (the measured peaks of the GPU pool cover HBM and bf16 only).  Each
// warp issues independent accumulator chains with no memory traffic; the
// result is flops / elapsed time over the whole grid.  Built into its own
// libqtxprobe.so by quatrex_b200/build.py and called only by
// `python -m quatrex_b200.kernel_bench fp64peak`.
#include <cuda_runtime.h>
#include <stdint.h>

#define QTX_OK 0
#define QTX_E_INVAL 1
#define QTX_E_CUDA 6
typedef int qtx_status;

namespace {

__global__ void dfma_probe_kernel(double* out, int iters) {
  double a0 = threadIdx.x * 1e-3, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6,
         a7 = a0 + 7;
  const double b = 0.999999, c = 1e-9;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      a0 = fma(a0, b, c); a1 = fma(a1, b, c); a2 = fma(a2, b, c); a3 = fma(a3, b, c);
      a4 = fma(a4, b, c); a5 = fma(a5, b, c); a6 = fma(a6, b, c); a7 = fma(a7, b, c);
    }
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
}

__global__ void dmma_probe_kernel(double* out, int iters) {
  double a0 = threadIdx.x * 1e-3, b0 = 0.5;
  double c[8][2] = {};
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                   : "+d"(c[u][0]), "+d"(c[u][1])
                   : "d"(a0), "d"(b0));
    }
  }
  double s = 0;
  for (int u = 0; u < 8; ++u) s += c[u][0] + c[u][1];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

// kind 0: DMMA m8n8k4 f64; kind 1: scalar DFMA.  Returns TFLOP/s in *tflops.
extern "C" qtx_status qtx_probe_fp64_peak(int32_t kind, double* tflops) {
  if (!tflops || kind < 0 || kind > 1) return QTX_E_INVAL;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return QTX_E_CUDA;
  const int threads = 512, blocks = sms * 4, iters = 20000;
  double* out = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  qtx_status st = QTX_OK;
  if (cudaMalloc(&out, sizeof(double) * blocks * threads) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
      cudaEventCreate(&e1) != cudaSuccess) {
    st = QTX_E_CUDA;
  } else {
    float ms = 0;
    for (int rep = 0; rep < 2; ++rep) {
      cudaEventRecord(e0);
      if (kind == 0) dmma_probe_kernel<<<blocks, threads>>>(out, iters / 4);
      else dfma_probe_kernel<<<blocks, threads>>>(out, iters);
      cudaEventRecord(e1);
      cudaEventSynchronize(e1);
      cudaEventElapsedTime(&ms, e0, e1);
    }
    double warps = (double)blocks * threads / 32;
    double flops = kind == 0 ? 2.0 * 8 * 8 * 4 * 8 * (iters / 4) * warps : 2.0 * 64 * iters * (double)blocks * threads;
    *tflops = flops / ms / 1e9;
    if (cudaGetLastError() != cudaSuccess) st = QTX_E_CUDA;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (out) cudaFree(out);
  return st;
}
