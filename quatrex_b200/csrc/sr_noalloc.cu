// Sancho-Rubio surface Green's function for callers that cannot allocate
// device memory.
//
// qtx_sancho_rubio needs nine n x n x batch complex work arrays and a few
// flags; it takes them from the stream-ordered pool of its context.  Some
// callers cannot let a library allocate: an application whose allocator owns
// every device byte (a caching allocator that reserved the memory up front, so
// a library's own cudaMalloc fails or fragments the pool), a plugin host that
// forbids libraries to allocate on their own, or a latency-critical loop in
// which cudaMalloc / cudaFree would synchronise the device and stall other
// streams.  qtx_sancho_rubio_noalloc serves them: the work arrays live in one
// fixed device array of this file, NOALLOC_SCRATCH_BYTES (16 MiB) long, which
// every GPU that loads the library keeps until the process exits.  The caller
// still provides the inputs and the output.  Nothing here calls cudaMalloc,
// cudaFree or any allocating routine.
//
// Use:
//  - every call looks up the device address of the array on the current
//    device (cudaGetSymbolAddress with that device current; cheap once the
//    module is loaded, and never stale after a context teardown such as
//    cudaDeviceReset);
//  - a call cannot run inside a stream capture: each iteration copies the
//    convergence count to pageable host memory and synchronises the stream;
//  - all calls share the one array: calls that overlap on the GPU (different
//    streams, or different host threads on the same device) race; serialise
//    them on one stream;
//  - the array keeps whatever the previous call left in it; every quantity
//    that must start at zero is cleared at the start of each call.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "kernels.h"

namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(16) << 20;

// The name g_sr_scratch in host code is only a host-side stand-in, never a
// device address: kernels receive the address cudaGetSymbolAddress returns.
static __device__ __align__(256) unsigned char g_sr_scratch[NOALLOC_SCRATCH_BYTES];

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

void set_err(char* err, int32_t err_len, const char* msg) {
  if (err && err_len > 0) {
    std::strncpy(err, msg, (size_t)err_len - 1);
    err[err_len - 1] = '\0';
  }
}

}  // namespace

extern "C" qtx_status qtx_sancho_rubio_noalloc(int32_t n, int64_t batch, const void* a_ii, int64_t stride_ii,
                                               const void* a_ij, int64_t stride_ij, const void* a_ji,
                                               int64_t stride_ji, double convergence_tol, int32_t max_iterations,
                                               void* x, int32_t* iterations, qtx_stream stream, char* err,
                                               int32_t err_len) {
  if (n < 1 || batch < 1 || !a_ii || !a_ij || !a_ji || !x || max_iterations < 1) {
    set_err(err, err_len, "qtx_sancho_rubio_noalloc: bad arguments");
    return QTX_E_INVAL;
  }
  const size_t mat_bytes = align_up(sizeof(cplx) * (size_t)n * n * batch, 256);
  const size_t need = 9 * mat_bytes + align_up(sizeof(int) * (3 * (size_t)batch + 2), 256);
  if (need > NOALLOC_SCRATCH_BYTES) {
    char msg[256];
    std::snprintf(msg, sizeof(msg),
                  "qtx_sancho_rubio_noalloc: n=%d, batch=%lld needs %zu bytes of work space, above the fixed "
                  "%zu-byte array (about 9 * 16 * n^2 * batch bytes are needed); use qtx_sancho_rubio or a "
                  "smaller batch",
                  n, (long long)batch, need, NOALLOC_SCRATCH_BYTES);
    set_err(err, err_len, msg);
    return QTX_E_INVAL;
  }
  // the array's address on the current device, looked up on every call
  unsigned char* base = nullptr;
  {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_sr_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      set_err(err, err_len, "qtx_sancho_rubio_noalloc: cudaGetSymbolAddress failed (no usable current device?)");
      return QTX_E_CUDA;
    }
    base = static_cast<unsigned char*>(p);
  }

  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const cplx ONE = {1.0, 0.0}, ZERO = {0.0, 0.0}, MONE = {-1.0, 0.0};
  auto slot = [&](int q) { return MutView{reinterpret_cast<cplx*>(base + q * mat_bytes), n, (int64_t)n * n}; };
  MutView eps = slot(0), eps_s = slot(1), alpha = slot(2), beta = slot(3), inv = slot(4), t0 = slot(5),
          t1 = slot(6), t2 = slot(7), t3 = slot(8);
  int* active = reinterpret_cast<int*>(base + 9 * mat_bytes);
  int* its = active + batch;
  int* num_active = its + batch;
  int* info = num_active + 2;  // zero pivots of the decimation inverses (sticky over the iterations)
  MatView aii{reinterpret_cast<const cplx*>(a_ii), n, stride_ii};
  MatView aij{reinterpret_cast<const cplx*>(a_ij), n, stride_ij};
  MatView aji{reinterpret_cast<const cplx*>(a_ji), n, stride_ji};

  auto mm = [&](cplx alpha_, MatView a, MatView b, MutView d, MatView c = MatView{}, cplx beta_ = {0, 0},
                MatView c2 = MatView{}, cplx gamma_ = {0, 0}) {
    GemmCall g;
    g.m = n; g.n = n; g.k = n; g.batch = batch;
    g.a = a; g.b = b; g.c = c; g.beta = beta_; g.c2 = c2; g.gamma = gamma_;
    g.d = d; g.alpha = alpha_; g.active = active;
    launch_zgemm(g, s);
  };

  bool converged = false;
  try {
    // everything that must start from a known state is written here
    launch_axpby(n, n, batch, ONE, aii, ZERO, MatView{}, eps, s);
    launch_axpby(n, n, batch, ONE, aii, ZERO, MatView{}, eps_s, s);
    launch_axpby(n, n, batch, ONE, aji, ZERO, MatView{}, alpha, s);
    launch_axpby(n, n, batch, ONE, aij, ZERO, MatView{}, beta, s);
    launch_fill_int(active, batch, 1, s);
    if (cudaMemsetAsync(its, 0, sizeof(int) * (size_t)batch, s) != cudaSuccess ||
        cudaMemsetAsync(info, 0, sizeof(int) * (size_t)batch, s) != cudaSuccess)
      throw QtxError(QTX_E_CUDA, "cudaMemsetAsync failed");
    for (int it = 0; it < max_iterations; ++it) {
      launch_zinv(n, batch, eps, inv, info, active, s, /*may_allocate=*/false);
      mm(ONE, alpha, inv, t0);                               // a inv
      mm(ONE, beta, inv, t1);                                // b inv
      mm(ONE, t0, beta, t2);                                 // a inv b
      launch_axpby(n, n, batch, ONE, eps_s, MONE, t2, eps_s, s, active);
      mm(MONE, t1, alpha, eps, eps, ONE, t2, MONE);          // eps - a inv b - b inv a
      mm(ONE, t0, alpha, t3);                                // a inv a
      mm(ONE, t1, beta, t2);                                 // b inv b
      std::swap(alpha.ptr, t3.ptr);
      std::swap(beta.ptr, t2.ptr);
      if (cudaMemsetAsync(num_active, 0, sizeof(int), s) != cudaSuccess)
        throw QtxError(QTX_E_CUDA, "cudaMemsetAsync failed");
      launch_sr_norm_update(n, batch, alpha, beta, convergence_tol, active, its, num_active, s);
      int h_active = 0;  // pageable host copy: no pinned buffer is allocated
      if (cudaMemcpyAsync(&h_active, num_active, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess)
        throw QtxError(QTX_E_CUDA, "convergence readback failed");
      if (h_active == 0) {
        converged = true;
        break;
      }
    }
    launch_zinv(n, batch, eps_s, MutView{reinterpret_cast<cplx*>(x), n, (int64_t)n * n}, info, nullptr, s,
                /*may_allocate=*/false);
    if (iterations &&
        cudaMemcpyAsync(iterations, its, sizeof(int) * (size_t)batch, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
      throw QtxError(QTX_E_CUDA, "iteration count copy failed");
    // pivot status of every batch entry, into pageable host memory
    std::vector<int> h_info((size_t)batch);
    if (cudaMemcpyAsync(h_info.data(), info, sizeof(int) * (size_t)batch, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      throw QtxError(QTX_E_CUDA, "pivot status readback failed");
    for (int64_t e = 0; e < batch; ++e)
      if (h_info[(size_t)e])
        throw QtxError(QTX_E_SINGULAR, "qtx_sancho_rubio_noalloc: exactly singular decimation block (batch entry " +
                                           std::to_string(e) + ", pivot " + std::to_string(h_info[(size_t)e]) + ")");
  } catch (const QtxError& e) {
    set_err(err, err_len, e.msg.c_str());
    return e.code;
  }
  if (!converged) {
    set_err(err, err_len, "Surface Green's function did not converge.");
    return QTX_E_NOT_CONVERGED;
  }
  set_err(err, err_len, "");
  return QTX_OK;
}
