// DSDBSparse construction on the device: the block-sorting permutation of a
// COO pattern (the device counterpart of compute_block_sort_index,
// src/qttools/kernels/datastructure/cupy/dsdbcoo.py:234-298, which launches one
// mask kernel and one compaction per block pair).
//
// Entry q with row r and column c belongs to block (i, j), i = the block row
// containing r, j = the block column containing c (binary search over the
// block offsets in shared memory).  Its key is i * nb + j, so sorting by key
// orders the blocks row-major as upstream, and the sort is stable (CUB radix
// sort, header-only in the CUDA toolkit), which keeps the original order
// inside a block as upstream's nonzero() compaction does.  Per-block counts
// come from warp-aggregated atomics.
#include <cub/device/device_radix_sort.cuh>

#include <vector>

#include "kernels.h"

namespace {

constexpr int KEY_THREADS = 256;
constexpr int MAX_SMEM_OFFS = 4097;  // block offsets kept in shared memory (nb <= 4096)

__device__ __forceinline__ int find_block(const int64_t* offs, int nb, int64_t x) {
  // largest i with offs[i] <= x (offs[0] = 0, offs[nb] = size); -1 / nb when outside
  if (x < 0 || x >= offs[nb]) return -1;
  int lo = 0, hi = nb;  // offs[lo] <= x < offs[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (offs[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(KEY_THREADS) block_key_kernel(int64_t nnz, const int64_t* __restrict__ rows,
                                                                const int64_t* __restrict__ cols,
                                                                const int64_t* __restrict__ offs_g, int nb,
                                                                uint32_t* keys, int64_t* idx,
                                                                unsigned long long* counts, int* bad) {
  __shared__ int64_t offs_s[MAX_SMEM_OFFS];
  for (int i = threadIdx.x; i <= nb; i += blockDim.x) offs_s[i] = offs_g[i];
  __syncthreads();
  const uint32_t sentinel = (uint32_t)nb * (uint32_t)nb;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nnz; q += (int64_t)gridDim.x * blockDim.x) {
    const int bi = find_block(offs_s, nb, rows[q]);
    const int bj = find_block(offs_s, nb, cols[q]);
    uint32_t key = sentinel;
    if (bi < 0 || bj < 0) atomicOr(bad, 1);
    else key = (uint32_t)bi * (uint32_t)nb + (uint32_t)bj;
    keys[q] = key;
    idx[q] = q;
    // one atomic per distinct key of the warp
    const unsigned active = __activemask();
    const unsigned peers = __match_any_sync(active, key);
    const int leader = __ffs(peers) - 1;
    if ((int)(threadIdx.x & 31) == leader && key != sentinel) atomicAdd(&counts[key], (unsigned long long)__popc(peers));
  }
}

// A(E) = (E + i eta) S - diag(V) - Sigma(E) - H on the data rows of one
// DSDBSparse pattern (all operands in the same entry order); S = I when
// `overlap` is null (entries with row == col), the potential applies to the
// diagonal entries.  One thread per (energy, entry), 2-D grid-stride.
__global__ void assemble_system_kernel(int64_t nnz, int64_t ne, const double* __restrict__ energies, double eta,
                                       const int64_t* __restrict__ rows, const int64_t* __restrict__ cols,
                                       const cplx* __restrict__ overlap, const double* __restrict__ potential,
                                       const cplx* __restrict__ h, const cplx* __restrict__ sigma,
                                       int64_t stride_sigma, cplx* __restrict__ a, int64_t stride_a) {
  for (int64_t e = blockIdx.y; e < ne; e += gridDim.y) {
    const cplx z = cmk(energies[e], eta);
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nnz; q += (int64_t)gridDim.x * blockDim.x) {
      const bool diag = rows[q] == cols[q];
      cplx v;
      if (overlap) v = cmul(z, overlap[q]);
      else v = diag ? z : cmk(0, 0);
      if (potential && diag) v.x -= potential[rows[q]];
      v = csub(v, h[q]);
      if (sigma) v = csub(v, sigma[e * stride_sigma + q]);
      a[e * stride_a + q] = v;
    }
  }
}

struct DevMem {
  void* p = nullptr;
  cudaStream_t s = nullptr;
  DevMem(size_t bytes, cudaStream_t st) : s(st) {
    if (bytes == 0) return;
    p = qtx_malloc_async(bytes, st);
    if (!p) throw QtxError(QTX_E_NOMEM, "qtx_block_sort_index: device allocation failed");
  }
  ~DevMem() {
    if (p) cudaFreeAsync(p, s);
  }
};

}  // namespace

// Declared in include/qtx_rgf.h.  Synchronous (the per-block counts are host
// data); errors are returned as codes.
extern "C" qtx_status qtx_block_sort_index(qtx_ctx* ctx, int64_t nnz, const int64_t* rows, const int64_t* cols,
                                           int32_t num_blocks, const int32_t* block_sizes, int64_t* sort_index,
                                           int64_t* block_nnz, qtx_stream stream) {
  (void)ctx;
  if (nnz < 0 || num_blocks < 1 || num_blocks > MAX_SMEM_OFFS - 1 || !block_sizes || !block_nnz ||
      (nnz > 0 && (!rows || !cols || !sort_index)))
    return QTX_E_INVAL;
  if ((int64_t)num_blocks * num_blocks >= (int64_t)UINT32_MAX) return QTX_E_INVAL;
  try {
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int nb = num_blocks;
    const size_t nkeys = (size_t)nb * nb;
    std::vector<int64_t> offs(nb + 1, 0);
    for (int i = 0; i < nb; ++i) {
      if (block_sizes[i] < 0) return QTX_E_INVAL;
      offs[i + 1] = offs[i] + block_sizes[i];
    }
    int end_bit = 1;
    while (end_bit < 32 && (1ull << end_bit) <= nkeys) ++end_bit;  // keys up to nkeys (sentinel)
    size_t temp_bytes = 0;
    QTX_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                                 (const int64_t*)nullptr, (int64_t*)nullptr, (int64_t)nnz, 0,
                                                 end_bit, s));
    const size_t k_bytes = sizeof(uint32_t) * (size_t)std::max<int64_t>(nnz, 1);
    const size_t i_bytes = sizeof(int64_t) * (size_t)std::max<int64_t>(nnz, 1);
    // every piece starts on a 256-byte boundary: the allocation is the sum of
    // the rounded sizes
    auto rounded = [](size_t bytes) { return (bytes + 255) / 256 * 256; };
    const size_t total = 2 * rounded(k_bytes) + rounded(i_bytes) + rounded(sizeof(int64_t) * (nb + 1)) +
                         rounded(sizeof(unsigned long long) * nkeys) + rounded(sizeof(int)) + rounded(temp_bytes);
    DevMem mem(total, s);
    char* cur = static_cast<char*>(mem.p);
    char* const end = cur + total;
    auto take = [&](size_t bytes) {
      char* p = cur;
      cur += rounded(bytes);
      if (cur > end) throw QtxError(QTX_E_INVAL, "qtx_block_sort_index: work space layout");
      return p;
    };
    uint32_t* keys = reinterpret_cast<uint32_t*>(take(k_bytes));
    uint32_t* keys_sorted = reinterpret_cast<uint32_t*>(take(k_bytes));
    int64_t* idx = reinterpret_cast<int64_t*>(take(i_bytes));
    int64_t* d_offs = reinterpret_cast<int64_t*>(take(sizeof(int64_t) * (nb + 1)));
    unsigned long long* counts = reinterpret_cast<unsigned long long*>(take(sizeof(unsigned long long) * nkeys));
    int* bad = reinterpret_cast<int*>(take(sizeof(int)));
    void* temp = take(temp_bytes);
    QTX_CUDA_TRY(cudaMemcpyAsync(d_offs, offs.data(), sizeof(int64_t) * (nb + 1), cudaMemcpyHostToDevice, s));
    QTX_CUDA_TRY(cudaMemsetAsync(counts, 0, sizeof(unsigned long long) * nkeys, s));
    QTX_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(int), s));
    if (nnz > 0) {
      const unsigned grid = (unsigned)std::min<int64_t>((nnz + KEY_THREADS - 1) / KEY_THREADS, 148 * 32);
      block_key_kernel<<<grid, KEY_THREADS, 0, s>>>(nnz, rows, cols, d_offs, nb, keys, idx, counts, bad);
      qtx_check_launch("block_key_kernel");
      QTX_CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys, keys_sorted, idx, sort_index,
                                                   (int64_t)nnz, 0, end_bit, s));
    }
    std::vector<unsigned long long> h_counts(nkeys);
    int h_bad = 0;
    QTX_CUDA_TRY(cudaMemcpyAsync(h_counts.data(), counts, sizeof(unsigned long long) * nkeys,
                                 cudaMemcpyDeviceToHost, s));
    QTX_CUDA_TRY(cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    QTX_CUDA_TRY(cudaStreamSynchronize(s));
    if (h_bad) return QTX_E_INVAL;
    for (size_t k = 0; k < nkeys; ++k) block_nnz[k] = (int64_t)h_counts[k];
    return QTX_OK;
  } catch (const QtxError& e) {
    return e.code;
  }
}

extern "C" qtx_status qtx_assemble_system(qtx_ctx* ctx, int64_t nnz, int64_t num_energies, const double* energies,
                                          double eta, const int64_t* rows, const int64_t* cols, const void* overlap,
                                          const double* potential, const void* hamiltonian, const void* sigma,
                                          int64_t stride_sigma, void* a, int64_t stride_a, qtx_stream stream) {
  (void)ctx;
  if (nnz < 0 || num_energies < 0 || (nnz > 0 && num_energies > 0 && (!energies || !rows || !cols || !hamiltonian ||
                                                                        !a || stride_a < nnz)) ||
      (sigma && stride_sigma < nnz))
    return QTX_E_INVAL;
  if (nnz == 0 || num_energies == 0) return QTX_OK;
  try {
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const unsigned gx = (unsigned)std::min<int64_t>((nnz + 255) / 256, 148 * 8);
    const unsigned gy = (unsigned)std::min<int64_t>(num_energies, 65535);
    assemble_system_kernel<<<dim3(gx, gy), 256, 0, s>>>(
        nnz, num_energies, energies, eta, rows, cols, reinterpret_cast<const cplx*>(overlap), potential,
        reinterpret_cast<const cplx*>(hamiltonian), reinterpret_cast<const cplx*>(sigma), stride_sigma,
        reinterpret_cast<cplx*>(a), stride_a);
    qtx_check_launch("assemble_system_kernel");
    return QTX_OK;
  } catch (const QtxError& e) {
    return e.code;
  }
}
