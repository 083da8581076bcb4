// Batched complex FP64 inverse: blocked in-place Gauss-Jordan elimination with
// partial (row) pivoting, one CTA per matrix.
//
// Replaces qttools.kernels.linalg.inv (src/qttools/kernels/linalg/inv.py:6-40,
// LAPACK getrf/getri or getrf/getrs on the GPU there).  Pivot choice follows
// the LAPACK izamax rule: the first row of maximal |Re| + |Im|.
//
// Algorithm (for an n x n matrix X, panel width W):
//   for each panel of columns [k0, k0 + w):
//     1. stage the n x w panel in shared memory and run unblocked in-place
//        Gauss-Jordan on it: pivot search, row swap (recorded), scale the
//        pivot row, eliminate the pivot column from every other row;
//     2. the other columns receive the same row operations at once: with the
//        composite row permutation sigma of the panel and the final panel
//        P, for every row i
//          X[i, c] <- [i not a pivot row] X[sigma(i), c]
//                     + sum_j P[i, j] X[sigma(k0 + j), c]
//        (a rank-w update, the bulk of the n^3 complex multiply-adds);
//   finally undo the row interchanges as column interchanges in reverse order.
// The matrix itself stays in global memory (L2 resident for the working set of
// one wave); the panel (n x (W+1) complex, padded against bank conflicts), one
// row slab of the update and the permutation live in shared memory.
#include "kernels.h"

namespace {

constexpr int THREADS = 256;
constexpr int CPT = 4;      // columns per thread in the rank-w update
constexpr int MAX_RPT = 8;  // rows per thread in the rank-w update

struct InvShape {
  int W;    // panel width
  int CW;   // columns per update slab
};

__host__ __device__ inline InvShape inv_shape(int n) {
  InvShape s;
  if (n <= 64) s.W = n;
  else if (n <= 256) s.W = 32;
  else s.W = 16;
  s.CW = (n <= 256) ? 32 : 16;
  return s;
}

inline size_t inv_smem_bytes(int n) {
  InvShape s = inv_shape(n);
  size_t panel = (size_t)n * (s.W + 1) * sizeof(cplx);
  size_t slab = (size_t)s.W * s.CW * sizeof(cplx);
  size_t fcol = (size_t)n * sizeof(cplx);
  size_t ints = (size_t)(2 * n) * sizeof(int);
  size_t red = 2 * (THREADS / 32) * sizeof(double) * 2;
  return panel + slab + fcol + ints + red + 64;
}

__device__ __forceinline__ void argmax_combine(double& v, int& i, double v2, int i2) {
  if (v2 > v || (v2 == v && i2 < i)) {
    v = v2;
    i = i2;
  }
}

__global__ void __launch_bounds__(THREADS, 1)
    zinv_gj_kernel(int n, int64_t batch, const cplx* __restrict__ a_base, int64_t lda, int64_t sa,
                   cplx* x_base, int64_t ldx, int64_t sx, int* info, const int* active) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const InvShape shp = inv_shape(n);
  const int W = shp.W, CW = shp.CW, LDP = W + 1;
  cplx* P = reinterpret_cast<cplx*>(smem_raw);
  cplx* R = P + (size_t)n * LDP;
  cplx* fcol = R + (size_t)W * CW;
  int* sigma = reinterpret_cast<int*>(fcol + n);
  int* perm = sigma + n;
  double* red_v = reinterpret_cast<double*>(perm + n);
  int* red_i = reinterpret_cast<int*>(red_v + THREADS / 32);
  __shared__ int s_piv;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  for (int64_t e = blockIdx.x; e < batch; e += gridDim.x) {
    if (active && !active[e]) continue;
    const cplx* A = a_base + e * sa;
    cplx* X = x_base + e * sx;
    int zero_pivot = 0;

    if (A != X || lda != ldx) {
      for (int idx = tid; idx < n * n; idx += THREADS) {
        int r = idx / n, c = idx % n;
        X[(int64_t)r * ldx + c] = A[(int64_t)r * lda + c];
      }
      __syncthreads();
    }

    for (int k0 = 0; k0 < n; k0 += W) {
      const int w = min(W, n - k0);
      for (int idx = tid; idx < n * w; idx += THREADS) {
        int r = idx / w, c = idx % w;
        P[r * LDP + c] = X[(int64_t)r * ldx + k0 + c];
      }
      for (int r = tid; r < n; r += THREADS) sigma[r] = r;
      __syncthreads();

      for (int kk = 0; kk < w; ++kk) {
        const int k = k0 + kk;
        // 1. pivot search over rows k..n-1 of panel column kk
        double bv = -1.0;
        int bi = n;
        for (int r = k + tid; r < n; r += THREADS) argmax_combine(bv, bi, cabs1(P[r * LDP + kk]), r);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          double v2 = __shfl_down_sync(0xffffffffu, bv, off);
          int i2 = __shfl_down_sync(0xffffffffu, bi, off);
          argmax_combine(bv, bi, v2, i2);
        }
        if (lane == 0) {
          red_v[warp] = bv;
          red_i[warp] = bi;
        }
        __syncthreads();
        if (tid == 0) {
          double v = red_v[0];
          int i = red_i[0];
          for (int q = 1; q < THREADS / 32; ++q) argmax_combine(v, i, red_v[q], red_i[q]);
          if (i >= n) i = k;
          s_piv = i;
          perm[k] = i;
          int t = sigma[k];
          sigma[k] = sigma[i];
          sigma[i] = t;
        }
        __syncthreads();
        const int p = s_piv;
        // 2. swap panel rows k and p
        if (p != k) {
          for (int c = tid; c < w; c += THREADS) {
            cplx t = P[k * LDP + c];
            P[k * LDP + c] = P[p * LDP + c];
            P[p * LDP + c] = t;
          }
        }
        __syncthreads();
        // 3. scale the pivot row; keep the pivot column for the elimination
        const cplx piv = P[k * LDP + kk];
        if (piv.x == 0.0 && piv.y == 0.0) zero_pivot = zero_pivot ? zero_pivot : k + 1;
        const cplx d = crecip(piv);
        for (int r = tid; r < n; r += THREADS) fcol[r] = P[r * LDP + kk];
        __syncthreads();
        for (int c = tid; c < w; c += THREADS) P[k * LDP + c] = (c == kk) ? d : cmul(P[k * LDP + c], d);
        __syncthreads();
        // 4. eliminate column kk from all other rows
        for (int idx = tid; idx < n * w; idx += THREADS) {
          int r = idx / w, c = idx % w;
          if (r == k) continue;
          cplx f = fcol[r];
          P[r * LDP + c] = (c == kk) ? cmul(cmk(-f.x, -f.y), d) : cfms(f, P[k * LDP + c], P[r * LDP + c]);
        }
        __syncthreads();
      }

      // write the finished panel back
      for (int idx = tid; idx < n * w; idx += THREADS) {
        int r = idx / w, c = idx % w;
        X[(int64_t)r * ldx + k0 + c] = P[r * LDP + c];
      }

      // rank-w update of all other columns, CW columns per slab
      const int tx = tid % (CW / CPT);
      const int ty = tid / (CW / CPT);
      const int TY = THREADS / (CW / CPT);
      for (int cs = 0; cs < n; cs += CW) {
        // (the panel columns themselves are skipped by the `ok` predicates)
        cplx y[MAX_RPT][CPT];
        // phase a: gather this thread's (permuted) rows and the pivot rows R
#pragma unroll
        for (int i = 0; i < MAX_RPT; ++i) {
          int r = ty + i * TY;
#pragma unroll
          for (int q = 0; q < CPT; ++q) {
            int c = cs + tx + q * (CW / CPT);
            bool ok = r < n && c < n && (c < k0 || c >= k0 + w);
            y[i][q] = ok ? X[(int64_t)sigma[r] * ldx + c] : cmk(0, 0);
          }
        }
        for (int idx = tid; idx < w * CW; idx += THREADS) {
          int j = idx / CW, cc = idx % CW;
          int c = cs + cc;
          bool ok = c < n && (c < k0 || c >= k0 + w);
          R[j * CW + cc] = ok ? X[(int64_t)sigma[k0 + j] * ldx + c] : cmk(0, 0);
        }
        __syncthreads();
        // phase b: X[r, c] = [r not pivot] y + sum_j P[r, j] R[j, c]
#pragma unroll
        for (int i = 0; i < MAX_RPT; ++i) {
          int r = ty + i * TY;
          if (r >= k0 && r < k0 + w) {
#pragma unroll
            for (int q = 0; q < CPT; ++q) y[i][q] = cmk(0, 0);
          }
        }
        for (int j = 0; j < w; ++j) {
          cplx rv[CPT];
#pragma unroll
          for (int q = 0; q < CPT; ++q) rv[q] = R[j * CW + tx + q * (CW / CPT)];
#pragma unroll
          for (int i = 0; i < MAX_RPT; ++i) {
            int r = ty + i * TY;
            if (r < n) {
              cplx pv = P[r * LDP + j];
#pragma unroll
              for (int q = 0; q < CPT; ++q) y[i][q] = cfma(pv, rv[q], y[i][q]);
            }
          }
        }
#pragma unroll
        for (int i = 0; i < MAX_RPT; ++i) {
          int r = ty + i * TY;
#pragma unroll
          for (int q = 0; q < CPT; ++q) {
            int c = cs + tx + q * (CW / CPT);
            bool ok = r < n && c < n && (c < k0 || c >= k0 + w);
            if (ok) X[(int64_t)r * ldx + c] = y[i][q];
          }
        }
        __syncthreads();
      }
    }

    // undo the row interchanges as column interchanges, in reverse order
    for (int c = tid; c < n; c += THREADS) sigma[c] = c;
    __syncthreads();
    if (tid == 0) {
      for (int k = n - 1; k >= 0; --k) {
        int p = perm[k];
        int t = sigma[k];
        sigma[k] = sigma[p];
        sigma[p] = t;
      }
    }
    __syncthreads();
    {
      // rows in slabs through the (now free) panel buffer
      const int rows_per_slab = max(1, (n * LDP) / n);
      for (int r0 = 0; r0 < n; r0 += rows_per_slab) {
        int nr = min(rows_per_slab, n - r0);
        for (int idx = tid; idx < nr * n; idx += THREADS) {
          int r = idx / n, c = idx % n;
          P[idx] = X[(int64_t)(r0 + r) * ldx + c];
        }
        __syncthreads();
        for (int idx = tid; idx < nr * n; idx += THREADS) {
          int r = idx / n, c = idx % n;
          X[(int64_t)(r0 + r) * ldx + c] = P[r * n + sigma[c]];
        }
        __syncthreads();
      }
    }
    if (info && tid == 0) info[e] = zero_pivot;
    __syncthreads();
  }
}

}  // namespace

void launch_zinv(int n, int64_t batch, MatView a, MutView x, int* info, const int* active, cudaStream_t stream) {
  if (n <= 0 || batch <= 0) return;
  if (n > 1024) throw QtxError(QTX_E_UNSUPPORTED, "qtx inverse: block size above 1024");
  size_t smem = inv_smem_bytes(n);
  static size_t configured = 0;
  if (smem > configured) {
    cudaFuncSetAttribute(zinv_gj_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    configured = smem;
  }
  InvShape s = inv_shape(n);
  // every row of the update must be owned: rows per thread <= MAX_RPT
  int ty = THREADS / (s.CW / CPT);
  if ((n + ty - 1) / ty > MAX_RPT) throw QtxError(QTX_E_UNSUPPORTED, "qtx inverse: block size too large");
  int grid = (int)(batch < 65535 ? batch : 65535);
  zinv_gj_kernel<<<grid, THREADS, smem, stream>>>(n, batch, a.ptr, a.ld, a.stride, x.ptr, x.ld, x.stride, info,
                                                  active);
  qtx_check_launch("zinv_gj_kernel");
}
