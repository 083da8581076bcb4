// Bandwidth-bound helper kernels of the RGF path: block gather/scatter
// between dense blocks and DSDBSparse data rows, Hermitian combinations,
// traces, diagonal sums, Sancho-Rubio convergence norms, A(E) assembly, the
// contact self-energy assembly and Fermi occupancies.  All are grid-stride
// loops over (batch, element) with coalesced row-major access; the transposed
// operands go through 32x32 shared-memory tiles.
#include <algorithm>

#include "kernels.h"

namespace {

constexpr int TB = 256;

inline unsigned grid_for(int64_t work) {
  int64_t g = (work + TB - 1) / TB;
  if (g > 148 * 32) g = 148 * 32;
  if (g < 1) g = 1;
  return (unsigned)g;
}

// out = s + w^H - w, square n x n; tiles of 32x32 for the transposed read
__global__ void skew_combine_kernel(int n, int64_t batch, const cplx* s, int64_t lds, int64_t ss, const cplx* w,
                                    int64_t ldw, int64_t sw, cplx* out, int64_t ldo, int64_t so) {
  __shared__ cplx tile[32][33];
  const int tiles = (n + 31) / 32;
  const int64_t total = batch * tiles * tiles;
  for (int64_t t = blockIdx.x; t < total; t += gridDim.x) {
    int64_t e = t / (tiles * tiles);
    int rem = (int)(t % (tiles * tiles));
    int tr = rem / tiles, tc = rem % tiles;
    // load w tile (tc, tr) transposed: rows tc*32.., cols tr*32..
    for (int q = threadIdx.x; q < 32 * 32; q += blockDim.x) {
      int r = q / 32, c = q % 32;
      int gr = tc * 32 + r, gc = tr * 32 + c;
      tile[r][c] = (gr < n && gc < n) ? w[e * sw + (int64_t)gr * ldw + gc] : cmk(0, 0);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < 32 * 32; q += blockDim.x) {
      int r = q / 32, c = q % 32;
      int gr = tr * 32 + r, gc = tc * 32 + c;
      if (gr < n && gc < n) {
        cplx wt = tile[c][r];  // w[gc][gr]
        cplx wv = w[e * sw + (int64_t)gr * ldw + gc];
        cplx sv = s[e * ss + (int64_t)gr * lds + gc];
        out[e * so + (int64_t)gr * ldo + gc] = cmk(sv.x + wt.x - wv.x, sv.y - wt.y - wv.y);
      }
    }
    __syncthreads();
  }
}

// X <- X - X^H in place by pairs of 32 x 32 tiles (ti <= tj) staged in shared
// memory, so both the rows and the mirrored columns are read and written
// coalesced.  The same arithmetic per element as sub_herm_kernel.
__global__ void __launch_bounds__(256)
    sub_herm_tiled_kernel(int n, int64_t batch, cplx* x, int64_t ld, int64_t sx) {
  __shared__ cplx ta[32][33], tb[32][33];
  const int nt = (n + 31) / 32;
  // triangular index -> (ti, tj), ti <= tj, row-major over the upper triangle
  const int pidx = blockIdx.x;
  int ti = 0, rest = pidx;
  while (rest >= nt - ti) {
    rest -= nt - ti;
    ++ti;
  }
  const int tj = ti + rest;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int64_t e = blockIdx.y; e < batch; e += gridDim.y) {
    cplx* base = x + e * sx;
    for (int r = ty; r < 32; r += 8) {
      const int ar = ti * 32 + r, ac = tj * 32 + tx;
      const int br = tj * 32 + r, bc = ti * 32 + tx;
      ta[r][tx] = (ar < n && ac < n) ? base[(int64_t)ar * ld + ac] : cmk(0, 0);
      tb[r][tx] = (br < n && bc < n) ? base[(int64_t)br * ld + bc] : cmk(0, 0);
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
      const int ar = ti * 32 + r, ac = tj * 32 + tx;
      if (ar < n && ac < n) {
        const cplx a = ta[r][tx], b = tb[tx][r];  // b = X[ac][ar]
        base[(int64_t)ar * ld + ac] = cmk(a.x - b.x, a.y + b.y);
      }
      if (ti != tj) {
        const int br = tj * 32 + r, bc = ti * 32 + tx;
        if (br < n && bc < n) {
          const cplx b = tb[r][tx], a = ta[tx][r];  // a = X[bc][br]
          base[(int64_t)br * ld + bc] = cmk(b.x - a.x, b.y + a.y);
        }
      }
    }
    __syncthreads();
  }
}

// x <- x - x^H in place (small blocks): each thread owns the pair (r, c), (c, r)
// with r <= c
__global__ void sub_herm_kernel(int n, int64_t batch, cplx* x, int64_t ld, int64_t sx) {
  const int64_t pairs = (int64_t)n * (n + 1) / 2;
  const int64_t total = batch * pairs;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t e = t / pairs;
    int64_t q = t % pairs;
    // invert q -> (r, c), r <= c, row-major over the upper triangle
    int r = (int)((2.0 * n + 1 - sqrt((2.0 * n + 1) * (2.0 * n + 1) - 8.0 * q)) / 2);
    while ((int64_t)r * n - (int64_t)r * (r - 1) / 2 > q) --r;
    while ((int64_t)(r + 1) * n - (int64_t)(r + 1) * r / 2 <= q) ++r;
    int c = r + (int)(q - ((int64_t)r * n - (int64_t)r * (r - 1) / 2));
    cplx* base = x + e * sx;
    cplx a = base[(int64_t)r * ld + c];
    cplx b = base[(int64_t)c * ld + r];
    // new a = a - conj(b); new b = b - conj(a)
    base[(int64_t)r * ld + c] = cmk(a.x - b.x, a.y + b.y);
    if (r != c) base[(int64_t)c * ld + r] = cmk(b.x - a.x, b.y + a.y);
    else base[(int64_t)r * ld + c] = cmk(0.0, 2.0 * a.y);
  }
}

__global__ void axpby_kernel(int rows, int cols, int64_t batch, cplx alpha, const cplx* x, int64_t ldx, int64_t sx,
                             cplx beta, const cplx* y, int64_t ldy, int64_t sy, cplx* out, int64_t ldo, int64_t so,
                             const int* active) {
  const int64_t per = (int64_t)rows * cols;
  const int64_t total = batch * per;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t e = t / per;
    if (active && !active[e]) continue;
    int q = (int)(t % per);
    int r = q / cols, c = q % cols;
    cplx v = cmul(alpha, x[e * sx + (int64_t)r * ldx + c]);
    if (y) v = cfma(beta, y[e * sy + (int64_t)r * ldy + c], v);
    out[e * so + (int64_t)r * ldo + c] = v;
  }
}

// scatter dense block -> data slice; mode 0 copy, 1 0.5(X - X^H), 2 -X^H
// (mode 2: the stored block is cols_out x rows_out = the transpose shape of x;
// `rows`/`cols` are the shape of the STORED block)
__global__ void block_scatter_kernel(int rows, int cols, int64_t batch, const cplx* x, int64_t ldx, int64_t sx,
                                     int mode, cplx* data, int64_t stride, int64_t nnz, const int32_t* index) {
  const int64_t total = batch * nnz;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t e = t / nnz;
    int64_t q = t % nnz;
    int lin = index ? index[q] : (int)q;
    int r = lin / cols, c = lin % cols;
    const cplx* xb = x + e * sx;
    cplx v;
    if (mode == 0) {
      v = xb[(int64_t)r * ldx + c];
    } else if (mode == 1) {
      cplx a = xb[(int64_t)r * ldx + c];
      cplx b = xb[(int64_t)c * ldx + r];
      v = cmk(0.5 * (a.x - b.x), 0.5 * (a.y + b.y));
    } else {
      cplx b = xb[(int64_t)c * ldx + r];
      v = cmk(-b.x, b.y);
    }
    data[e * stride + q] = v;
  }
}

__global__ void block_gather_kernel(int rows, int cols, int64_t batch, const cplx* data, int64_t stride, int64_t nnz,
                                    const int32_t* index, cplx* out, int64_t ldo, int64_t so) {
  // zero the dense block first (grid-stride), then scatter the entries
  const int64_t per = (int64_t)rows * cols;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < batch * per; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t e = t / per;
    int q = (int)(t % per);
    out[e * so + (int64_t)(q / cols) * ldo + (q % cols)] = cmk(0, 0);
  }
}
__global__ void block_gather_fill_kernel(int rows, int cols, int64_t batch, const cplx* data, int64_t stride,
                                         int64_t nnz, const int32_t* index, cplx* out, int64_t ldo, int64_t so) {
  const int64_t total = batch * nnz;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t e = t / nnz;
    int64_t q = t % nnz;
    int lin = index ? index[q] : (int)q;
    int r = lin / cols, c = lin % cols;
    out[e * so + (int64_t)r * ldo + c] = data[e * stride + q];
  }
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  return v;
}

// one CTA per batch entry: block reduction of a complex sum
__device__ cplx block_sum(cplx v) {
  __shared__ double sre[32], sim[32];
  double re = warp_sum(v.x), im = warp_sum(v.y);
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    sre[warp] = re;
    sim[warp] = im;
  }
  __syncthreads();
  cplx out = cmk(0, 0);
  if (threadIdx.x == 0) {
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      out.x += sre[w];
      out.y += sim[w];
    }
  }
  __syncthreads();
  return out;
}

__global__ void trace_product_kernel(int rows, int cols, int64_t batch, const cplx* x, int64_t ldx, int64_t sx,
                                     const cplx* y, int64_t ldy, int64_t sy, cplx scale, cplx* tr, int accumulate) {
  for (int64_t e = blockIdx.x; e < batch; e += gridDim.x) {
    cplx acc = cmk(0, 0);
    for (int q = threadIdx.x; q < rows * cols; q += blockDim.x) {
      int r = q / cols, c = q % cols;
      acc = cfma(x[e * sx + (int64_t)r * ldx + c], y[e * sy + (int64_t)c * ldy + r], acc);
    }
    cplx s = block_sum(acc);
    if (threadIdx.x == 0) {
      s = cmul(s, scale);
      tr[e] = accumulate ? cadd(tr[e], s) : s;
    }
  }
}

__global__ void trace_product_h_kernel(int rows, int cols, int64_t batch, const cplx* x, int64_t ldx, int64_t sx,
                                       const cplx* y, int64_t ldy, int64_t sy, cplx* tr) {
  for (int64_t e = blockIdx.x; e < batch; e += gridDim.x) {
    cplx acc = cmk(0, 0);
    for (int q = threadIdx.x; q < rows * cols; q += blockDim.x) {
      int r = q / cols, c = q % cols;
      acc = cfma(x[e * sx + (int64_t)r * ldx + c], cconj(y[e * sy + (int64_t)r * ldy + c]), acc);
    }
    cplx s = block_sum(acc);
    if (threadIdx.x == 0) tr[e] = s;
  }
}

// Sancho-Rubio convergence measure ||abs(alpha) + abs(beta)||_F / 2 of every
// active energy (sancho_rubio.py:76-79), one CTA of SRN_THREADS per energy,
// contiguous blocks read by linear index with four independent sums per
// thread.
constexpr int SRN_THREADS = 1024;

__device__ __forceinline__ double sr_norm_term(cplx av, cplx bv) {
  const double s = hypot(av.x, av.y) + hypot(bv.x, bv.y);
  return s * s;
}

__global__ void __launch_bounds__(SRN_THREADS)
    sr_norm_kernel(int n, int64_t batch, const cplx* a, int64_t lda, int64_t sa, const cplx* b, int64_t ldb,
                   int64_t sb, double tol, int* active, int* iterations, int* num_active) {
  const int nn = n * n;
  for (int64_t e = blockIdx.x; e < batch; e += gridDim.x) {
    if (!active[e]) continue;
    const cplx* ae = a + e * sa;
    const cplx* be = b + e * sb;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (lda == n && ldb == n) {
      int q = threadIdx.x;
      for (; q + 3 * SRN_THREADS < nn; q += 4 * SRN_THREADS) {
#pragma unroll
        for (int u = 0; u < 4; ++u) acc[u] += sr_norm_term(ae[q + u * SRN_THREADS], be[q + u * SRN_THREADS]);
      }
      for (; q < nn; q += SRN_THREADS) acc[0] += sr_norm_term(ae[q], be[q]);
    } else {
      for (int q = threadIdx.x; q < nn; q += SRN_THREADS) {
        const int r = q / n, c = q % n;
        acc[0] += sr_norm_term(ae[(int64_t)r * lda + c], be[(int64_t)r * ldb + c]);
      }
    }
    cplx s = block_sum(cmk((acc[0] + acc[1]) + (acc[2] + acc[3]), 0));
    if (threadIdx.x == 0) {
      double delta = sqrt(s.x) / 2.0;
      if (iterations) iterations[e] += 1;
      if (delta < tol) {
        active[e] = 0;
      } else {
        atomicAdd(num_active, 1);
      }
    }
  }
}

__global__ void assemble_diag_kernel(int n, int64_t batch, const cplx* h, const double* energies, double eta,
                                     cplx* out, int64_t ldo, int64_t so) {
  const int64_t per = (int64_t)n * n;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < batch * per; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t e = t / per;
    int q = (int)(t % per);
    int r = q / n, c = q % n;
    cplx hv = h[q];
    cplx v = cmk(-hv.x, -hv.y);
    if (r == c) {
      v.x += energies[e];
      v.y += eta;
    }
    out[e * so + (int64_t)r * ldo + c] = v;
  }
}

__global__ void neg_herm_kernel(int n, const cplx* h, cplx* out) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n * n; q += gridDim.x * blockDim.x) {
    int r = q / n, c = q % n;
    cplx v = h[(int64_t)c * n + r];
    out[q] = cmk(-v.x, v.y);
  }
}

__global__ void obc_lg_kernel(int n, int64_t batch, const cplx* s, int64_t lds, int64_t ss, const double* occ,
                              cplx* sl, int64_t ldl, int64_t sls, cplx* sg, int64_t ldg, int64_t sgs, cplx* gam,
                              int64_t ldgam, int64_t sgam) {
  const int64_t per = (int64_t)n * n;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < batch * per; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t e = t / per;
    int q = (int)(t % per);
    int r = q / n, c = q % n;
    cplx a = s[e * ss + (int64_t)r * lds + c];
    cplx b = s[e * ss + (int64_t)c * lds + r];
    // gamma = i (a - conj(b))
    cplx d = cmk(a.x - b.x, a.y + b.y);
    cplx g = cmk(-d.y, d.x);
    double f = occ[e];
    // i f gamma, i (f - 1) gamma
    cplx ig = cmk(-g.y, g.x);
    if (sl) sl[e * sls + (int64_t)r * ldl + c] = cscale(ig, f);
    if (sg) sg[e * sgs + (int64_t)r * ldg + c] = cscale(ig, f - 1.0);
    if (gam) gam[e * sgam + (int64_t)r * ldgam + c] = g;
  }
}

__global__ void fermi_kernel(int64_t batch, const double* energies, double mu, double kt, double* occ) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < batch; e += (int64_t)gridDim.x * blockDim.x)
    occ[e] = 1.0 / (1.0 + exp((energies[e] - mu) / kt));
}

__global__ void fill_int_kernel(int* p, int64_t count, int value) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count; t += (int64_t)gridDim.x * blockDim.x)
    p[t] = value;
}

// out = alpha op(x) + beta op(y) over (batch, rows, cols) blocks, op(z) = z or
// z^H (then z is cols x rows).  Transposed operands go through a 32 x 33
// shared-memory tile so that both the read and the write are coalesced.
template <int OPX, int OPY>
__global__ void block_combine_kernel(int rows, int cols, int64_t batch, cplx alpha, const cplx* x, int64_t ldx,
                                     int64_t sx, cplx beta, const cplx* y, int64_t ldy, int64_t sy, cplx* out,
                                     int64_t ldo, int64_t so) {
  __shared__ cplx tx[32][33];
  __shared__ cplx ty[32][33];
  const int tiles_c = (cols + 31) / 32;
  const int tr = blockIdx.x / tiles_c, tc = blockIdx.x % tiles_c;
  const int r0 = tr * 32, c0 = tc * 32;
  const int lx = threadIdx.x & 31, ly = threadIdx.x >> 5;  // 32 x 8 threads
  for (int64_t e = blockIdx.y; e < batch; e += gridDim.y) {
    const cplx* xe = x + e * sx;
    const cplx* ye = y ? y + e * sy : nullptr;
    if (OPX || OPY) {
      // stage the transposed operands: element (c, r) of the source lands at tile[r - r0][c - c0]
      for (int k = ly; k < 32; k += 8) {
        const int sr = c0 + k, sc = r0 + lx;  // source row (an output column), source column
        if (OPX) tx[lx][k] = (sr < cols && sc < rows) ? xe[(int64_t)sr * ldx + sc] : cmk(0, 0);
        if (OPY && ye) ty[lx][k] = (sr < cols && sc < rows) ? ye[(int64_t)sr * ldy + sc] : cmk(0, 0);
      }
      __syncthreads();
    }
    for (int k = ly; k < 32; k += 8) {
      const int r = r0 + k, c = c0 + lx;
      if (r < rows && c < cols) {
        const cplx vx = OPX ? cconj(tx[k][lx]) : xe[(int64_t)r * ldx + c];
        cplx v = cmul(alpha, vx);
        if (ye) {
          const cplx vy = OPY ? cconj(ty[k][lx]) : ye[(int64_t)r * ldy + c];
          v = cfma(beta, vy, v);
        }
        out[e * so + (int64_t)r * ldo + c] = v;
      }
    }
    if (OPX || OPY) __syncthreads();
  }
}

// Small status reads for the host without a copy engine: one CTA scans
// src[0, n) and stores into mapped page-locked host memory
// out[0] = 1 + index of the first nonzero entry (0: none), out[1] = that
// entry, out[2] = src[0].  (A cudaMemcpy of a status word queues behind any
// large device-to-host copy in flight on the copy engine.)
__global__ void flag_reduce_kernel(const int* src, int64_t n, int* out) {
  __shared__ unsigned long long first;
  if (threadIdx.x == 0) first = ~0ull;
  __syncthreads();
  for (int64_t t = threadIdx.x; t < n; t += blockDim.x)
    if (src[t] != 0) atomicMin(&first, (unsigned long long)t);
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile int* o = out;
    const bool any = first != ~0ull;
    o[0] = any ? (int)(first + 1) : 0;
    o[1] = any ? src[first] : 0;
    o[2] = n > 0 ? src[0] : 0;
    __threadfence_system();
  }
}

// One CTA column per block slice (blockIdx.y), CTAs stride over the data rows:
// flags[k] = 1 once any entry of slice k is nonzero (NaN counts as nonzero).
// Slice k is entries [slices[2k], slices[2k] + slices[2k + 1]) of every row.
__global__ void block_nonzero_kernel(const int64_t* slices, const cplx* data, int64_t stride, int64_t rows,
                                     int* flags) {
  const int k = blockIdx.y;
  const int64_t off = slices[2 * k], nnz = slices[2 * k + 1];
  if (off < 0 || nnz <= 0) return;
  volatile int* f = flags + k;
  for (int64_t r = blockIdx.x; r < rows; r += gridDim.x) {
    if (*f) return;
    const double2* row = reinterpret_cast<const double2*>(data + r * stride + off);
    bool any = false;
    for (int64_t q = threadIdx.x; q < nnz; q += blockDim.x) {
      const double2 v = row[q];
      any |= (v.x != 0.0) || (v.y != 0.0) || (v.x != v.x) || (v.y != v.y);
    }
    if (__syncthreads_or(any)) {
      if (threadIdx.x == 0) *f = 1;
      return;
    }
  }
}

__global__ void copy_int_kernel(int* dst, int64_t dst_stride, const int* src, int64_t src_stride, int64_t count) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count; t += (int64_t)gridDim.x * blockDim.x)
    dst[t * dst_stride] = src[t * src_stride];
}

__global__ void real_part_kernel(int64_t count, const cplx* src, double* dst) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count; t += (int64_t)gridDim.x * blockDim.x)
    dst[t] = src[t].x;
}

}  // namespace

namespace {
// abs_res[e] = ||x_ref - x||_F, rel_res[e] = abs_res[e] / ||x_ref||_F
__global__ void residual_norm_kernel(int n, int64_t batch, const cplx* xr, int64_t sr, const cplx* x, int64_t sx,
                                     double* abs_res, double* rel_res) {
  for (int64_t e = blockIdx.x; e < batch; e += gridDim.x) {
    double d2 = 0, r2 = 0;
    for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
      cplx a = xr[e * sr + q], b = x[e * sx + q];
      double dx = a.x - b.x, dy = a.y - b.y;
      d2 += dx * dx + dy * dy;
      r2 += a.x * a.x + a.y * a.y;
    }
    cplx s = block_sum(cmk(d2, r2));
    if (threadIdx.x == 0) {
      abs_res[e] = sqrt(s.x);
      rel_res[e] = s.y > 0 ? sqrt(s.x) / sqrt(s.y) : INFINITY;
    }
  }
}
}  // namespace

void launch_residual_norm(int n, int64_t batch, MatView x_ref, MatView x, double* abs_res, double* rel_res,
                          cudaStream_t stream) {
  unsigned g = (unsigned)(batch < 65535 ? batch : 65535);
  residual_norm_kernel<<<g, TB, 0, stream>>>(n, batch, x_ref.ptr, x_ref.stride, x.ptr, x.stride, abs_res, rel_res);
  qtx_check_launch("residual_norm_kernel");
}

void launch_skew_combine(int n, int64_t batch, MatView s, MatView w, MutView out, cudaStream_t stream) {
  int tiles = (n + 31) / 32;
  skew_combine_kernel<<<grid_for(batch * tiles * tiles * TB), TB, 0, stream>>>(
      n, batch, s.ptr, s.ld, s.stride, w.ptr, w.ld, w.stride, out.ptr, out.ld, out.stride);
  qtx_check_launch("skew_combine_kernel");
}

void launch_sub_herm_inplace(int n, int64_t batch, MutView x, cudaStream_t stream) {
  if (n <= 0 || batch <= 0) return;
  if (n >= 64) {
    const int nt = (n + 31) / 32;
    const unsigned pairs = (unsigned)(nt * (nt + 1) / 2);
    const unsigned gy = (unsigned)(batch < 65535 ? batch : 65535);
    sub_herm_tiled_kernel<<<dim3(pairs, gy), 256, 0, stream>>>(n, batch, x.ptr, x.ld, x.stride);
    qtx_check_launch("sub_herm_tiled_kernel");
    return;
  }
  sub_herm_kernel<<<grid_for(batch * (int64_t)n * (n + 1) / 2), TB, 0, stream>>>(n, batch, x.ptr, x.ld, x.stride);
  qtx_check_launch("sub_herm_kernel");
}

void launch_axpby(int rows, int cols, int64_t batch, cplx alpha, MatView x, cplx beta, MatView y, MutView out,
                  cudaStream_t stream, const int* active) {
  axpby_kernel<<<grid_for(batch * (int64_t)rows * cols), TB, 0, stream>>>(
      rows, cols, batch, alpha, x.ptr, x.ld, x.stride, beta, y.ptr, y.ld, y.stride, out.ptr, out.ld, out.stride,
      active);
  qtx_check_launch("axpby_kernel");
}

namespace {
__global__ void energy_shift_kernel(int64_t batch, const double* energies, double eta, cplx* shift) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < batch; e += (int64_t)gridDim.x * blockDim.x)
    shift[e] = cmk(energies[e], eta);
}
}  // namespace

void launch_energy_shift(int64_t batch, const double* energies, double eta, cplx* shift, cudaStream_t stream) {
  energy_shift_kernel<<<grid_for(batch), TB, 0, stream>>>(batch, energies, eta, shift);
  qtx_check_launch("energy_shift_kernel");
}

void launch_block_scatter(int rows, int cols, int64_t batch, MatView x, int mode, cplx* data, int64_t stride,
                          int64_t nnz, const int32_t* index, cudaStream_t stream) {
  if (nnz <= 0) return;
  block_scatter_kernel<<<grid_for(batch * nnz), TB, 0, stream>>>(rows, cols, batch, x.ptr, x.ld, x.stride, mode,
                                                                 data, stride, nnz, index);
  qtx_check_launch("block_scatter_kernel");
}

void launch_block_gather(int rows, int cols, int64_t batch, const cplx* data, int64_t stride, int64_t nnz,
                         const int32_t* index, MutView out, cudaStream_t stream) {
  block_gather_kernel<<<grid_for(batch * (int64_t)rows * cols), TB, 0, stream>>>(rows, cols, batch, data, stride,
                                                                                nnz, index, out.ptr, out.ld,
                                                                                out.stride);
  qtx_check_launch("block_gather_kernel");
  if (nnz <= 0) return;
  block_gather_fill_kernel<<<grid_for(batch * nnz), TB, 0, stream>>>(rows, cols, batch, data, stride, nnz, index,
                                                                     out.ptr, out.ld, out.stride);
  qtx_check_launch("block_gather_fill_kernel");
}

void launch_trace_product(int rows, int cols, int64_t batch, MatView x, MatView y, cplx scale, cplx* tr,
                          bool accumulate, cudaStream_t stream) {
  unsigned g = (unsigned)(batch < 65535 ? batch : 65535);
  trace_product_kernel<<<g, TB, 0, stream>>>(rows, cols, batch, x.ptr, x.ld, x.stride, y.ptr, y.ld, y.stride, scale,
                                             tr, accumulate ? 1 : 0);
  qtx_check_launch("trace_product_kernel");
}

void launch_trace_product_h(int rows, int cols, int64_t batch, MatView x, MatView y, cplx* tr, cudaStream_t stream) {
  unsigned g = (unsigned)(batch < 65535 ? batch : 65535);
  trace_product_h_kernel<<<g, TB, 0, stream>>>(rows, cols, batch, x.ptr, x.ld, x.stride, y.ptr, y.ld, y.stride, tr);
  qtx_check_launch("trace_product_h_kernel");
}


void launch_sr_norm_update(int n, int64_t batch, MatView alpha, MatView beta, double tol, int* active,
                           int* iterations, int* num_active, cudaStream_t stream) {
  unsigned g = (unsigned)(batch < 65535 ? batch : 65535);
  sr_norm_kernel<<<g, SRN_THREADS, 0, stream>>>(n, batch, alpha.ptr, alpha.ld, alpha.stride, beta.ptr, beta.ld,
                                                beta.stride, tol, active, iterations, num_active);
  qtx_check_launch("sr_norm_kernel");
}

void launch_assemble_diag(int n, int64_t batch, const cplx* h, const double* energies, double eta, MutView out,
                          cudaStream_t stream) {
  assemble_diag_kernel<<<grid_for(batch * (int64_t)n * n), TB, 0, stream>>>(n, batch, h, energies, eta, out.ptr,
                                                                            out.ld, out.stride);
  qtx_check_launch("assemble_diag_kernel");
}

void launch_neg_herm(int n, const cplx* h, cplx* out, cudaStream_t stream) {
  neg_herm_kernel<<<grid_for((int64_t)n * n), TB, 0, stream>>>(n, h, out);
  qtx_check_launch("neg_herm_kernel");
}

void launch_obc_lesser_greater(int n, int64_t batch, MatView sigma_r, const double* occ, MutView sl, MutView sg,
                               MutView gamma, cudaStream_t stream) {
  obc_lg_kernel<<<grid_for(batch * (int64_t)n * n), TB, 0, stream>>>(n, batch, sigma_r.ptr, sigma_r.ld,
                                                                     sigma_r.stride, occ, sl.ptr, sl.ld, sl.stride,
                                                                     sg.ptr, sg.ld, sg.stride, gamma.ptr, gamma.ld,
                                                                     gamma.stride);
  qtx_check_launch("obc_lg_kernel");
}

void launch_fermi(int64_t batch, const double* energies, double mu, double kt, double* occ, cudaStream_t stream) {
  fermi_kernel<<<grid_for(batch), TB, 0, stream>>>(batch, energies, mu, kt, occ);
  qtx_check_launch("fermi_kernel");
}

void launch_fill_int(int* p, int64_t count, int value, cudaStream_t stream) {
  if (count <= 0) return;
  fill_int_kernel<<<grid_for(count), TB, 0, stream>>>(p, count, value);
  qtx_check_launch("fill_int_kernel");
}

void launch_flag_reduce(const int* src, int64_t n, int* mapped_out, cudaStream_t stream) {
  flag_reduce_kernel<<<1, 256, 0, stream>>>(src, n, mapped_out);
  qtx_check_launch("flag_reduce_kernel");
}

void launch_block_combine(int rows, int cols, int64_t batch, cplx alpha, MatView x, int op_x, cplx beta, MatView y,
                          int op_y, MutView out, cudaStream_t stream) {
  if (rows <= 0 || cols <= 0 || batch <= 0) return;
  const unsigned tiles = (unsigned)(((rows + 31) / 32) * ((cols + 31) / 32));
  const dim3 grid(tiles, (unsigned)std::min<int64_t>(batch, 65535));
  const cplx* yp = y.ptr;
  if (op_x == OP_N && op_y == OP_N)
    block_combine_kernel<0, 0><<<grid, 256, 0, stream>>>(rows, cols, batch, alpha, x.ptr, x.ld, x.stride, beta, yp,
                                                         y.ld, y.stride, out.ptr, out.ld, out.stride);
  else if (op_x == OP_C && op_y == OP_N)
    block_combine_kernel<1, 0><<<grid, 256, 0, stream>>>(rows, cols, batch, alpha, x.ptr, x.ld, x.stride, beta, yp,
                                                         y.ld, y.stride, out.ptr, out.ld, out.stride);
  else if (op_x == OP_N && op_y == OP_C)
    block_combine_kernel<0, 1><<<grid, 256, 0, stream>>>(rows, cols, batch, alpha, x.ptr, x.ld, x.stride, beta, yp,
                                                         y.ld, y.stride, out.ptr, out.ld, out.stride);
  else
    block_combine_kernel<1, 1><<<grid, 256, 0, stream>>>(rows, cols, batch, alpha, x.ptr, x.ld, x.stride, beta, yp,
                                                         y.ld, y.stride, out.ptr, out.ld, out.stride);
  qtx_check_launch("block_combine_kernel");
}

void launch_block_nonzero(int num_slices, const int64_t* slices, const cplx* data, int64_t stride, int64_t rows,
                          int* flags, cudaStream_t stream) {
  if (num_slices <= 0 || rows <= 0) return;
  const unsigned gx = (unsigned)std::min<int64_t>(rows, 256);
  block_nonzero_kernel<<<dim3(gx, (unsigned)num_slices), TB, 0, stream>>>(slices, data, stride, rows, flags);
  qtx_check_launch("block_nonzero_kernel");
}

void launch_copy_int(int* dst, int64_t dst_stride, const int* src, int64_t src_stride, int64_t count,
                     cudaStream_t stream) {
  if (count <= 0) return;
  copy_int_kernel<<<grid_for(count), TB, 0, stream>>>(dst, dst_stride, src, src_stride, count);
  qtx_check_launch("copy_int_kernel");
}

void launch_real_part(int64_t count, const cplx* src, double* dst, cudaStream_t stream) {
  if (count <= 0) return;
  real_part_kernel<<<grid_for(count), TB, 0, stream>>>(count, src, dst);
  qtx_check_launch("real_part_kernel");
}

namespace {
__global__ void keldysh_combine_kernel(int n, int64_t batch, const cplx* xl, int64_t ldl, int64_t sl, const cplx* xr,
                                       int64_t ldr, int64_t sr, const double* occ_l, const double* occ_r,
                                       double sign_r, int sym, cplx* out_l, int64_t so_l, cplx* out_g, int64_t so_g) {
  const int64_t per = (int64_t)n * n;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < batch * per; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = t / per;
    const int q = (int)(t % per);
    const int r = q / n, c = q % n;
    const double fl = occ_l[e], fr = occ_r[e];
    const cplx a = xl[e * sl + (int64_t)r * ldl + c], b = xr[e * sr + (int64_t)r * ldr + c];
    const cplx yl = keldysh_mix(fl, a, sign_r * fr, b);
    const cplx yg = keldysh_mix(fl - 1.0, a, sign_r * (fr - 1.0), b);
    if (!sym) {
      if (out_l) out_l[e * so_l + q] = yl;
      if (out_g) out_g[e * so_g + q] = yg;
      continue;
    }
    const cplx at = xl[e * sl + (int64_t)c * ldl + r], bt = xr[e * sr + (int64_t)c * ldr + r];
    const cplx ylt = keldysh_mix(fl, at, sign_r * fr, bt);
    const cplx ygt = keldysh_mix(fl - 1.0, at, sign_r * (fr - 1.0), bt);
    if (out_l) out_l[e * so_l + q] = cmk(0.5 * (yl.x - ylt.x), 0.5 * (yl.y + ylt.y));
    if (out_g) out_g[e * so_g + q] = cmk(0.5 * (yg.x - ygt.x), 0.5 * (yg.y + ygt.y));
  }
}
__global__ void keldysh_density_kernel(int n, int64_t batch, const cplx* xl, int64_t ldl, int64_t sl, const cplx* xr,
                                       int64_t ldr, int64_t sr, const double* occ_l, const double* occ_r,
                                       double* density, double* hole, int64_t out_stride, int out_col) {
  for (int64_t e = blockIdx.x; e < batch; e += gridDim.x) {
    const double fl = occ_l[e], fr = occ_r[e];
    double dl = 0, dg = 0;
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
      const cplx a = xl[e * sl + (int64_t)r * ldl + r], b = xr[e * sr + (int64_t)r * ldr + r];
      dl += keldysh_mix(fl, a, fr, b).y;
      dg += keldysh_mix(fl - 1.0, a, fr - 1.0, b).y;
    }
    const cplx s = block_sum(cmk(dl, dg));
    if (threadIdx.x == 0) {
      if (density) density[e * out_stride + out_col] = s.x;
      if (hole) hole[e * out_stride + out_col] = -s.y;
    }
  }
}
}  // namespace

void launch_keldysh_combine(int n, int64_t batch, MatView xl, MatView xr, const double* occ_l, const double* occ_r,
                            double sign_r, bool sym, cplx* out_l, int64_t stride_l, cplx* out_g, int64_t stride_g,
                            cudaStream_t stream) {
  if (!out_l && !out_g) return;
  keldysh_combine_kernel<<<grid_for(batch * (int64_t)n * n), TB, 0, stream>>>(
      n, batch, xl.ptr, xl.ld, xl.stride, xr.ptr, xr.ld, xr.stride, occ_l, occ_r, sign_r, sym ? 1 : 0, out_l, stride_l,
      out_g, stride_g);
  qtx_check_launch("keldysh_combine_kernel");
}

void launch_keldysh_density(int n, int64_t batch, MatView xl, MatView xr, const double* occ_l, const double* occ_r,
                            double* density, double* hole, int64_t out_stride, int out_col, cudaStream_t stream) {
  if (!density && !hole) return;
  const unsigned g = (unsigned)(batch < 65535 ? batch : 65535);
  keldysh_density_kernel<<<g, TB, 0, stream>>>(n, batch, xl.ptr, xl.ld, xl.stride, xr.ptr, xr.ld, xr.stride, occ_l,
                                                occ_r, density, hole, out_stride, out_col);
  qtx_check_launch("keldysh_density_kernel");
}

namespace {
__global__ void block_dos_kernel(int n, int64_t batch, const cplx* g, int64_t ld, int64_t sg, double* out,
                                 int64_t out_stride, int out_col) {
  for (int64_t e = blockIdx.x; e < batch; e += gridDim.x) {
    double acc = 0;
    for (int r = threadIdx.x; r < n; r += blockDim.x) acc += g[e * sg + (int64_t)r * ld + r].y;
    const cplx s = block_sum(cmk(acc, 0));
    if (threadIdx.x == 0) out[e * out_stride + out_col] = -s.x / n;
  }
}
// One CTA of LC_THREADS per energy (one energy per SM at the usual batch):
// contiguous blocks are read by linear index, four independent elements per
// thread and step, so the reduction streams at HBM speed.
constexpr int LC_THREADS = 1024;

__device__ __forceinline__ cplx layer_current_term(double fl, double frs, cplx l, cplx r, cplx hv) {
  const cplx y = keldysh_mix(fl, l, frs, r);
  return csub(cmul(hv, cmk(-y.x, y.y)), cmul(y, cconj(hv)));
}

__global__ void __launch_bounds__(LC_THREADS)
    layer_current_kernel(int n, int64_t batch, const cplx* xl, int64_t ldl, int64_t sl, const cplx* xr,
                         int64_t ldr, int64_t sr, const double* occ_l, const double* occ_r, double sign_r,
                         const cplx* h, cplx* out, int64_t out_stride, int out_col) {
  const int nn = n * n;
  for (int64_t e = blockIdx.x; e < batch; e += gridDim.x) {
    const double fl = occ_l[e], frs = sign_r * occ_r[e];
    const cplx* le = xl + e * sl;
    const cplx* re = xr + e * sr;
    cplx acc[4] = {cmk(0, 0), cmk(0, 0), cmk(0, 0), cmk(0, 0)};
    if (ldl == n && ldr == n) {
      int q = threadIdx.x;
      for (; q + 3 * LC_THREADS < nn; q += 4 * LC_THREADS) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int qu = q + u * LC_THREADS;
          acc[u] = cadd(acc[u], layer_current_term(fl, frs, le[qu], re[qu], h[qu]));
        }
      }
      for (; q < nn; q += LC_THREADS) acc[0] = cadd(acc[0], layer_current_term(fl, frs, le[q], re[q], h[q]));
    } else {
      for (int q = threadIdx.x; q < nn; q += LC_THREADS) {
        const int r = q / n, c = q % n;
        acc[0] = cadd(acc[0], layer_current_term(fl, frs, le[(int64_t)r * ldl + c], re[(int64_t)r * ldr + c], h[q]));
      }
    }
    const cplx s = block_sum(cadd(cadd(acc[0], acc[1]), cadd(acc[2], acc[3])));
    if (threadIdx.x == 0) out[e * out_stride + out_col] = s;
  }
}
}  // namespace

void launch_block_dos(int n, int64_t batch, MatView g, double* out, int64_t out_stride, int out_col,
                      cudaStream_t stream) {
  if (!out) return;
  const unsigned grid = (unsigned)(batch < 65535 ? batch : 65535);
  block_dos_kernel<<<grid, TB, 0, stream>>>(n, batch, g.ptr, g.ld, g.stride, out, out_stride, out_col);
  qtx_check_launch("block_dos_kernel");
}

void launch_layer_current(int n, int64_t batch, MatView xl, MatView xr, const double* occ_l, const double* occ_r,
                          double sign_r, const cplx* coupling, cplx* out, int64_t out_stride, int out_col,
                          cudaStream_t stream) {
  if (!out) return;
  const unsigned grid = (unsigned)(batch < 65535 ? batch : 65535);
  layer_current_kernel<<<grid, LC_THREADS, 0, stream>>>(n, batch, xl.ptr, xl.ld, xl.stride, xr.ptr, xr.ld, xr.stride,
                                                        occ_l, occ_r, sign_r, coupling, out, out_stride, out_col);
  qtx_check_launch("layer_current_kernel");
}
