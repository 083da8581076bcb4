// Batched complex FP64 inverse: blocked in-place Gauss-Jordan elimination with
// partial (row) pivoting, one CTA per matrix, bulk work on the FP64 tensor path.
//
// Replaces qttools.kernels.linalg.inv (src/qttools/kernels/linalg/inv.py:6-40,
// LAPACK getrf/getri, or getrf/getrs on the GPU).  Pivot choice follows the
// LAPACK izamax rule: the first row (in the current row order) of maximal
// |Re| + |Im|.
//
// Algorithm for an n x n matrix X (a copy of A), panel width w:
//   for each panel of columns [k0, k0 + w):
//     1. stage the n x w panel in shared memory (rows in the current order of
//        X) and eliminate it column by column without moving rows: pick the
//        pivot row among the rows not yet used, eliminate the column from all
//        other rows, scale the pivot row (two barriers per column);
//     2. turn the pivot sequence into the row permutation sigma that the
//        classic row-swapping Gauss-Jordan would apply (position k0 + j takes
//        pivot row p_j, the displaced row goes to p_j's position), and record
//        each swap for the final column unscrambling;
//     3. apply the panel's row operations to every other column at once, a
//        rank-w update on DMMA (mma.sync m16n8k4 f64) tiles:
//          X[i, c] <- [i not in panel] X[sigma(i), c]
//                     + sum_j P[sigma(i), j] X[p_j, c]
//        in column slabs of CW, the k0 + j pivot rows staged in shared memory;
//   finally undo the row interchanges as column interchanges in reverse order.
// The matrix itself stays in global memory (L2 resident for a wave of
// matrices); shared memory holds the panel (n x Wp, XOR-swizzled so that both
// row-per-thread access and DMMA fragment loads are conflict-free), two slabs
// of pivot rows and the permutation arrays.
#include "kernels.h"

namespace {

constexpr int THREADS = 256;
constexpr int NWARPS = THREADS / 32;

struct InvShape {
  int w;    // panel width
  int wp;   // panel storage width (multiple of 8)
  int cw;   // columns per update slab (multiple of 32)
  int tpr;  // threads per panel row in the elimination
};

__host__ __device__ inline InvShape inv_shape(int n) {
  InvShape s;
  s.w = n <= 32 ? n : (n <= 256 ? (n <= 96 ? 16 : 32) : 16);
  s.wp = (s.w + 7) / 8 * 8;
  int row_tiles = (n + 31) / 32;
  int col_tiles = row_tiles >= NWARPS ? 1 : NWARPS / row_tiles;
  s.cw = 32 * col_tiles;
  int tpr = 1;
  while (tpr * 2 * n <= THREADS && tpr * 2 <= s.w) tpr *= 2;
  s.tpr = tpr;
  return s;
}

// complex elements of the update slabs: pivot rows and panel rows, double
// buffered (none when one panel covers the matrix)
__host__ __device__ inline int slab_elems(int n, const InvShape& s) { return s.w >= n ? 0 : 4 * s.w * (s.cw + 2); }

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool pred) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  int bytes = pred ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

inline size_t inv_smem_bytes(int n) {
  InvShape s = inv_shape(n);
  size_t panel = (size_t)n * s.wp * sizeof(cplx);
  size_t slabs = (size_t)slab_elems(n, s) * sizeof(cplx);
  size_t ints = (size_t)(3 * n + 32 + 4) * sizeof(int);
  size_t red = 2 * NWARPS * (sizeof(double) + sizeof(int) + sizeof(cplx));
  size_t pivrow = (size_t)2 * NWARPS * s.wp * sizeof(cplx);  // pivot candidates, two column parities
  return panel + slabs + ints + red + pivrow + 256;
}

// swizzled panel index: row r, column c (c < wp, wp multiple of 8)
__device__ __forceinline__ int pidx(int r, int c, int wp) {
  int sw = ((r & 1) << 2) | ((r >> 1) & 3);
  return r * wp + (c ^ sw);
}

__device__ __forceinline__ void dmma(double (&c)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

__device__ __forceinline__ void argmax_combine(double& v, int& i, double v2, int i2) {
  if (v2 > v || (v2 == v && i2 < i)) {
    v = v2;
    i = i2;
  }
}

template <int TPR, int RPT, int CPT>
__global__ void __launch_bounds__(THREADS, 1)
    zinv_gj_kernel(int n, int64_t batch, const cplx* __restrict__ a_base, int64_t lda, int64_t sa,
                   cplx* x_base, int64_t ldx, int64_t sx, int* info, const int* active) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const InvShape shp = inv_shape(n);
  const int W = shp.w, WP = shp.wp, CW = shp.cw;
  const int LDR = CW + 2;
  cplx* P = reinterpret_cast<cplx*>(smem_raw);
  cplx* Rs = P + (size_t)n * WP;                 // two slabs of W x LDR (pivot rows, panel rows)
  int* pos2row = reinterpret_cast<int*>(Rs + slab_elems(n, shp));
  int* row2pos = pos2row + n;
  int* perm = row2pos + n;                       // swap partner of each column (final unscramble)
  // doubles after the int arrays: round the offset up to 16 bytes (3n ints is
  // not a multiple of 8 bytes for odd n)
  int* pivs = perm + n;                          // pivot row of each column of the current panel
  double* red_v = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(pivs + 32) + 15) & ~uintptr_t(15));
  cplx* red_piv = reinterpret_cast<cplx*>(red_v + 2 * NWARPS);  // column-kk entry of each warp's candidate
  int* red_i = reinterpret_cast<int*>(red_piv + 2 * NWARPS);
  // per warp and column parity: the panel row of the warp's pivot candidate
  cplx* cand = reinterpret_cast<cplx*>(red_i + 2 * NWARPS + 2);
  cand = reinterpret_cast<cplx*>((reinterpret_cast<uintptr_t>(cand) + 15) & ~uintptr_t(15));

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  // elimination ownership: thread -> (rows r0 + q * rstride, columns cl + j * TPR)
  const int rstride = THREADS / TPR;
  const int r_own = tid / TPR;
  const int c_own = tid % TPR;

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
    }
    __syncthreads();

    for (int k0 = 0; k0 < n; k0 += W) {
      const int w = min(W, n - k0);
      // ---- 1. stage the panel (rows in the current order of X)
      for (int idx = tid; idx < n * w; idx += THREADS) {
        int r = idx / w, c = idx % w;
        P[pidx(r, c, WP)] = X[(int64_t)r * ldx + k0 + c];
      }
      for (int r = tid; r < n; r += THREADS) {
        pos2row[r] = r;
        row2pos[r] = r;
      }
      __syncthreads();

      // The thread's panel entries live in registers during the elimination:
      // reg[q][j] = P[r_own + q * rstride][c_own + j * TPR].  The column factor
      // of a row comes from the lane of the row's group that holds column kk;
      // the pivot row is broadcast through shared memory.
      cplx reg[RPT][CPT];
#pragma unroll
      for (int q = 0; q < RPT; ++q)
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
          const int r = r_own + q * rstride, c = c_own + j * TPR;
          reg[q][j] = (r < n && c < w) ? P[pidx(r, c, WP)] : cmk(0, 0);
        }
      const int grp0 = lane - c_own;  // first lane of this row's group (groups never straddle warps)
      // rows before k0 are the pivots of earlier panels (rows are in the new order now)
      if constexpr (CPT == 1) {
        // One column per lane: lane c_own holds column c_own of the rows
        // r_own + q * rstride; the factors of column kk come by shuffle from
        // the lane that holds it, the pivot row is one shared-memory word per
        // lane.  One barrier per column (each warp publishes its candidate's
        // row before it).
        uint32_t used_bits = 0;
#pragma unroll
        for (int q = 0; q < RPT; ++q)
          if (r_own + q * rstride < k0) used_bits |= 1u << q;
#pragma unroll 1
        for (int kk = 0; kk < w; ++kk) {
          const int k = k0 + kk;
          const int src = grp0 + kk % TPR;
          double bv = -1.0;
          int bi = n;
          if (c_own == kk % TPR) {
#pragma unroll
            for (int q = 0; q < RPT; ++q) {
              const int r = r_own + q * rstride;
              if (r < n && !((used_bits >> q) & 1u)) argmax_combine(bv, bi, cabs1(reg[q][0]), r);
            }
          }
#pragma unroll
          for (int off = 16; off > 0; off >>= 1) {
            double v2 = __shfl_xor_sync(0xffffffffu, bv, off);
            int i2 = __shfl_xor_sync(0xffffffffu, bi, off);
            argmax_combine(bv, bi, v2, i2);
          }
          const int par = kk & 1;
          cplx* my_cand = cand + (size_t)(par * NWARPS + warp) * WP;
#pragma unroll
          for (int q = 0; q < RPT; ++q)
            if (r_own + q * rstride == bi && c_own < w) my_cand[c_own] = reg[q][0];
          const int slot = par * NWARPS;
          if (lane == 0) {
            red_v[slot + warp] = bv;
            red_i[slot + warp] = bi;
          }
          __syncthreads();  // candidates of every warp visible
          double v = red_v[slot];
          int p = red_i[slot], pw = 0;
          for (int q = 1; q < NWARPS; ++q) {
            const double vq = red_v[slot + q];
            const int iq = red_i[slot + q];
            if (vq > v || (vq == v && iq < p)) {
              v = vq;
              p = iq;
              pw = q;
            }
          }
          const cplx* prow = cand + (size_t)(par * NWARPS + pw) * WP;
          const cplx piv = prow[kk];
          if (piv.x == 0.0 && piv.y == 0.0 && !zero_pivot) zero_pivot = k + 1;
          const cplx d = crecip_pivot(piv);
          if (tid == 0) pivs[kk] = p;
          const cplx pc = c_own < w ? prow[c_own] : cmk(0, 0);
          const cplx pd = cmul(pc, d);
#pragma unroll
          for (int q = 0; q < RPT; ++q) {
            // every lane takes part in the shuffle, whatever its row
            const double fx = __shfl_sync(0xffffffffu, reg[q][0].x, src);
            const double fy = __shfl_sync(0xffffffffu, reg[q][0].y, src);
            const int r = r_own + q * rstride;
            if (r >= n || c_own >= w) continue;
            if (r == p) {
              used_bits |= 1u << q;
              reg[q][0] = (c_own == kk) ? d : pd;
            } else {
              const cplx fd = cmul(cmk(fx, fy), d);
              reg[q][0] = (c_own == kk) ? cmk(-fd.x, -fd.y) : cfms(fd, pc, reg[q][0]);
            }
          }
        }
      } else {
        bool used[RPT];
#pragma unroll
        for (int q = 0; q < RPT; ++q) used[q] = r_own + q * rstride < k0;
        // One barrier per column: every warp publishes the panel row of its own
        // best candidate before the barrier, so afterwards the winner's row is
        // read directly.  Column kk of the register rows is picked by static
        // selects; with 32 register columns the loop stays rolled (one copy of
        // its body fits the instruction cache), narrower rows unroll it.
        constexpr int kKUnroll = (CPT >= 2 && CPT <= 16) ? 32 : 1;
#pragma unroll kKUnroll
        for (int kk = 0; kk < w; ++kk) {
          const int k = k0 + kk;
          // each row reads and clears its column-kk entry: the staged pivot
          // row carries 1 there, so the update below is one x - fd p for
          // every entry (-fd at column kk) and p d for the pivot row (d at kk)
          cplx colv[RPT];
#pragma unroll
          for (int q = 0; q < RPT; ++q) {
            cplx v = cmk(0, 0);
#pragma unroll
            for (int j = 0; j < CPT; ++j)
              if (c_own + j * TPR == kk) {
                v = reg[q][j];
                reg[q][j] = cmk(0, 0);
              }
            colv[q] = v;
          }
          // pivot search: the owner of (r, kk) looks at row r if it is not a pivot yet
          double bv = -1.0;
          int bi = n;
          if (c_own == kk % TPR) {
#pragma unroll
            for (int q = 0; q < RPT; ++q) {
              const int r = r_own + q * rstride;
              if (r < n && !used[q]) argmax_combine(bv, bi, cabs1(colv[q]), r);
            }
          }
          // butterfly: every lane ends with the warp's best candidate
#pragma unroll
          for (int off = 16; off > 0; off >>= 1) {
            double v2 = __shfl_xor_sync(0xffffffffu, bv, off);
            int i2 = __shfl_xor_sync(0xffffffffu, bi, off);
            argmax_combine(bv, bi, v2, i2);
          }
          // factors of this thread's rows (column kk, from the group's owner lane)
          cplx f[RPT];
#pragma unroll
          for (int q = 0; q < RPT; ++q) {
            const double fx = __shfl_sync(0xffffffffu, colv[q].x, grp0 + kk % TPR);
            const double fy = __shfl_sync(0xffffffffu, colv[q].y, grp0 + kk % TPR);
            f[q] = cmk(fx, fy);
          }
          const int par = kk & 1;
          cplx* my_cand = cand + (size_t)(par * NWARPS + warp) * WP;
          const int slot = par * NWARPS;
#pragma unroll
          for (int q = 0; q < RPT; ++q) {
            if (r_own + q * rstride == bi) {
#pragma unroll
              for (int j = 0; j < CPT; ++j) {
                const int c = c_own + j * TPR;
                if (c < w) my_cand[c] = reg[q][j];
              }
              if (c_own == kk % TPR) {
                my_cand[kk] = cmk(1, 0);
                red_piv[slot + warp] = colv[q];
              }
            }
          }
          if (lane == 0) {
            red_v[slot + warp] = bv;
            red_i[slot + warp] = bi;
          }
          __syncthreads();  // S: candidates of every warp visible
          // best over the warps, lane-parallel: every group of NWARPS lanes
          // holds all candidates (same choice as a scan in warp order)
          double v = red_v[slot + lane % NWARPS];
          int p = red_i[slot + lane % NWARPS];
#pragma unroll
          for (int off = NWARPS / 2; off > 0; off >>= 1) {
            const double v2 = __shfl_xor_sync(0xffffffffu, v, off);
            const int i2 = __shfl_xor_sync(0xffffffffu, p, off);
            argmax_combine(v, p, v2, i2);
          }
          // the global best is the best of the warp that owns row p
          const int pw = ((p % rstride) * TPR) >> 5;
          const cplx* prow = cand + (size_t)(par * NWARPS + pw) * WP;
          const cplx piv = red_piv[slot + pw];
          if (piv.x == 0.0 && piv.y == 0.0 && !zero_pivot) zero_pivot = k + 1;
          const cplx d = crecip_pivot(piv);
          if (tid == 0) pivs[kk] = p;
#pragma unroll
          for (int q = 0; q < RPT; ++q) {
            const int r = r_own + q * rstride;
            if (r >= n) continue;
            if (r == p) {
              used[q] = true;
#pragma unroll
              for (int j = 0; j < CPT; ++j) {
                const int c = c_own + j * TPR;
                if (c < w) reg[q][j] = cmul(prow[c], d);
              }
            } else {
              const cplx fd = cmul(f[q], d);
#pragma unroll
              for (int j = 0; j < CPT; ++j) {
                const int c = c_own + j * TPR;
                if (c < w) reg[q][j] = cfms(fd, prow[c], reg[q][j]);
              }
            }
          }
        }
      }
      // classic row-swap semantics of the panel's pivots: position k0 + kk
      // receives row pivs[kk], the displaced row goes to the pivot's position
      if (tid == 0) {
        for (int kk = 0; kk < w; ++kk) {
          const int k = k0 + kk, p = pivs[kk];
          const int qpos = row2pos[p];
          const int rk = pos2row[k];
          pos2row[k] = p;
          row2pos[p] = k;
          pos2row[qpos] = rk;
          row2pos[rk] = qpos;
          perm[k] = qpos;
        }
      }
      // panel back to shared memory for the update
#pragma unroll
      for (int q = 0; q < RPT; ++q)
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
          const int r = r_own + q * rstride, c = c_own + j * TPR;
          if (r < n && c < w) P[pidx(r, c, WP)] = reg[q][j];
        }
      __syncthreads();

      // ---- 3. rank-w update of the other columns, slabs of CW columns.
      // Output position i reads X[sigma(i)], and sigma(i) is either i itself or
      // a row of [k0, k0 + w) (a row displaced by a pivot swap); the pivot rows
      // X[p_j] and the rows of [k0, k0 + w) of the slab are staged in shared
      // memory first, so afterwards every thread reads and writes only its own
      // positions of X and one barrier per slab suffices.
      const int row_tiles = (n + 31) / 32;
      const int col_tiles = CW / 32;
      const int nslab = (n + CW - 1) / CW;
      // slabs with at least one column outside the panel, staged double buffered
      auto next_slab = [&](int from) {
        int sl = from;
        while (sl < nslab && (sl * CW >= k0 && min(sl * CW + CW, n) <= k0 + w)) ++sl;
        return sl;
      };
      auto stage = [&](int sl, int buf) {
        cplx* Rb = Rs + (size_t)buf * 2 * W * LDR;
        cplx* Db = Rb + (size_t)W * LDR;
        const int cs = sl * CW;
        for (int idx = tid; idx < w * CW; idx += THREADS) {
          int j = idx / CW, cc = idx % CW;
          int c = cs + cc;
          bool ok = c < n;
          cp_async16(&Rb[j * LDR + cc], ok ? &X[(int64_t)pos2row[k0 + j] * ldx + c] : X, ok);
          cp_async16(&Db[j * LDR + cc], ok ? &X[(int64_t)(k0 + j) * ldx + c] : X, ok);
        }
        cp_async_commit();
      };
      int slab = next_slab(0);
      int buf = 0;
      if (slab < nslab) stage(slab, 0);
      while (slab < nslab) {
        const int c0 = slab * CW;
        const int nxt = next_slab(slab + 1);
        // the other buffer was last read before the barrier that ended the
        // previous slab, so it can be refilled now
        if (nxt < nslab) stage(nxt, buf ^ 1);
        else cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        cplx* R = Rs + (size_t)buf * 2 * W * LDR;  // pivot rows p_j      (w x CW)
        cplx* D = R + (size_t)W * LDR;             // rows k0 + j         (w x CW)
        for (int tile = warp; tile < row_tiles * col_tiles; tile += NWARPS) {
          const int rt = tile / col_tiles, ct = tile % col_tiles;
          const int row0 = rt * 32, col0 = ct * 32;
          double acc_re[2][4][4], acc_im[2][4][4];
#pragma unroll
          for (int mi = 0; mi < 2; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
              for (int q = 0; q < 4; ++q) {
                int i = row0 + mi * 16 + g + ((q >> 1) << 3);
                int cc = col0 + ni * 8 + 2 * t + (q & 1);
                int c = c0 + cc;
                cplx y = cmk(0, 0);
                if (i < n && c < n && !(i >= k0 && i < k0 + w)) {
                  int src = pos2row[i];
                  y = (src == i) ? X[(int64_t)i * ldx + c] : D[(src - k0) * LDR + cc];
                }
                acc_re[mi][ni][q] = y.x;
                acc_im[mi][ni][q] = y.y;
              }
          int prow_idx[2][2];
#pragma unroll
          for (int mi = 0; mi < 2; ++mi) {
            int i0 = row0 + mi * 16 + g, i1 = i0 + 8;
            prow_idx[mi][0] = i0 < n ? pos2row[i0] : -1;
            prow_idx[mi][1] = i1 < n ? pos2row[i1] : -1;
          }
          for (int kk = 0; kk < w; kk += 4) {
            const int kc = kk + t;
            cplx af[2][2], bf[4];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
              for (int h = 0; h < 2; ++h) {
                int pr = prow_idx[mi][h];
                af[mi][h] = (pr >= 0 && kc < w) ? P[pidx(pr, kc, WP)] : cmk(0, 0);
              }
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) bf[ni] = (kc < w) ? R[kc * LDR + col0 + ni * 8 + g] : cmk(0, 0);
            // real parts first, then imaginary: 16 independent accumulators
            // separate the two products that feed the same accumulator
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
              for (int ni = 0; ni < 4; ++ni) {
                dmma(acc_re[mi][ni], af[mi][0].x, af[mi][1].x, bf[ni].x);
                dmma(acc_im[mi][ni], af[mi][0].x, af[mi][1].x, bf[ni].y);
              }
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
              for (int ni = 0; ni < 4; ++ni) {
                dmma(acc_re[mi][ni], -af[mi][0].y, -af[mi][1].y, bf[ni].y);
                dmma(acc_im[mi][ni], af[mi][0].y, af[mi][1].y, bf[ni].x);
              }
          }
#pragma unroll
          for (int mi = 0; mi < 2; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
              for (int q = 0; q < 4; ++q) {
                int i = row0 + mi * 16 + g + ((q >> 1) << 3);
                int c = c0 + col0 + ni * 8 + 2 * t + (q & 1);
                if (i < n && c < n && !(c >= k0 && c < k0 + w))
                  X[(int64_t)i * ldx + c] = cmk(acc_re[mi][ni][q], acc_im[mi][ni][q]);
              }
        }
        __syncthreads();
        slab = nxt;
        buf ^= 1;
      }
      cp_async_wait<0>();
      // ---- panel columns: final panel values in the new row order
      for (int idx = tid; idx < n * w; idx += THREADS) {
        int i = idx / w, c = idx % w;
        X[(int64_t)i * ldx + k0 + c] = P[pidx(pos2row[i], c, WP)];
      }
      // rows are now in the new order: the pivot rows so far sit at positions < k0 + w
      __syncthreads();
    }

    // ---- undo the row interchanges as column interchanges, in reverse order
    int* colsrc = pos2row;  // reuse: column permutation
    for (int c = tid; c < n; c += THREADS) colsrc[c] = c;
    __syncthreads();
    if (tid == 0) {
      for (int k = n - 1; k >= 0; --k) {
        int q = perm[k];
        int tmp = colsrc[k];
        colsrc[k] = colsrc[q];
        colsrc[q] = tmp;
      }
    }
    __syncthreads();
    {
      const int rows_per_slab = max(1, (int)((size_t)n * WP / n));
      for (int r0 = 0; r0 < n; r0 += rows_per_slab) {
        int nr = min(rows_per_slab, n - r0);
        for (int idx = tid; idx < nr * n; idx += THREADS) {
          int r = idx / n, c = idx % n;
          P[idx] = X[(int64_t)(r0 + r) * ldx + c];
        }
        __syncthreads();
        for (int idx = tid; idx < nr * n; idx += THREADS) {
          int r = idx / n, c = idx % n;
          X[(int64_t)(r0 + r) * ldx + c] = P[r * n + colsrc[c]];
        }
        __syncthreads();
      }
    }
    // sticky: callers zero info once and read it after several launches
    if (info && tid == 0 && zero_pivot) info[e] = zero_pivot;
    __syncthreads();
  }
}

}  // namespace

namespace {

template <int TPR, int RPT, int CPT>
void launch_inv_t(int n, int64_t batch, MatView a, MutView x, int* info, const int* active, size_t smem,
                  cudaStream_t stream) {
  qtx_opt_in_smem((const void*)zinv_gj_kernel<TPR, RPT, CPT>, smem);
  int grid = (int)(batch < 65535 ? batch : 65535);
  zinv_gj_kernel<TPR, RPT, CPT><<<grid, THREADS, smem, stream>>>(n, batch, a.ptr, a.ld, a.stride, x.ptr, x.ld,
                                                                  x.stride, info, active);
}

}  // namespace

void launch_zinv(int n, int64_t batch, MatView a, MutView x, int* info, const int* active, cudaStream_t stream) {
  if (n <= 0 || batch <= 0) return;
  if (n > 512) throw QtxError(QTX_E_UNSUPPORTED, "qtx inverse: block size above 512");
  const size_t smem = inv_smem_bytes(n);
  const InvShape s = inv_shape(n);
  // every panel row / column must be owned by the elimination mapping
  const int rpt = (n + (THREADS / s.tpr) - 1) / (THREADS / s.tpr);
  const int cpt = (s.w + s.tpr - 1) / s.tpr;
  // (threads per row, rows per thread) -> instance with enough register columns
  if (s.tpr == 1 && rpt == 1 && cpt <= 32) launch_inv_t<1, 1, 32>(n, batch, a, x, info, active, smem, stream);
  else if (s.tpr == 1 && rpt == 2 && cpt <= 16) launch_inv_t<1, 2, 16>(n, batch, a, x, info, active, smem, stream);
  else if (s.tpr == 2 && rpt == 1 && cpt <= 16) launch_inv_t<2, 1, 16>(n, batch, a, x, info, active, smem, stream);
  else if (s.tpr == 4 && rpt == 1 && cpt <= 4) launch_inv_t<4, 1, 4>(n, batch, a, x, info, active, smem, stream);
  else if (s.tpr == 8 && rpt == 1 && cpt <= 4) launch_inv_t<8, 1, 4>(n, batch, a, x, info, active, smem, stream);
  else if (s.tpr == 16 && rpt == 1 && cpt <= 1) launch_inv_t<16, 1, 1>(n, batch, a, x, info, active, smem, stream);
  else throw QtxError(QTX_E_UNSUPPORTED, "qtx inverse: block size outside the supported shapes");
  qtx_check_launch("zinv_gj_kernel");
}
