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
//     1. stage the n x w panel (rows in the current order of X) into the
//        threads' registers through shared memory and eliminate it column by
//        column without moving rows: pick the pivot row among the rows not
//        yet used, eliminate the column from all other rows, scale the pivot
//        row (one barrier per column: every warp publishes its candidate row
//        before it);
//     2. turn the pivot sequence into the row permutation sigma that the
//        classic row-swapping Gauss-Jordan would apply (position k0 + j takes
//        pivot row p_j, the displaced row goes to p_j's position), and record
//        each swap for the final column unscrambling;
//     3. apply the panel's row operations to every other column at once, a
//        rank-w update on DMMA (mma.sync m16n8k4 f64) tiles:
//          X[i, c] <- [i not in panel] X[sigma(i), c]
//                     + sum_j P[sigma(i), j] X[p_j, c]
//        in column slabs of CW, the k0 + j pivot rows staged in shared memory
//        (for small batches the updates of one panel run as a separate launch
//        spread over the GPU, the split path below);
//   finally undo the row interchanges as column interchanges in reverse order.
// The matrix itself stays in global memory (L2 resident for a wave of
// matrices); shared memory holds the panel (n x Wp, XOR-swizzled so that both
// row-per-thread access and DMMA fragment loads are conflict-free), two slabs
// of pivot rows and the permutation arrays.
#include <algorithm>
#include <cstdlib>

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

// Two adjacent complex elements in one 32-byte access.  The caller guarantees
// 32-byte alignment: pair_access_ok() for the matrix and an even column.
__device__ __forceinline__ void ld_pair(const cplx* p, cplx& a, cplx& b) {
  asm volatile("ld.global.v4.f64 {%0,%1,%2,%3}, [%4];\n"
               : "=d"(a.x), "=d"(a.y), "=d"(b.x), "=d"(b.y)
               : "l"(p));
}
__device__ __forceinline__ void st_pair(cplx* p, cplx a, cplx b) {
  asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};\n" ::"l"(p), "d"(a.x), "d"(a.y), "d"(b.x), "d"(b.y)
               : "memory");
}
// Element (i, c) of X with c even starts on a 32-byte boundary, and the pair
// (c, c + 1) lies on one side of every even column boundary (n, panel edges
// k0 and k0 + w, which are even when n is).
__device__ __forceinline__ bool pair_access_ok(const cplx* X, int64_t ldx, int n) {
  return (reinterpret_cast<uintptr_t>(X) & 31) == 0 && (ldx & 1) == 0 && (n & 1) == 0;
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

// Shared-memory arrays of one matrix's elimination (see zinv_gj_kernel).
struct GjSmem {
  cplx* P;
  int* pos2row;
  int* row2pos;
  int* perm;
  int* pivs;
  double* red_v;
  cplx* red_piv;
  int* red_i;
  cplx* cand;
};

__device__ inline GjSmem gj_smem_layout(unsigned char* base, int n, int wp, int slab) {
  GjSmem s;
  s.P = reinterpret_cast<cplx*>(base);
  cplx* Rs = s.P + (size_t)n * wp;
  s.pos2row = reinterpret_cast<int*>(Rs + slab);
  s.row2pos = s.pos2row + n;
  s.perm = s.row2pos + n;  // swap partner of each column (final unscramble)
  // doubles after the int arrays: round the offset up to 16 bytes (3n ints is
  // not a multiple of 8 bytes for odd n)
  s.pivs = s.perm + n;  // pivot row of each column of the current panel
  s.red_v = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(s.pivs + 32) + 15) & ~uintptr_t(15));
  s.red_piv = reinterpret_cast<cplx*>(s.red_v + 2 * NWARPS);  // column-kk entry of each warp's candidate
  s.red_i = reinterpret_cast<int*>(s.red_piv + 2 * NWARPS);
  // per warp and column parity: the panel row of the warp's pivot candidate
  s.cand = reinterpret_cast<cplx*>(s.red_i + 2 * NWARPS + 2);
  s.cand = reinterpret_cast<cplx*>((reinterpret_cast<uintptr_t>(s.cand) + 15) & ~uintptr_t(15));
  return s;
}

// Steps 1 and 2 for the panel [k0, k0 + w) of X (rows in the current order):
// eliminate it in shared memory / registers, turn its pivots into the row
// permutation sigma (pos2row / row2pos, relative to the current order) and
// the swaps perm[k0 .. k0 + w), and leave the eliminated panel in P (rows in
// the current order).  Ends with a CTA barrier.
template <int TPR, int RPT, int CPT, int ROT>
__device__ __forceinline__ void gj_panel(int n, int k0, int w, int WP, const cplx* X, int64_t ldx, const GjSmem& sm,
                                         int& zero_pivot) {
  cplx* P = sm.P;
  int* pos2row = sm.pos2row;
  int* row2pos = sm.row2pos;
  int* perm = sm.perm;
  int* pivs = sm.pivs;
  double* red_v = sm.red_v;
  cplx* red_piv = sm.red_piv;
  int* red_i = sm.red_i;
  cplx* cand = sm.cand;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // elimination ownership: thread -> (rows r0 + q * rstride, columns cl + j * TPR)
  const int rstride = THREADS / TPR;
  const int r_own = tid / TPR;
  const int c_own = tid % TPR;
    // ---- 1. stage the panel (rows in the current order of X), every
    // element in flight at once (asynchronous copies)
    for (int idx = tid; idx < n * w; idx += THREADS) {
      int r = idx / w, c = idx % w;
      cp_async16(&P[pidx(r, c, WP)], &X[(int64_t)r * ldx + k0 + c], true);
    }
    cp_async_commit();
    for (int r = tid; r < n; r += THREADS) {
      pos2row[r] = r;
      row2pos[r] = r;
    }
    cp_async_wait<0>();
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
    bool rotated = false;
    if constexpr (TPR == 1 && RPT == 1 && CPT == 32) {
      if constexpr (ROT == 1) {
        // Register rotation: at step kk, reg[0][j] holds panel column
        // (kk + j) mod 32, so the step's column is always reg[0][0] (no
        // selects over the row) and every update is unpredicated (columns
        // at or beyond w stay zero: the published pivot rows carry zeros
        // there).  The same pivots and the same update of every non-pivot
        // row as the generic loop.
        rotated = true;
        bool used = r_own < k0;
        auto rotate = [&]() {
          const cplx t0 = reg[0][0];
#pragma unroll
          for (int j = 0; j < 31; ++j) reg[0][j] = reg[0][j + 1];
          reg[0][31] = t0;
        };
#pragma unroll 1
        for (int kk = 0; kk < w; ++kk) {
          const int k = k0 + kk;
          const cplx colv = reg[0][0];
          reg[0][0] = cmk(0, 0);
          double bv = -1.0;
          int bi = n;
          if (r_own < n && !used) {
            bv = cabs1(colv);
            bi = r_own;
          }
#pragma unroll
          for (int off = 16; off > 0; off >>= 1) {
            double v2 = __shfl_xor_sync(0xffffffffu, bv, off);
            int i2 = __shfl_xor_sync(0xffffffffu, bi, off);
            argmax_combine(bv, bi, v2, i2);
          }
          const int par = kk & 1;
          cplx* my_cand = cand + (size_t)(par * NWARPS + warp) * WP;
          const int slot = par * NWARPS;
          if (r_own == bi) {
#pragma unroll
            for (int j = 0; j < 32; ++j) my_cand[j] = reg[0][j];
            my_cand[0] = cmk(1, 0);
            red_piv[slot + warp] = colv;
          }
          if (lane == 0) {
            red_v[slot + warp] = bv;
            red_i[slot + warp] = bi;
          }
          __syncthreads();  // candidates of every warp visible
          double v = red_v[slot + lane % NWARPS];
          int p = red_i[slot + lane % NWARPS];
#pragma unroll
          for (int off = NWARPS / 2; off > 0; off >>= 1) {
            const double v2 = __shfl_xor_sync(0xffffffffu, v, off);
            const int i2 = __shfl_xor_sync(0xffffffffu, p, off);
            argmax_combine(v, p, v2, i2);
          }
          const int pw = p >> 5;  // one row per thread: row p lives in warp p / 32
          const cplx* prow = cand + (size_t)(par * NWARPS + pw) * WP;
          const cplx piv = red_piv[slot + pw];
          if (piv.x == 0.0 && piv.y == 0.0 && !zero_pivot) zero_pivot = k + 1;
          const cplx d = crecip_pivot(piv);
          if (tid == 0) pivs[kk] = p;
          if (r_own < n) {
            // the pivot row as 0 - (-d) p: one update formula for every
            // row, so the warp holding the pivot row does not run two
            // branches while the others wait at the next barrier
            const bool is_p = r_own == p;
            used = used || is_p;
            const cplx fd = is_p ? cmk(-d.x, -d.y) : cmul(colv, d);
            if (is_p) {
#pragma unroll
              for (int j = 0; j < 32; ++j) reg[0][j] = cmk(0, 0);
            }
#pragma unroll
            for (int j = 0; j < 32; ++j) reg[0][j] = cfms(fd, prow[j], reg[0][j]);
          }
          rotate();
        }
        for (int extra = w; extra < 32; ++extra) rotate();  // natural column order again
      }
    }
    if (rotated) {
    } else if constexpr (CPT == 1) {
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
}

template <int TPR, int RPT, int CPT, int ROT>
__global__ void __launch_bounds__(THREADS, 1)
    zinv_gj_kernel(int n, int64_t batch, const cplx* __restrict__ a_base, int64_t lda, int64_t sa,
                   cplx* x_base, int64_t ldx, int64_t sx, int* info, const int* active) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const InvShape shp = inv_shape(n);
  const int W = shp.w, WP = shp.wp, CW = shp.cw;
  const int LDR = CW + 2;
  const GjSmem sm = gj_smem_layout(smem_raw, n, WP, slab_elems(n, shp));
  cplx* P = sm.P;
  cplx* Rs = P + (size_t)n * WP;  // two slabs of W x LDR (pivot rows, panel rows)
  int* pos2row = sm.pos2row;
  int* perm = sm.perm;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;

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
      gj_panel<TPR, RPT, CPT, ROT>(n, k0, w, WP, X, ldx, sm, zero_pivot);

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
      const int ntiles = row_tiles * col_tiles;
      // Accumulator start values of a tile: output position i starts from
      // X[sigma(i)].  Rows with sigma(i) == i load straight from X under one
      // predicate each (no branch between global and shared memory), so the
      // 32 loads of a thread are in flight together; the few rows displaced
      // by a pivot swap are then patched from the staged rows D.
      auto load_own = [&](int tile, int c0, double (&are)[2][4][4], double (&aim)[2][4][4]) {
        const int row0 = (tile / col_tiles) * 32, col0 = (tile % col_tiles) * 32;
        bool own[2][2];
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int i = row0 + mi * 16 + g + 8 * h;
            own[mi][h] = i < n && !(i >= k0 && i < k0 + w) && pos2row[i] == i;
          }
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
          for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int i = row0 + mi * 16 + g + ((q >> 1) << 3);
              const int c = c0 + col0 + ni * 8 + 2 * t + (q & 1);
              are[mi][ni][q] = 0.0;
              aim[mi][ni][q] = 0.0;
              if (own[mi][q >> 1] && c < n) {
                const cplx y = X[(int64_t)i * ldx + c];
                are[mi][ni][q] = y.x;
                aim[mi][ni][q] = y.y;
              }
            }
      };
      auto patch_displaced = [&](int tile, int c0, const cplx* D, double (&are)[2][4][4],
                                 double (&aim)[2][4][4]) {
        const int row0 = (tile / col_tiles) * 32, col0 = (tile % col_tiles) * 32;
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int i = row0 + mi * 16 + g + 8 * h;
            if (i < n && !(i >= k0 && i < k0 + w)) {
              const int src = pos2row[i];
              if (src != i) {
#pragma unroll
                for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                  for (int q2 = 0; q2 < 2; ++q2) {
                    const int cc = col0 + ni * 8 + 2 * t + q2;
                    if (c0 + cc < n) {
                      const cplx y = D[(src - k0) * LDR + cc];
                      are[mi][ni][2 * h + q2] = y.x;
                      aim[mi][ni][2 * h + q2] = y.y;
                    }
                  }
              }
            }
          }
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
        for (int tile = warp; tile < ntiles; tile += NWARPS) {
          const int rt = tile / col_tiles, ct = tile % col_tiles;
          const int row0 = rt * 32, col0 = ct * 32;
          double acc_re[2][4][4], acc_im[2][4][4];
          load_own(tile, c0, acc_re, acc_im);
          patch_displaced(tile, c0, D, acc_re, acc_im);
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

// ---------------------------------------------------------------------------
// Split path for batches smaller than the GPU: the elimination and update of
// zinv_gj_kernel, but every panel is two launches -- one CTA per matrix
// eliminates the panel, then (matrix x 32-column slab x 128-row group) CTAs
// apply its rank-w update -- so the updates of a few matrices spread over the
// whole GPU (the column chain of the elimination stays one CTA per matrix).
// Per matrix the panel launch leaves in global scratch the eliminated panel
// P (n x W, rows in the order before the panel's permutation), sigma
// (pos2row) and the column swaps; a row-copy launch adds the pivot rows
// R = X[sigma(k0 + j)] and the panel-position rows D = X[k0 + j] (n columns
// each); the update CTAs read R and D from the scratch, so no CTA reads a row
// of X that another CTA of the same launch writes.

struct SplitScratch {
  cplx* p;      // batch x n x W
  cplx* r;      // batch x W x n
  cplx* d;      // batch x W x n
  int* sigma;   // batch x n
  int* perm;    // batch x n
};

template <int TPR, int RPT, int CPT, int ROT>
__global__ void __launch_bounds__(THREADS, 1)
    zinv_split_panel_kernel(int n, int64_t batch, const cplx* __restrict__ a_base, int64_t lda, int64_t sa,
                            cplx* x_base, int64_t ldx, int64_t sx, int k0, SplitScratch sc, int* info,
                            const int* active) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const InvShape shp = inv_shape(n);
  const int W = shp.w, WP = shp.wp;
  const GjSmem sm = gj_smem_layout(smem_raw, n, WP, 0);
  const int tid = threadIdx.x;
  const int w = min(W, n - k0);
  for (int64_t e = blockIdx.x; e < batch; e += gridDim.x) {
    if (active && !active[e]) continue;
    cplx* X = x_base + e * sx;
    if (k0 == 0) {
      const cplx* A = a_base + e * sa;
      if (A != X || lda != ldx) {
        for (int idx = tid; idx < n * n; idx += THREADS) {
          int r = idx / n, c = idx % n;
          X[(int64_t)r * ldx + c] = A[(int64_t)r * lda + c];
        }
      }
      __syncthreads();
    }
    int zero_pivot = 0;
    gj_panel<TPR, RPT, CPT, ROT>(n, k0, w, WP, X, ldx, sm, zero_pivot);
    cplx* pe = sc.p + e * (int64_t)n * W;
    for (int idx = tid; idx < n * w; idx += THREADS) {
      const int r = idx / w, c = idx % w;
      pe[(int64_t)r * W + c] = sm.P[pidx(r, c, WP)];
    }
    for (int r = tid; r < n; r += THREADS) sc.sigma[e * n + r] = sm.pos2row[r];
    for (int kk = tid; kk < w; kk += THREADS) sc.perm[e * n + k0 + kk] = sm.perm[k0 + kk];
    __syncthreads();  // sigma and the panel copied before the panel columns change
    for (int idx = tid; idx < n * w; idx += THREADS) {
      const int i = idx / w, c = idx % w;
      X[(int64_t)i * ldx + k0 + c] = sm.P[pidx(sm.pos2row[i], c, WP)];
    }
    // the first exact zero pivot of the matrix (earlier panels win)
    if (info && tid == 0 && zero_pivot && info[e] == 0) info[e] = zero_pivot;
    __syncthreads();
  }
}

// The pivot rows R = X[sigma(k0 + j)] and the panel-position rows
// D = X[k0 + j] of every matrix, copied before the update moves them (one
// CTA per row and matrix; the panel columns of X may already hold their final
// values, the update does not read them from these copies).
__global__ void __launch_bounds__(256)
    zinv_split_rows_kernel(int n, int64_t batch, const cplx* x_base, int64_t ldx, int64_t sx, int k0, int W,
                           SplitScratch sc, const int* active) {
  const int j = blockIdx.x;
  for (int64_t e = blockIdx.y; e < batch; e += gridDim.y) {
    if (active && !active[e]) continue;
    const cplx* X = x_base + e * sx;
    const int src = sc.sigma[e * n + k0 + j];
    cplx* re = sc.r + (e * (int64_t)W + j) * n;
    cplx* de = sc.d + (e * (int64_t)W + j) * n;
    for (int c = threadIdx.x; c < n; c += blockDim.x) {
      re[c] = X[(int64_t)src * ldx + c];
      de[c] = X[(int64_t)(k0 + j) * ldx + c];
    }
  }
}

constexpr int SPLIT_ROWS = 128;     // output rows per update CTA
constexpr int SPLIT_THREADS = 128;  // four warps, one 32 x 32 tile each
constexpr int SPLIT_CW = 32;        // columns per update CTA
constexpr int SPLIT_LDR = SPLIT_CW + 2;

inline size_t split_update_smem(int W) {
  return (size_t)SPLIT_ROWS * 32 * sizeof(cplx) + (size_t)2 * W * SPLIT_LDR * sizeof(cplx) +
         (size_t)SPLIT_ROWS * sizeof(int) + 64;
}

__global__ void __launch_bounds__(SPLIT_THREADS, 2)
    zinv_split_update_kernel(int n, int64_t batch, cplx* x_base, int64_t ldx, int64_t sx, int k0, int w, int W,
                             SplitScratch sc, const int* active) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx* Prow = reinterpret_cast<cplx*>(smem_raw);  // P rows of the CTA's outputs, swizzled, 32 columns
  cplx* R = Prow + SPLIT_ROWS * 32;                 // w x SPLIT_LDR
  cplx* D = R + W * SPLIT_LDR;                      // w x SPLIT_LDR
  int* srow = reinterpret_cast<int*>(D + W * SPLIT_LDR);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int ngroups = (n + SPLIT_ROWS - 1) / SPLIT_ROWS;
  const int slab = blockIdx.x / ngroups, grp = blockIdx.x % ngroups;
  const int c0 = slab * SPLIT_CW, r0 = grp * SPLIT_ROWS;
  // a slab inside the panel has nothing to update
  if (c0 >= k0 && min(c0 + SPLIT_CW, n) <= k0 + w) return;
  for (int64_t e = blockIdx.y; e < batch; e += gridDim.y) {
    if (active && !active[e]) continue;
    cplx* X = x_base + e * sx;
    const bool pairs = pair_access_ok(X, ldx, n);
    const int* sig = sc.sigma + e * n;
    const cplx* pe = sc.p + e * (int64_t)n * W;
    const cplx* re = sc.r + e * (int64_t)W * n;
    const cplx* de = sc.d + e * (int64_t)W * n;
    for (int li = tid; li < SPLIT_ROWS; li += SPLIT_THREADS) srow[li] = r0 + li < n ? sig[r0 + li] : -1;
    __syncthreads();
    for (int idx = tid; idx < SPLIT_ROWS * 32; idx += SPLIT_THREADS) {
      const int li = idx >> 5, c = idx & 31;
      const int src = srow[li];
      const bool ok = src >= 0 && c < w;
      cp_async16(&Prow[pidx(li, c, 32)], ok ? &pe[(int64_t)src * W + c] : pe, ok);
    }
    for (int idx = tid; idx < w * SPLIT_CW; idx += SPLIT_THREADS) {
      const int j = idx / SPLIT_CW, cc = idx % SPLIT_CW;
      const bool ok = c0 + cc < n;
      cp_async16(&R[j * SPLIT_LDR + cc], ok ? &re[(int64_t)j * n + c0 + cc] : re, ok);
      cp_async16(&D[j * SPLIT_LDR + cc], ok ? &de[(int64_t)j * n + c0 + cc] : de, ok);
    }
    cp_async_commit();
    // one 32 x 32 tile per warp: rows r0 + 32 warp .., columns c0 ..
    // Output position i starts from row sigma(i): itself, or a row of
    // [k0, k0 + w) displaced by a pivot swap; positions inside the panel start
    // from zero.  The rows that start from themselves load while the staged
    // copies are in flight (only this CTA writes these positions of X); the
    // displaced rows are patched from the staged D after the barrier.
    const int lrow0 = warp * 32;
    const bool has_tile = r0 + lrow0 < n;
    double acc_re[2][4][4], acc_im[2][4][4];
    int src_of[2][2];  // sigma(i), or -1 where position i starts from zero
    if (has_tile) {
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int hq = 0; hq < 2; ++hq) {
          const int li = lrow0 + mi * 16 + g + hq * 8;
          const int i = r0 + li;
          const bool rv = i < n && !(i >= k0 && i < k0 + w);
          const int src = rv ? srow[li] : -1;
          src_of[mi][hq] = src;
#pragma unroll
          for (int ni = 0; ni < 4; ++ni) {
            const int c = c0 + ni * 8 + 2 * t;  // even
            cplx y0 = cmk(0, 0), y1 = cmk(0, 0);
            if (src == i) {
              const cplx* p = X + (int64_t)i * ldx + c;
              if (pairs) {
                if (c < n) ld_pair(p, y0, y1);
              } else {
                if (c < n) y0 = p[0];
                if (c + 1 < n) y1 = p[1];
              }
            }
            acc_re[mi][ni][hq * 2] = y0.x;
            acc_im[mi][ni][hq * 2] = y0.y;
            acc_re[mi][ni][hq * 2 + 1] = y1.x;
            acc_im[mi][ni][hq * 2 + 1] = y1.y;
          }
        }
    }
    cp_async_wait<0>();
    __syncthreads();
    if (has_tile) {
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int hq = 0; hq < 2; ++hq) {
          const int i = r0 + lrow0 + mi * 16 + g + hq * 8;
          const int src = src_of[mi][hq];
          if (src >= 0 && src != i) {
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
              for (int ql = 0; ql < 2; ++ql) {
                const int cc = ni * 8 + 2 * t + ql;
                if (c0 + cc < n) {
                  const cplx y = D[(src - k0) * SPLIT_LDR + cc];
                  acc_re[mi][ni][hq * 2 + ql] = y.x;
                  acc_im[mi][ni][hq * 2 + ql] = y.y;
                }
              }
          }
        }
      for (int kk = 0; kk < w; kk += 4) {
        const int kc = kk + t;
        cplx af[2][2];
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int li = lrow0 + mi * 16 + g + h * 8;
            af[mi][h] = (kc < w) ? Prow[pidx(li, kc, 32)] : cmk(0, 0);
          }
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
          const cplx bf = (kc < w) ? R[kc * SPLIT_LDR + ni * 8 + g] : cmk(0, 0);
#pragma unroll
          for (int mi = 0; mi < 2; ++mi) {
            dmma(acc_re[mi][ni], af[mi][0].x, af[mi][1].x, bf.x);
            dmma(acc_im[mi][ni], af[mi][0].x, af[mi][1].x, bf.y);
          }
#pragma unroll
          for (int mi = 0; mi < 2; ++mi) {
            dmma(acc_re[mi][ni], -af[mi][0].y, -af[mi][1].y, bf.y);
            dmma(acc_im[mi][ni], af[mi][0].y, af[mi][1].y, bf.x);
          }
        }
      }
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int hq = 0; hq < 2; ++hq) {
          const int i = r0 + lrow0 + mi * 16 + g + hq * 8;
          if (i >= n) continue;
#pragma unroll
          for (int ni = 0; ni < 4; ++ni) {
            const int c = c0 + ni * 8 + 2 * t;  // even
            const cplx v0 = cmk(acc_re[mi][ni][hq * 2], acc_im[mi][ni][hq * 2]);
            const cplx v1 = cmk(acc_re[mi][ni][hq * 2 + 1], acc_im[mi][ni][hq * 2 + 1]);
            cplx* p = X + (int64_t)i * ldx + c;
            if (pairs) {
              if (c < n && !(c >= k0 && c < k0 + w)) st_pair(p, v0, v1);
            } else {
              if (c < n && !(c >= k0 && c < k0 + w)) p[0] = v0;
              if (c + 1 < n && !(c + 1 >= k0 && c + 1 < k0 + w)) p[1] = v1;
            }
          }
        }
    }
    __syncthreads();
  }
}

// Undo the row interchanges as column interchanges (reverse order),
// UNS_ROWS rows per CTA.
constexpr int UNS_ROWS = 8;

inline size_t split_unscramble_smem(int n) {
  return 2 * ((n * sizeof(int) + 15) & ~size_t(15)) + (size_t)UNS_ROWS * n * sizeof(cplx);
}

__global__ void __launch_bounds__(THREADS)
    zinv_split_unscramble_kernel(int n, int64_t batch, cplx* x_base, int64_t ldx, int64_t sx, SplitScratch sc,
                                 const int* active) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const size_t iw = (n * sizeof(int) + 15) & ~size_t(15);
  int* colsrc = reinterpret_cast<int*>(smem_raw);
  int* perm = reinterpret_cast<int*>(smem_raw + iw);
  cplx* rows = reinterpret_cast<cplx*>(smem_raw + 2 * iw);
  const int tid = threadIdx.x;
  const int r0 = blockIdx.x * UNS_ROWS, nr = min(UNS_ROWS, n - r0);
  for (int64_t e = blockIdx.y; e < batch; e += gridDim.y) {
    if (active && !active[e]) continue;
    cplx* X = x_base + e * sx;
    for (int c = tid; c < n; c += THREADS) {
      colsrc[c] = c;
      perm[c] = sc.perm[e * n + c];
    }
    __syncthreads();
    if (tid == 0) {
      for (int k = n - 1; k >= 0; --k) {
        const int q = perm[k];
        const int tmp = colsrc[k];
        colsrc[k] = colsrc[q];
        colsrc[q] = tmp;
      }
    }
    for (int idx = tid; idx < nr * n; idx += THREADS) {
      const int r = idx / n, c = idx % n;
      rows[idx] = X[(int64_t)(r0 + r) * ldx + c];
    }
    __syncthreads();
    for (int idx = tid; idx < nr * n; idx += THREADS) {
      const int r = idx / n, c = idx % n;
      X[(int64_t)(r0 + r) * ldx + c] = rows[r * n + colsrc[c]];
    }
    __syncthreads();
  }
}

}  // namespace

namespace {

// Column loop of the 32-column panel elimination (b in 129..256),
// QTX_INV_ROTATE: 1 (the default) the rotated register row with one update
// formula for every row, 0 the select-based loop of the other shapes.
// Measured on B200, b = 256, batch 148 / batch 16 (split path): select loop
// 1.82 / 0.98 ms; rotation alone 1.72 / 0.89 ms (bit for bit the same
// results as the select loop); rotation with the uniform pivot-row update
// 1.67 / 0.84 ms (the pivot row then differs by FP64 rounding).  Rotation
// with each step's updates deferred into the next step's reduction was
// slower (more spills at 255 registers) and is not built.
int rotate_panel() {
  static int v = [] {
    const char* env = getenv("QTX_INV_ROTATE");
    return env ? atoi(env) : 1;
  }();
  return v;
}

template <int TPR, int RPT, int CPT, int ROT>
void launch_inv_r(int n, int64_t batch, MatView a, MutView x, int* info, const int* active, size_t smem,
                  cudaStream_t stream) {
  qtx_opt_in_smem((const void*)zinv_gj_kernel<TPR, RPT, CPT, ROT>, smem);
  int grid = (int)(batch < 65535 ? batch : 65535);
  zinv_gj_kernel<TPR, RPT, CPT, ROT><<<grid, THREADS, smem, stream>>>(n, batch, a.ptr, a.ld, a.stride, x.ptr,
                                                                       x.ld, x.stride, info, active);
}

template <int TPR, int RPT, int CPT>
void launch_inv_t(int n, int64_t batch, MatView a, MutView x, int* info, const int* active, size_t smem,
                  cudaStream_t stream) {
  if constexpr (TPR == 1 && RPT == 1 && CPT == 32) {
    const int r = rotate_panel();
    if (r != 0) return launch_inv_r<TPR, RPT, CPT, 1>(n, batch, a, x, info, active, smem, stream);
  }
  launch_inv_r<TPR, RPT, CPT, 0>(n, batch, a, x, info, active, smem, stream);
}

}  // namespace

namespace {

template <int TPR, int RPT, int CPT, int ROT>
void launch_split_r(int n, int64_t batch, MatView a, MutView x, int* info, const int* active, cudaStream_t stream) {
  const InvShape s = inv_shape(n);
  const int W = s.w;
  const size_t psmem = inv_smem_bytes(n) - (size_t)slab_elems(n, s) * sizeof(cplx);
  const size_t usmem = split_update_smem(W);
  const size_t xsmem = split_unscramble_smem(n);
  qtx_opt_in_smem((const void*)zinv_split_panel_kernel<TPR, RPT, CPT, ROT>, psmem);
  qtx_opt_in_smem((const void*)zinv_split_update_kernel, usmem);
  qtx_opt_in_smem((const void*)zinv_split_unscramble_kernel, xsmem);
  const size_t bytes = sizeof(cplx) * (size_t)batch * (3 * (size_t)n * W) + sizeof(int) * (size_t)batch * 2 * n + 256;
  unsigned char* buf = static_cast<unsigned char*>(qtx_malloc_async(bytes, stream));
  if (!buf) throw QtxError(QTX_E_NOMEM, "qtx inverse: scratch allocation failed");
  SplitScratch sc;
  sc.p = reinterpret_cast<cplx*>(buf);
  sc.r = sc.p + (size_t)batch * n * W;
  sc.d = sc.r + (size_t)batch * W * n;
  sc.sigma = reinterpret_cast<int*>(sc.d + (size_t)batch * W * n);
  sc.perm = sc.sigma + (size_t)batch * n;

  const unsigned gb = (unsigned)(batch < 65535 ? batch : 65535);
  const int nslab = (n + SPLIT_CW - 1) / SPLIT_CW, ngroups = (n + SPLIT_ROWS - 1) / SPLIT_ROWS;
  for (int k0 = 0; k0 < n; k0 += W) {
    const int w = std::min(W, n - k0);
    zinv_split_panel_kernel<TPR, RPT, CPT, ROT><<<gb, THREADS, psmem, stream>>>(n, batch, a.ptr, a.ld, a.stride,
                                                                               x.ptr, x.ld, x.stride, k0, sc, info,
                                                                               active);
    zinv_split_rows_kernel<<<dim3(w, gb), 256, 0, stream>>>(n, batch, x.ptr, x.ld, x.stride, k0, W, sc, active);
    zinv_split_update_kernel<<<dim3(nslab * ngroups, gb), SPLIT_THREADS, usmem, stream>>>(n, batch, x.ptr, x.ld,
                                                                                         x.stride, k0, w, W, sc,
                                                                                         active);
  }
  zinv_split_unscramble_kernel<<<dim3((n + UNS_ROWS - 1) / UNS_ROWS, gb), THREADS, xsmem, stream>>>(
      n, batch, x.ptr, x.ld, x.stride, sc, active);
  cudaFreeAsync(buf, stream);
}

template <int TPR, int RPT, int CPT>
void launch_split_t(int n, int64_t batch, MatView a, MutView x, int* info, const int* active, cudaStream_t stream) {
  if constexpr (TPR == 1 && RPT == 1 && CPT == 32) {
    const int r = rotate_panel();
    if (r != 0) return launch_split_r<TPR, RPT, CPT, 1>(n, batch, a, x, info, active, stream);
  }
  launch_split_r<TPR, RPT, CPT, 0>(n, batch, a, x, info, active, stream);
}

// Batches below split_below(n) matrices take the split path (the fused
// kernel keeps one matrix per SM, so a small batch leaves most SMs idle
// during the updates).  Crossovers measured on B200 (kernel_bench inv, fused
// vs split): b = 128 between 64 and 100 matrices, b = 256 at about 105
// (1.61 vs 1.57 ms at 100, 1.63 vs 1.74 ms at 120), b = 512 between 100 and
// 148 (12.7 vs 10.9 ms at 100, 13.0 vs 14.9 ms at 148).  QTX_INV_SPLIT_BELOW
// sets one threshold for every size (0: never split).
int64_t split_below(int n) {
  static const int64_t env = [] {
    const char* v = getenv("QTX_INV_SPLIT_BELOW");
    return v ? (int64_t)atoll(v) : (int64_t)-1;
  }();
  if (env >= 0) return env;
  return n <= 128 ? 80 : (n <= 256 ? 110 : 124);
}

}  // namespace

size_t zinv_workspace_bytes(int n, int64_t batch) {
  if (n <= 64 || n > 512 || batch >= split_below(n)) return 0;
  const size_t W = (size_t)inv_shape(n).w;
  return sizeof(cplx) * (size_t)batch * 3 * (size_t)n * W + sizeof(int) * (size_t)batch * 2 * n + 256;
}

void launch_zinv(int n, int64_t batch, MatView a, MutView x, int* info, const int* active, cudaStream_t stream,
                 bool may_allocate) {
  if (n <= 0 || batch <= 0) return;
  if (n > 512) throw QtxError(QTX_E_UNSUPPORTED, "qtx inverse: block size above 512");
  const size_t smem = inv_smem_bytes(n);
  const InvShape s = inv_shape(n);
  // every panel row / column must be owned by the elimination mapping
  const int rpt = (n + (THREADS / s.tpr) - 1) / (THREADS / s.tpr);
  const int cpt = (s.w + s.tpr - 1) / s.tpr;
  if (may_allocate && n > 64 && batch < split_below(n)) {
    if (s.tpr == 1 && rpt == 1 && cpt <= 32) launch_split_t<1, 1, 32>(n, batch, a, x, info, active, stream);
    else if (s.tpr == 1 && rpt == 2 && cpt <= 16) launch_split_t<1, 2, 16>(n, batch, a, x, info, active, stream);
    else if (s.tpr == 2 && rpt == 1 && cpt <= 16) launch_split_t<2, 1, 16>(n, batch, a, x, info, active, stream);
    else throw QtxError(QTX_E_UNSUPPORTED, "qtx inverse: block size outside the supported shapes");
    qtx_check_launch("zinv_split");
    return;
  }
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
