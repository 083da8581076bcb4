// Grouped transport solve: the persistent launch of the batching form.
//
// The energies of several generator-form problems (each its own H, number of
// blocks, energy grid and contacts) that share one block size b <= 64 are
// solved by ONE persistent kernel launch.  A CTA takes the next (problem,
// energy) pair from a global counter and runs that energy's whole transport
// solve by itself: Sancho-Rubio decimation of both leads (its own convergence
// loop, no host round trip), the contact self-energies, the forward and
// backward RGF sweeps of G^R and of the Keldysh G^<, G^> blocks, and the
// observables.  Problems of uneven size therefore share one launch with no
// per-step kernel boundaries: a CTA that finishes a short problem takes the
// next pair, and the pairs are handed out longest problem first.  At b <= 64
// the layered path (one launch per block product over an energy batch) is
// bound by launch and dependency latency; here a CTA never waits for another.
//
// The recursion is that of transport_contacts / transport_sweep (rgf.cu),
// product for product, on b x b blocks in the CTA's own global-memory work
// space (an energy's working set of a few hundred KB stays in L1/L2):
//   * cta_gemm: D = alpha op(A) op(B) + beta C + gamma C2 (+ s I), 4M complex
//     products on DMMA (mma.sync m16n8k4 f64) from a 4-stage cp.async ring of
//     8-wide K slices; per output element the K order and the DMMA sequence
//     are those of zgemm_dmma_kernel.
//   * cta_inverse: Gauss-Jordan with implicit partial pivoting (LAPACK izamax
//     rule: first row of maximal |Re| + |Im|), the matrix in registers with
//     THREADS / BT threads per row, one barrier per column, the row and
//     column permutations applied on the store.
// There are no inter-CTA waits: the only shared state is the work counter
// and the error flags.
#include "kernels.h"

namespace {

// Tile class BT (32 or 64) of the block size: 4 warps of 16 x 16 warp tiles
// (4 CTAs per SM) or 8 warps of 32 x 16 warp tiles (2 CTAs per SM).  The
// recursion is a chain of dependent block operations, so these warps are all
// the latency hiding a CTA has: at most 128 registers a thread keep them
// resident.
template <int BT>
struct GCfg {
  static constexpr int THREADS = BT <= 32 ? 128 : 256;
  static constexpr int NWARPS = THREADS / 32, WARPS_N = NWARPS / 2;
  static constexpr int BK = 8, ST = 4;
  static constexpr int LDK = BK + 4;  // tile stored [row][k]
  static constexpr int LDM = BT + 2;  // tile stored [k][row]
  static constexpr int TILE = (BT * LDK > BK * LDM) ? BT * LDK : BK * LDM;
  static constexpr int WM = BT / 2, WN = BT / WARPS_N, MI = WM / 16, NI = WN / 8;
  static constexpr int GEMM_ELEMS = ST * 2 * TILE;
  static constexpr int TPR = THREADS / BT, CPT = BT / TPR;  // inverse: threads per row, columns per thread
  static constexpr int CAND_ELEMS = 2 * NWARPS * BT;
  static constexpr int REGION = GEMM_ELEMS > CAND_ELEMS ? GEMM_ELEMS : CAND_ELEMS;
  static constexpr int MIN_BLOCKS = BT <= 32 ? 4 : 2;
};

template <int BT>
struct Misc {
  double red_v[2][GCfg<BT>::NWARPS];
  int red_i[2][GCfg<BT>::NWARPS];
  cplx red_piv[2][GCfg<BT>::NWARPS];  // column-k entry of each warp's candidate
  int pivs[BT];  // pivot row of each step
  int pos[BT];   // step at which each row was the pivot
  double sum[2 * GCfg<BT>::NWARPS];
  unsigned long long item;
};

template <int BT>
constexpr size_t smem_bytes() {
  return sizeof(cplx) * GCfg<BT>::REGION + sizeof(Misc<BT>);
}

// Dynamic shared memory: the product staging ring (or the inverse's pivot
// candidates) followed by Misc.  The helpers below are separate functions,
// so they derive these pointers from the __shared__ symbol themselves: a
// pointer handed in as an argument would turn every access into a generic one.
extern __shared__ __align__(16) unsigned char grouped_smem[];
template <int BT>
__device__ __forceinline__ cplx* smem_region() {
  return reinterpret_cast<cplx*>(grouped_smem);
}
template <int BT>
__device__ __forceinline__ Misc<BT>* smem_misc() {
  return reinterpret_cast<Misc<BT>*>(grouped_smem + sizeof(cplx) * GCfg<BT>::REGION);
}

__device__ __forceinline__ void dmma(double (&c)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

// The operands were written by this CTA's own threads before a barrier: the
// copies go through L1 (.ca), the same path as the threads' loads.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool pred) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int bytes = pred ? 16 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// One block product of the recursion.  All matrices are n x n, row-major with
// leading dimension n.  k is n, or 0 for the epilogue alone.  d may alias c
// or c2, never a or b.
struct GArgs {
  const cplx* a = nullptr;
  const cplx* b = nullptr;
  const cplx* c = nullptr;
  const cplx* c2 = nullptr;
  cplx* d = nullptr;
  cplx alpha = {1, 0}, beta = {0, 0}, gamma = {0, 0}, shift = {0, 0};
  int opa = OP_N, opb = OP_N, k = 0, has_shift = 0;
};

template <int BT, int OPA, int OPB>
__device__ __forceinline__ void gemm_stage(cplx* sa, const GArgs& g, int n, int k0, int tid) {
  using C = GCfg<BT>;
  cplx* sb = sa + C::TILE;
#pragma unroll
  for (int r = 0; r < (BT * C::BK) / C::THREADS; ++r) {
    const int idx = tid + r * C::THREADS;
    if (OPA == OP_N) {
      const int row = idx / C::BK, col = idx % C::BK, gk = k0 + col;
      const bool ok = row < n && gk < g.k;
      cp_async16(sa + row * C::LDK + col, ok ? g.a + (int64_t)row * n + gk : g.a, ok);
    } else {
      const int krow = idx / BT, mcol = idx % BT, gk = k0 + krow;
      const bool ok = mcol < n && gk < g.k;
      cp_async16(sa + krow * C::LDM + mcol, ok ? g.a + (int64_t)gk * n + mcol : g.a, ok);
    }
    if (OPB == OP_N) {
      const int krow = idx / BT, ncol = idx % BT, gk = k0 + krow;
      const bool ok = ncol < n && gk < g.k;
      cp_async16(sb + krow * C::LDM + ncol, ok ? g.b + (int64_t)gk * n + ncol : g.b, ok);
    } else {
      const int nrow = idx / C::BK, kcol = idx % C::BK, gk = k0 + kcol;
      const bool ok = nrow < n && gk < g.k;
      cp_async16(sb + nrow * C::LDK + kcol, ok ? g.b + (int64_t)nrow * n + gk : g.b, ok);
    }
  }
}

template <int BT, int OPA>
__device__ __forceinline__ cplx frag_a(const cplx* sm, int m, int k) {
  if (OPA == OP_N) return sm[m * GCfg<BT>::LDK + k];
  const cplx v = sm[k * GCfg<BT>::LDM + m];
  return make_double2(v.x, -v.y);
}
template <int BT, int OPB>
__device__ __forceinline__ cplx frag_b(const cplx* sm, int k, int n) {
  if (OPB == OP_N) return sm[k * GCfg<BT>::LDM + n];
  const cplx v = sm[n * GCfg<BT>::LDK + k];
  return make_double2(v.x, -v.y);
}

template <int BT, int OPA, int OPB>
__device__ __forceinline__ void gemm_body(const GArgs& g, int n) {
  using C = GCfg<BT>;
  cplx* smem = smem_region<BT>();
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, gq = lane >> 2, t = lane & 3;
  const int wm0 = (warp / C::WARPS_N) * C::WM, wn0 = (warp % C::WARPS_N) * C::WN;
  const int ktiles = (g.k + C::BK - 1) / C::BK;
  double acc_re[C::MI][C::NI][4], acc_im[C::MI][C::NI][4];
#pragma unroll
  for (int i = 0; i < C::MI; ++i)
#pragma unroll
    for (int j = 0; j < C::NI; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc_re[i][j][q] = acc_im[i][j][q] = 0.0;

#pragma unroll
  for (int s = 0; s < C::ST - 1; ++s) {
    if (s < ktiles) gemm_stage<BT, OPA, OPB>(smem + s * 2 * C::TILE, g, n, s * C::BK, tid);
    cp_async_commit();
  }
  for (int kt = 0; kt < ktiles; ++kt) {
    cp_async_wait<C::ST - 2>();
    __syncthreads();
    {
      const int nk = kt + C::ST - 1;
      if (nk < ktiles) gemm_stage<BT, OPA, OPB>(smem + (nk % C::ST) * 2 * C::TILE, g, n, nk * C::BK, tid);
      cp_async_commit();
    }
    const cplx* sa = smem + (kt % C::ST) * 2 * C::TILE;
    const cplx* sb = sa + C::TILE;
#pragma unroll
    for (int kk = 0; kk < C::BK; kk += 4) {
      cplx af[C::MI][2], bf[C::NI];
#pragma unroll
      for (int mi = 0; mi < C::MI; ++mi) {
        af[mi][0] = frag_a<BT, OPA>(sa, wm0 + mi * 16 + gq, kk + t);
        af[mi][1] = frag_a<BT, OPA>(sa, wm0 + mi * 16 + gq + 8, kk + t);
      }
#pragma unroll
      for (int ni = 0; ni < C::NI; ++ni) bf[ni] = frag_b<BT, OPB>(sb, kk + t, wn0 + ni * 8 + gq);
      // first product of every accumulator, then the second: each
      // accumulator still sees Ar Br, -Ai Bi (Re) and Ar Bi, Ai Br (Im) in
      // that order, with 2 MI NI independent DMMAs between dependent ones
#pragma unroll
      for (int mi = 0; mi < C::MI; ++mi)
#pragma unroll
        for (int ni = 0; ni < C::NI; ++ni) {
          dmma(acc_re[mi][ni], af[mi][0].x, af[mi][1].x, bf[ni].x);
          dmma(acc_im[mi][ni], af[mi][0].x, af[mi][1].x, bf[ni].y);
        }
#pragma unroll
      for (int mi = 0; mi < C::MI; ++mi)
#pragma unroll
        for (int ni = 0; ni < C::NI; ++ni) {
          dmma(acc_re[mi][ni], -af[mi][0].y, -af[mi][1].y, bf[ni].y);
          dmma(acc_im[mi][ni], af[mi][0].y, af[mi][1].y, bf[ni].x);
        }
    }
  }
  cp_async_wait<0>();
  __syncthreads();
#pragma unroll
  for (int mi = 0; mi < C::MI; ++mi)
#pragma unroll
    for (int ni = 0; ni < C::NI; ++ni)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int row = wm0 + mi * 16 + gq + ((q >> 1) << 3);
        const int col = wn0 + ni * 8 + 2 * t + (q & 1);
        if (row < n && col < n) {
          const int64_t o = (int64_t)row * n + col;
          cplx v = cmul(g.alpha, cmk(acc_re[mi][ni][q], acc_im[mi][ni][q]));
          if (g.c) v = cfma(g.beta, g.c[o], v);
          if (g.c2) v = cfma(g.gamma, g.c2[o], v);
          if (g.has_shift && row == col) v = cadd(v, g.shift);
          g.d[o] = v;
        }
      }
  __syncthreads();
}

template <int BT>
__device__ __noinline__ void cta_gemm(const GArgs g, int n) {
  if (g.opa == OP_N) {
    if (g.opb == OP_N) gemm_body<BT, OP_N, OP_N>(g, n);
    else gemm_body<BT, OP_N, OP_C>(g, n);
  } else {
    if (g.opb == OP_N) gemm_body<BT, OP_C, OP_N>(g, n);
    else gemm_body<BT, OP_C, OP_C>(g, n);
  }
}

__device__ __forceinline__ void argmax_combine(double& v, int& i, double v2, int i2) {
  if (v2 > v || (v2 == v && i2 < i)) {
    v = v2;
    i = i2;
  }
}

// X = A^-1 (n x n, n <= BT; X must not alias A).  Returns 0, or 1 + the first
// column whose pivot is exactly zero (the result then holds inf/NaN).
//
// Rows stay where they are (implicit pivoting): step k picks pivot row p_k
// among the rows not used yet and stores the elimination in place.  The
// row-swapping form would hold row p_k at position k, so with pos(r) the step
// at which row r was the pivot, X[pos(r)][p_c] = M[r][c]: every thread writes
// its own elements once, through the pivot list and its inverse.
//
// The in-place step is x_rc <- x_rc - (x_rk / piv) p_c for c != k and
// -x_rk / piv at c = k.  The staged pivot row carries 1 at column k and every
// row clears its own column-k entry when it reads it, so one branch-free
// x - fd p covers both (the pivot row's own entries p_c / piv likewise); the
// pivot value itself travels through shared memory.
template <int BT>
__device__ __noinline__ int cta_inverse(const cplx* A, cplx* X, int n) {
  using C = GCfg<BT>;
  cplx* cand = smem_region<BT>();
  Misc<BT>* ms = smem_misc<BT>();
  constexpr int TPR = C::TPR, CPT = C::CPT;
  constexpr int ROWS_PER_WARP = 32 / TPR;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r_own = tid / TPR, c_own = tid % TPR;
  const int grp0 = lane - c_own;  // first lane of this row's group
  cplx reg[CPT];
#pragma unroll
  for (int j = 0; j < CPT; ++j) {
    const int c = c_own + j * TPR;
    reg[j] = (r_own < n && c < n) ? A[(int64_t)r_own * n + c] : cmk(0, 0);
  }
  // staged rows are written at columns < n only: the rest stays zero, so the
  // padding columns of every register row stay zero too
  for (int q = tid; q < C::CAND_ELEMS; q += C::THREADS) cand[q] = cmk(0, 0);
  __syncthreads();
  bool used = r_own >= n;
  int zero = 0;
#pragma unroll 1
  for (int kk = 0; kk < n; ++kk) {
    const int kc = kk % TPR;  // lanes c_own == kc hold column kk
    cplx colv = cmk(0, 0);
#pragma unroll
    for (int j = 0; j < CPT; ++j)
      if (c_own + j * TPR == kk) {
        colv = reg[j];
        reg[j] = cmk(0, 0);
      }
    double bv = -1.0;
    int bi = n;
    if (c_own == kc && !used) {
      bv = cabs1(colv);
      bi = r_own;
    }
    // the warp's best row among the lanes holding column kk (lanes that share
    // c_own differ in the bits above log2(TPR)); then lane kc tells the rest
#pragma unroll
    for (int off = 16; off >= TPR; off >>= 1) {
      const double v2 = __shfl_xor_sync(0xffffffffu, bv, off);
      const int i2 = __shfl_xor_sync(0xffffffffu, bi, off);
      argmax_combine(bv, bi, v2, i2);
    }
    bi = __shfl_sync(0xffffffffu, bi, kc);
    const int src = grp0 + kc;
    const cplx f = cmk(__shfl_sync(0xffffffffu, colv.x, src), __shfl_sync(0xffffffffu, colv.y, src));
    const int par = kk & 1;
    if (bi < n && r_own == bi) {
      cplx* my_cand = cand + (par * C::NWARPS + warp) * BT;
#pragma unroll
      for (int j = 0; j < CPT; ++j) {
        const int c = c_own + j * TPR;
        if (c < n) my_cand[c] = reg[j];
      }
      if (c_own == kc) {
        my_cand[kk] = cmk(1, 0);
        ms->red_piv[par][warp] = colv;
      }
    }
    if (lane == kc) {
      ms->red_v[par][warp] = bv;
      ms->red_i[par][warp] = bi;
    }
    __syncthreads();  // every warp's candidate row visible
    // best over the warps: every group of NWARPS lanes holds all candidates
    double v = ms->red_v[par][lane % C::NWARPS];
    int p = ms->red_i[par][lane % C::NWARPS];
#pragma unroll
    for (int off = C::NWARPS / 2; off > 0; off >>= 1) {
      const double v2 = __shfl_xor_sync(0xffffffffu, v, off);
      const int i2 = __shfl_xor_sync(0xffffffffu, p, off);
      argmax_combine(v, p, v2, i2);
    }
    // the global best is also the best of its own warp, whose row is staged
    const int pw = p / ROWS_PER_WARP;
    const cplx* prow = cand + (par * C::NWARPS + pw) * BT;
    const cplx piv = ms->red_piv[par][pw];
    if (piv.x == 0.0 && piv.y == 0.0 && !zero) zero = kk + 1;
    const cplx d = crecip_pivot(piv);
    if (tid == 0) ms->pivs[kk] = p;
    if (r_own == p) {
      used = true;
#pragma unroll
      for (int j = 0; j < CPT; ++j) reg[j] = cmul(prow[c_own + j * TPR], d);
    } else {
      const cplx fd = cmul(f, d);
#pragma unroll
      for (int j = 0; j < CPT; ++j) reg[j] = cfms(fd, prow[c_own + j * TPR], reg[j]);
    }
  }
  __syncthreads();
  for (int k = tid; k < n; k += C::THREADS) ms->pos[ms->pivs[k]] = k;
  __syncthreads();
  if (r_own < n) {
    const int i = ms->pos[r_own];
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
      const int c = c_own + j * TPR;
      if (c < n) X[(int64_t)i * n + ms->pivs[c]] = reg[j];
    }
  }
  __syncthreads();
  return zero;
}

// Sum over the CTA (every thread receives it).
template <int BT>
__device__ cplx cta_sum(cplx v) {
  Misc<BT>* ms = smem_misc<BT>();
  constexpr int NW = GCfg<BT>::NWARPS;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    v.x += __shfl_down_sync(0xffffffffu, v.x, off);
    v.y += __shfl_down_sync(0xffffffffu, v.y, off);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    ms->sum[warp] = v.x;
    ms->sum[NW + warp] = v.y;
  }
  __syncthreads();
  cplx s = cmk(0, 0);
#pragma unroll
  for (int w = 0; w < NW; ++w) {
    s.x += ms->sum[w];
    s.y += ms->sum[NW + w];
  }
  __syncthreads();
  return s;
}

// ---- element-wise block operations (each ends with a barrier) -------------
// d = alpha x (+ beta y)
__device__ void blk_axpby(int n, cplx alpha, const cplx* x, cplx beta, const cplx* y, cplx* d) {
  for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
    cplx v = cmul(alpha, x[q]);
    if (y) v = cfma(beta, y[q], v);
    d[q] = v;
  }
  __syncthreads();
}
// x <- x - x^H in place
__device__ void blk_sub_herm(int n, cplx* x) {
  for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
    const int r = q / n, c = q % n;
    if (r > c) continue;
    const cplx a = x[q], b = x[c * n + r];
    if (r == c) {
      x[q] = cmk(0.0, 2.0 * a.y);
    } else {
      x[q] = cmk(a.x - b.x, a.y + b.y);
      x[c * n + r] = cmk(b.x - a.x, b.y + a.y);
    }
  }
  __syncthreads();
}
// gamma = i (s - s^H); sl = i f gamma; sg = i (f - 1) gamma
__device__ void blk_obc_lesser_greater(int n, const cplx* s, double f, cplx* sl, cplx* sg, cplx* gam) {
  for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
    const int r = q / n, c = q % n;
    const cplx a = s[q], b = s[c * n + r];
    const cplx dd = cmk(a.x - b.x, a.y + b.y);
    const cplx g = cmk(-dd.y, dd.x);
    const cplx ig = cmk(-g.y, g.x);
    sl[q] = cscale(ig, f);
    sg[q] = cscale(ig, f - 1.0);
    gam[q] = g;
  }
  __syncthreads();
}
// Y< = f_L xl + s f_R xr, Y> = (f_L - 1) xl + s (f_R - 1) xr  (keldysh_mix);
// sym: write 0.5 (Y - Y^H).  out_l / out_g may be null.
__device__ void blk_keldysh_combine(int n, const cplx* xl, const cplx* xr, double fl, double fr, double sign_r,
                                    bool sym, cplx* out_l, cplx* out_g) {
  if (out_l || out_g) {
    for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
      const int r = q / n, c = q % n;
      const cplx a = xl[q], b = xr[q];
      const cplx yl = keldysh_mix(fl, a, sign_r * fr, b);
      const cplx yg = keldysh_mix(fl - 1.0, a, sign_r * (fr - 1.0), b);
      if (!sym) {
        if (out_l) out_l[q] = yl;
        if (out_g) out_g[q] = yg;
        continue;
      }
      const cplx at = xl[c * n + r], bt = xr[c * n + r];
      const cplx ylt = keldysh_mix(fl, at, sign_r * fr, bt);
      const cplx ygt = keldysh_mix(fl - 1.0, at, sign_r * (fr - 1.0), bt);
      if (out_l) out_l[q] = cmk(0.5 * (yl.x - ylt.x), 0.5 * (yl.y + ylt.y));
      if (out_g) out_g[q] = cmk(0.5 * (yg.x - ygt.x), 0.5 * (yg.y + ygt.y));
    }
  }
  __syncthreads();
}
// Tr[x y]
template <int BT>
__device__ cplx blk_trace_product(int n, const cplx* x, const cplx* y) {
  cplx acc = cmk(0, 0);
  for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
    const int r = q / n, c = q % n;
    acc = cfma(x[q], y[c * n + r], acc);
  }
  return cta_sum<BT>(acc);
}
// -(1/n) sum_r Im g[r][r]: the block's density of states (G^R)
template <int BT>
__device__ double blk_block_dos(int n, const cplx* g) {
  double acc = 0;
  for (int r = threadIdx.x; r < n; r += blockDim.x) acc += g[r * n + r].y;
  return -cta_sum<BT>(cmk(acc, 0)).x / n;
}
// sum_rc H[r][c] (-conj Y[r][c]) - Y[r][c] conj H[r][c], Y = f_L xl + s f_R xr:
// the layer current across an interface with coupling H and G^< upper block Y
template <int BT>
__device__ cplx blk_layer_current(int n, const cplx* xl, const cplx* xr, double fl, double fr, double sign_r,
                                  const cplx* h) {
  cplx acc = cmk(0, 0);
  for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
    const cplx y = keldysh_mix(fl, xl[q], sign_r * fr, xr[q]);
    const cplx hv = h[q];
    acc = cadd(acc, csub(cmul(hv, cmk(-y.x, y.y)), cmul(y, cconj(hv))));
  }
  return cta_sum<BT>(acc);
}
// (sum_r Im Y<_rr, -sum_r Im Y>_rr) of the combination above (sign 1)
template <int BT>
__device__ cplx blk_keldysh_density(int n, const cplx* xl, const cplx* xr, double fl, double fr) {
  double dl = 0, dg = 0;
  for (int r = threadIdx.x; r < n; r += blockDim.x) {
    const cplx a = xl[r * n + r], b = xr[r * n + r];
    dl += keldysh_mix(fl, a, fr, b).y;
    dg += keldysh_mix(fl - 1.0, a, fr - 1.0, b).y;
  }
  const cplx s = cta_sum<BT>(cmk(dl, dg));
  return cmk(s.x, -s.y);
}

// Sancho-Rubio decimation of one lead (the loop of sancho_rubio_impl for one
// energy; sancho_rubio.py:65-84): eps = eps_s = (E + i eta) I - H_lead,
// alpha = A_ji, beta = A_ij with A_ij = -U (left) or -U^H (right).  Writes
// g = inv(eps_s) to `g`, returns the iterations done (negative when the
// criterion was never met).
template <int BT>
__device__ __noinline__ int cta_sancho_rubio(int n, double energy, double eta, const cplx* h, const cplx* u,
                                            bool left, double tol, int max_iter, cplx* g, cplx* const* T) {
  cplx *eps = T[0], *eps_s = T[1], *alpha = T[2], *beta = T[3], *inv = T[4];
  cplx *t0 = T[5], *t1 = T[6], *t2 = T[7], *t3 = T[8];
  for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
    const int r = q / n, c = q % n;
    const cplx hv = h[q];
    cplx v = cmk(-hv.x, -hv.y);
    if (r == c) {
      v.x += energy;
      v.y += eta;
    }
    eps[q] = v;
    eps_s[q] = v;
    const cplx uv = u[q], ut = u[c * n + r];
    const cplx up = cmk(-uv.x, -uv.y), lo = cmk(-ut.x, ut.y);
    alpha[q] = left ? lo : up;
    beta[q] = left ? up : lo;
  }
  __syncthreads();
  const cplx ONE = cmk(1, 0), MONE = cmk(-1, 0);
  int its = 0;
  bool converged = false;
  for (int it = 0; it < max_iter; ++it) {
    cta_inverse<BT>(eps, inv, n);
    GArgs g0;
    g0.k = n;
    GArgs a = g0;
    a.a = alpha; a.b = inv; a.d = t0;
    cta_gemm<BT>(a, n);  // a inv
    a = g0;
    a.a = beta; a.b = inv; a.d = t1;
    cta_gemm<BT>(a, n);  // b inv
    a = g0;
    a.a = t0; a.b = beta; a.d = t2;
    cta_gemm<BT>(a, n);  // a inv b
    blk_axpby(n, ONE, eps_s, MONE, t2, eps_s);
    a = g0;  // eps = eps - b inv a - a inv b
    a.a = t1; a.b = alpha; a.d = eps; a.alpha = MONE; a.c = eps; a.beta = ONE; a.c2 = t2; a.gamma = MONE;
    cta_gemm<BT>(a, n);
    a = g0;
    a.a = t0; a.b = alpha; a.d = t3;
    cta_gemm<BT>(a, n);  // a inv a
    a = g0;
    a.a = t1; a.b = beta; a.d = t2;
    cta_gemm<BT>(a, n);  // b inv b
    cplx* tmp = alpha;
    alpha = t3;
    t3 = tmp;
    tmp = beta;
    beta = t2;
    t2 = tmp;
    ++its;
    double acc = 0;
    for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
      const cplx av = alpha[q], bv = beta[q];
      const double s = hypot(av.x, av.y) + hypot(bv.x, bv.y);
      acc += s * s;
    }
    const double delta = sqrt(cta_sum<BT>(cmk(acc, 0)).x) / 2.0;
    if (delta < tol) {
      converged = true;
      break;
    }
  }
  cta_inverse<BT>(eps_s, g, n);
  return converged ? its : -its;
}

// The whole transport solve of energy e of problem P (transport_contacts and
// transport_sweep of rgf.cu for one energy).
template <int BT>
__device__ __noinline__ void solve_energy(const GroupedProblem* P, int pidx, int64_t e, cplx* ws, int max_nb,
                                          int* flags) {
  const int nb = P->nb, n = P->b;
  const int64_t bb = (int64_t)n * n;
  auto XR = [&](int i) { return ws + i * bb; };
  auto XL = [&](int i) { return ws + (max_nb + i) * bb; };
  auto XG = [&](int i) { return ws + (2 * max_nb + i) * bb; };
  cplx* T[10];
  cplx* Cb[10];  // g_L, g_R, SigR_L, SigR_R, SigL_L, SigL_R, SigG_L, SigG_R, Gam_L, Gam_R
  for (int q = 0; q < 10; ++q) {
    T[q] = ws + (3 * max_nb + q) * bb;
    Cb[q] = ws + (3 * max_nb + 10 + q) * bb;
  }
  const cplx* Hd = P->h_diag;
  const cplx* U = P->h_upper;
  auto hd = [&](int i) { return Hd + i * bb; };
  auto uu = [&](int i) { return U + i * bb; };
  const double energy = P->energies[e];
  const cplx shift = cmk(energy, P->eta);
  const cplx ONE = cmk(1, 0), MONE = cmk(-1, 0);
  GArgs g0;
  g0.k = n;
  int zero = 0;

  // ---- contacts
  const int its_l = cta_sancho_rubio<BT>(n, energy, P->eta, hd(0), uu(0), true, P->sr_tol, P->sr_max_iterations,
                                         Cb[0], T);
  const int its_r = cta_sancho_rubio<BT>(n, energy, P->eta, hd(nb - 1), uu(nb - 2), false, P->sr_tol,
                                         P->sr_max_iterations, Cb[1], T);
  if (threadIdx.x == 0) {
    if (P->sr_iterations) {
      P->sr_iterations[2 * e] = its_l < 0 ? -its_l : its_l;
      P->sr_iterations[2 * e + 1] = its_r < 0 ? -its_r : its_r;
    }
    if (its_l < 0 || its_r < 0) {
      atomicOr(flags, 2);
      atomicOr(flags + 1 + pidx, 2);
    }
  }
  GArgs a = g0;  // Sigma^R_L = A_10 g_L A_01 = (-U_0^H) g_L (-U_0)
  a.a = uu(0); a.opa = OP_C; a.b = Cb[0]; a.d = T[1]; a.alpha = MONE;
  cta_gemm<BT>(a, n);
  a = g0;
  a.a = T[1]; a.b = uu(0); a.d = Cb[2]; a.alpha = MONE;
  cta_gemm<BT>(a, n);
  a = g0;  // Sigma^R_R = A_mn g_R A_nm = (-U) g_R (-U^H)
  a.a = uu(nb - 2); a.b = Cb[1]; a.d = T[1]; a.alpha = MONE;
  cta_gemm<BT>(a, n);
  a = g0;
  a.a = T[1]; a.b = uu(nb - 2); a.opb = OP_C; a.d = Cb[3]; a.alpha = MONE;
  cta_gemm<BT>(a, n);
  const double f_l = 1.0 / (1.0 + exp((energy - P->mu_left) / P->kt));
  const double f_r = 1.0 / (1.0 + exp((energy - P->mu_right) / P->kt));
  blk_obc_lesser_greater(n, Cb[2], f_l, Cb[4], Cb[6], Cb[8]);
  blk_obc_lesser_greater(n, Cb[3], f_r, Cb[5], Cb[7], Cb[9]);

  // ---- first block: x_0 = inv((E + i eta) I - H_00 - Sigma^R_L), X_L,0 = x_0 (i Gamma_L) x_0^H
  // (the Keldysh part runs for the two contact sources, as transport_sweep in
  // rgf.cu: X_L from i Gamma_L at block 0, X_R from i Gamma_R at block nb - 1,
  // G^< = f_L X_L + f_R X_R, G^> = (f_L - 1) X_L + (f_R - 1) X_R)
  const cplx I1 = cmk(0, 1);
  a = g0;
  a.k = 0; a.d = T[1]; a.c = hd(0); a.beta = MONE; a.c2 = Cb[2]; a.gamma = MONE; a.has_shift = 1; a.shift = shift;
  cta_gemm<BT>(a, n);
  zero |= cta_inverse<BT>(T[1], XR(0), n);
  a = g0;
  a.a = XR(0); a.b = Cb[8]; a.d = T[2]; a.alpha = I1;
  cta_gemm<BT>(a, n);
  a = g0;
  a.a = T[2]; a.b = XR(0); a.opb = OP_C; a.d = XL(0);
  cta_gemm<BT>(a, n);
  // ---- forward sweep
  for (int i = 0; i + 1 < nb; ++i) {
    const int j = i + 1;
    a = g0;  // A_ji x_i = -U_i^H x_i
    a.a = uu(i); a.opa = OP_C; a.b = XR(i); a.d = T[0]; a.alpha = MONE;
    cta_gemm<BT>(a, n);
    a = g0;  // (E + i eta) I - H_jj - Sigma^R_j - A_ji x_i A_ij
    a.a = T[0]; a.b = uu(i); a.d = T[1]; a.c = hd(j); a.beta = MONE; a.has_shift = 1; a.shift = shift;
    if (j == nb - 1) {
      a.c2 = Cb[3];
      a.gamma = MONE;
    }
    cta_gemm<BT>(a, n);
    zero |= cta_inverse<BT>(T[1], XR(j), n);
    a = g0;  // W = x_j A_ji = -x_j U_i^H ; X_L,j = W X_L,i W^H  (no source past block 0)
    a.a = XR(j); a.b = uu(i); a.opb = OP_C; a.d = T[3]; a.alpha = MONE;
    cta_gemm<BT>(a, n);
    a = g0;
    a.a = T[3]; a.b = XL(i); a.d = T[4];
    cta_gemm<BT>(a, n);
    a = g0;
    a.a = T[4]; a.b = T[3]; a.opb = OP_C; a.d = XL(j);
    cta_gemm<BT>(a, n);
  }
  // ---- last block: X_R,n = x_n (i Gamma_R) x_n^H
  const int nl = nb - 1;
  a = g0;
  a.a = XR(nl); a.b = Cb[9]; a.d = T[2]; a.alpha = I1;
  cta_gemm<BT>(a, n);
  a = g0;
  a.a = T[2]; a.b = XR(nl); a.opb = OP_C; a.d = XG(nl);
  cta_gemm<BT>(a, n);
  const int64_t o_diag = (e * nb + nl) * bb;
  blk_keldysh_combine(n, XL(nl), XG(nl), f_l, f_r, 1.0, true, P->gl_diag ? P->gl_diag + o_diag : nullptr,
                      P->gg_diag ? P->gg_diag + o_diag : nullptr);
  if (P->gr_diag) blk_axpby(n, ONE, XR(nl), ONE, nullptr, P->gr_diag + o_diag);
  if (P->dos) {
    const double v = blk_block_dos<BT>(n, XR(nl));
    if (threadIdx.x == 0) P->dos[e * nb + nl] = v;
  }
  if (P->density || P->hole_density) {
    const cplx dh = blk_keldysh_density<BT>(n, XL(nl), XG(nl), f_l, f_r);
    if (threadIdx.x == 0) {
      if (P->density) P->density[e * nb + nl] = dh.x;
      if (P->hole_density) P->hole_density[e * nb + nl] = dh.y;
    }
  }
  if (P->current_right) {
    blk_keldysh_combine(n, XL(nl), XG(nl), f_l, f_r, 1.0, true, T[6], T[7]);
    const cplx c1 = blk_trace_product<BT>(n, Cb[7], T[6]);
    const cplx c2 = blk_trace_product<BT>(n, T[7], Cb[5]);
    if (threadIdx.x == 0) P->current_right[e] = cadd(c1, cmul(MONE, c2));
  }
  cplx* corner = T[8];
  cplx* corner2 = T[9];
  if (P->transmission) blk_axpby(n, ONE, XR(nl), ONE, nullptr, corner);
  const bool uppers = P->gl_upper || P->gg_upper || P->layer_current;
  // ---- backward sweep
  cplx* g_next = XR(nl);  // G^R_jj of the block after i
  cplx* spare = T[4];
  for (int i = nb - 2; i >= 0; --i) {
    const int j = i + 1;
    const int64_t o_up = (e * (nb - 1) + i) * bb;
    a = g0;  // P1 = x_i A_ij = -x_i U_i
    a.a = XR(i); a.b = uu(i); a.d = T[0]; a.alpha = MONE;
    cta_gemm<BT>(a, n);
    a = g0;  // P2 = G_jj A_ji = -G_jj U_i^H
    a.a = g_next; a.b = uu(i); a.opb = OP_C; a.d = T[1]; a.alpha = MONE;
    cta_gemm<BT>(a, n);
    if (P->gr_upper) {
      a = g0;  // G^R_ij = -P1 G_jj, only an output
      a.a = T[0]; a.b = g_next; a.d = P->gr_upper + o_up; a.alpha = MONE;
      cta_gemm<BT>(a, n);
    }
    a = g0;  // P4 = P1 P2
    a.a = T[0]; a.b = T[1]; a.d = T[3];
    cta_gemm<BT>(a, n);
    if (P->gr_lower) {
      a = g0;
      a.a = T[1]; a.b = XR(i); a.d = P->gr_lower + o_up; a.alpha = MONE;
      cta_gemm<BT>(a, n);
    }
    if (P->transmission) {
      a = g0;  // G_{i,N-1} = -(x_i A_ij) G_{j,N-1}
      a.a = T[0]; a.b = corner; a.d = corner2; a.alpha = MONE;
      cta_gemm<BT>(a, n);
      cplx* tmp = corner;
      corner = corner2;
      corner2 = tmp;
    }
    a = g0;  // X_L: t1 = P4 X_i - (P4 X_i)^H
    a.a = T[3]; a.b = XL(i); a.d = T[5];
    cta_gemm<BT>(a, n);
    blk_sub_herm(n, T[5]);
    a = g0;  // t2 = P1 X_j
    a.a = T[0]; a.b = XL(j); a.d = T[6];
    cta_gemm<BT>(a, n);
    if (uppers) {
      a = g0;  // X_ij = -t2 - X_i P2^H
      a.a = XL(i); a.b = T[1]; a.opb = OP_C; a.d = T[7]; a.alpha = MONE; a.c = T[6]; a.beta = MONE;
      cta_gemm<BT>(a, n);
    }
    a = g0;  // X_i += t2 P1^H + t1
    a.a = T[6]; a.b = T[0]; a.opb = OP_C; a.d = XL(i); a.c = XL(i); a.beta = ONE; a.c2 = T[5]; a.gamma = ONE;
    cta_gemm<BT>(a, n);
    a = g0;  // X_R (zero in the forward sweep): t2 = P1 X_j, X_ij = -t2, X_i = t2 P1^H
    a.a = T[0]; a.b = XG(j); a.d = T[5];
    cta_gemm<BT>(a, n);
    a = g0;
    a.a = T[5]; a.b = T[0]; a.opb = OP_C; a.d = XG(i);
    cta_gemm<BT>(a, n);
    if (uppers)
      blk_keldysh_combine(n, T[7], T[5], f_l, f_r, -1.0, false, P->gl_upper ? P->gl_upper + o_up : nullptr,
                          P->gg_upper ? P->gg_upper + o_up : nullptr);
    if (P->layer_current) {
      const cplx v = blk_layer_current<BT>(n, T[7], T[5], f_l, f_r, -1.0, uu(i));
      if (threadIdx.x == 0) P->layer_current[e * (nb - 1) + i] = v;
    }
    const int64_t o_d = (e * nb + i) * bb;
    blk_keldysh_combine(n, XL(i), XG(i), f_l, f_r, 1.0, true, P->gl_diag ? P->gl_diag + o_d : nullptr,
                        P->gg_diag ? P->gg_diag + o_d : nullptr);
    if (P->density || P->hole_density) {
      const cplx dh = blk_keldysh_density<BT>(n, XL(i), XG(i), f_l, f_r);
      if (threadIdx.x == 0) {
        if (P->density) P->density[e * nb + i] = dh.x;
        if (P->hole_density) P->hole_density[e * nb + i] = dh.y;
      }
    }
    a = g0;  // G_ii = x_i + P4 x_i
    a.a = T[3]; a.b = XR(i); a.d = spare; a.c = XR(i); a.beta = ONE;
    cta_gemm<BT>(a, n);
    cplx* freed = XR(i);
    g_next = spare;
    spare = freed;
    if (P->gr_diag) blk_axpby(n, ONE, g_next, ONE, nullptr, P->gr_diag + (e * nb + i) * bb);
    if (P->dos) {
      const double v = blk_block_dos<BT>(n, g_next);
      if (threadIdx.x == 0) P->dos[e * nb + i] = v;
    }
  }
  if (P->current_left) {
    blk_keldysh_combine(n, XL(0), XG(0), f_l, f_r, 1.0, true, T[6], T[7]);
    const cplx c1 = blk_trace_product<BT>(n, Cb[6], T[6]);
    const cplx c2 = blk_trace_product<BT>(n, T[7], Cb[4]);
    if (threadIdx.x == 0) P->current_left[e] = cadd(c1, cmul(MONE, c2));
  }
  if (P->transmission) {
    // T = Tr[Gamma_L G_0N Gamma_R G_0N^H]
    a = g0;
    a.a = Cb[8]; a.b = corner; a.d = T[0];
    cta_gemm<BT>(a, n);
    a = g0;
    a.a = T[0]; a.b = Cb[9]; a.d = T[1];
    cta_gemm<BT>(a, n);
    cplx acc = cmk(0, 0);
    for (int q = threadIdx.x; q < n * n; q += blockDim.x) acc = cfma(T[1][q], cconj(corner[q]), acc);
    const cplx tr = cta_sum<BT>(acc);
    if (threadIdx.x == 0) P->transmission[e] = tr.x;
  }
  if (zero && threadIdx.x == 0) {
    atomicOr(flags, 1);
    atomicOr(flags + 1 + pidx, 1);
  }
}

template <int BT>
__global__ void __launch_bounds__(GCfg<BT>::THREADS, GCfg<BT>::MIN_BLOCKS)
    transport_grouped_kernel(const GroupedProblem* problems, int count, int64_t items, unsigned long long* counter,
                             int* flags, cplx* ws, int64_t ws_elems, int max_nb) {
  Misc<BT>* ms = smem_misc<BT>();
  cplx* my_ws = ws + (int64_t)blockIdx.x * ws_elems;
  for (;;) {
    if (threadIdx.x == 0) ms->item = atomicAdd(counter, 1ull);
    __syncthreads();
    const int64_t item = (int64_t)ms->item;
    __syncthreads();
    if (item >= items) break;
    // the problem holding this pair: last one whose first pair is <= item
    int lo = 0, hi = count;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (problems[mid].item0 <= item) lo = mid;
      else hi = mid;
    }
    solve_energy<BT>(problems + lo, lo, item - problems[lo].item0, my_ws, max_nb, flags);
  }
}

// Resident CTAs of the persistent launch on the current device (host
// arithmetic callers such as the footprint query may run without a device:
// then one CTA per SM of a B200 is assumed).
template <int BT>
int resident_ctas() {
  try {
    qtx_opt_in_smem((const void*)transport_grouped_kernel<BT>, smem_bytes<BT>());
  } catch (const QtxError&) {
    cudaGetLastError();
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, transport_grouped_kernel<BT>, GCfg<BT>::THREADS,
                                                    smem_bytes<BT>()) != cudaSuccess) {
    cudaGetLastError();
    per_sm = 1;
  }
  if (per_sm < 1) per_sm = 1;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    sms = 148;
  }
  return per_sm * sms;
}

}  // namespace

int grouped_grid(int b, int64_t items) {
  const int resident = b <= 32 ? resident_ctas<32>() : resident_ctas<64>();
  return (int)(items < resident ? items : resident);
}

int64_t grouped_ws_elems(int max_nb, int b) { return (int64_t)(3 * max_nb + 20) * b * b; }

void launch_transport_grouped(int b, const GroupedProblem* problems, int count, int64_t items,
                              unsigned long long* counter, int* flags, cplx* ws, int64_t ws_elems, int max_nb, int grid,
                              cudaStream_t stream) {
  if (items <= 0 || grid <= 0) return;
  if (b < 1 || b > GROUPED_MAX_B) throw QtxError(QTX_E_UNSUPPORTED, "grouped transport: block size above 64");
  if (b <= 32) {
    qtx_opt_in_smem((const void*)transport_grouped_kernel<32>, smem_bytes<32>());
    transport_grouped_kernel<32><<<grid, GCfg<32>::THREADS, smem_bytes<32>(), stream>>>(problems, count, items, counter, flags, ws,
                                                                         ws_elems, max_nb);
  } else {
    qtx_opt_in_smem((const void*)transport_grouped_kernel<64>, smem_bytes<64>());
    transport_grouped_kernel<64><<<grid, GCfg<64>::THREADS, smem_bytes<64>(), stream>>>(problems, count, items, counter, flags, ws,
                                                                         ws_elems, max_nb);
  }
  qtx_check_launch("transport_grouped_kernel");
}
