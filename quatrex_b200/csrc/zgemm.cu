// Batched complex FP64 GEMM on the sm_100a FP64 tensor path (DMMA,
// mma.sync m16n8k4 f64), the work-horse of every RGF block product.
//
// D = alpha op(A) op(B) + beta C + gamma C2 over a strided batch, op in
// {none, conjugate transpose}.  Complex products use the 4M real
// decomposition on split fragments: Re += Ar Br - Ai Bi, Im += Ar Bi + Ai Br,
// four DMMAs per 16x8 complex tile step.
//
// CTA tile 64x64 (complex), K step 16, double-buffered cp.async pipeline (one
// barrier per 128 DMMAs of a warp; 80 KB, two CTAs per SM), 4 warps each
// owning a 32x32 complex warp tile (2 x 4 DMMA tiles, real and imaginary
// accumulators: 64 doubles per thread).  Tiles stay complex-interleaved in
// shared memory so one 16-byte load yields both parts of an element; the
// padded row strides (20 / 66 complex) make every 8-lane fragment load hit 8
// distinct 16-byte bank groups.
#include "kernels.h"

namespace {

constexpr int BM = 64, BN = 64, BK = 16, STAGES = 2, THREADS = 128;
constexpr int LD_KMAJOR = BK + 4;   // tile stored [row][k]: 20 complex = 320 B rows
constexpr int LD_MMAJOR = BM + 2;   // tile stored [k][row]: 66 complex = 1056 B rows
constexpr int TILE_ELEMS = (BM * LD_KMAJOR > BK * LD_MMAJOR) ? BM * LD_KMAJOR : BK * LD_MMAJOR;
constexpr int SMEM_BYTES = STAGES * 2 * TILE_ELEMS * (int)sizeof(cplx);

__device__ __forceinline__ void dmma(double (&c)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool pred) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int bytes = pred ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

struct Params {
  int m, n, k;
  int64_t batch;
  const cplx* a; int64_t lda, sa;
  const cplx* b; int64_t ldb, sb;
  const cplx* c; int64_t ldc, sc; cplx beta;
  const cplx* c2; int64_t ldc2, sc2; cplx gamma;
  cplx* d; int64_t ldd, sd; cplx alpha;
  const int* active;
  const cplx* diag_shift;
};

// Load one K-slice of op(A) (BM x BK) into shared memory.
template <int OPA>
__device__ __forceinline__ void load_a(cplx* sm, const Params& p, const cplx* a, int m0, int k0, int tid) {
#pragma unroll
  for (int r = 0; r < (BM * BK) / THREADS; ++r) {
    int idx = tid + r * THREADS;
    if (OPA == OP_N) {
      int row = idx / BK, col = idx % BK;  // A stored m x k
      int gm = m0 + row, gk = k0 + col;
      bool ok = gm < p.m && gk < p.k;
      const cplx* src = ok ? a + (int64_t)gm * p.lda + gk : a;
      cp_async16(sm + row * LD_KMAJOR + col, src, ok);
    } else {
      int krow = idx / BM, mcol = idx % BM;  // A stored k x m
      int gk = k0 + krow, gm = m0 + mcol;
      bool ok = gm < p.m && gk < p.k;
      const cplx* src = ok ? a + (int64_t)gk * p.lda + gm : a;
      cp_async16(sm + krow * LD_MMAJOR + mcol, src, ok);
    }
  }
}

// Load one K-slice of op(B) (BK x BN) into shared memory.
template <int OPB>
__device__ __forceinline__ void load_b(cplx* sm, const Params& p, const cplx* b, int n0, int k0, int tid) {
#pragma unroll
  for (int r = 0; r < (BN * BK) / THREADS; ++r) {
    int idx = tid + r * THREADS;
    if (OPB == OP_N) {
      int krow = idx / BN, ncol = idx % BN;  // B stored k x n
      int gk = k0 + krow, gn = n0 + ncol;
      bool ok = gn < p.n && gk < p.k;
      const cplx* src = ok ? b + (int64_t)gk * p.ldb + gn : b;
      cp_async16(sm + krow * LD_MMAJOR + ncol, src, ok);
    } else {
      int nrow = idx / BK, kcol = idx % BK;  // B stored n x k
      int gn = n0 + nrow, gk = k0 + kcol;
      bool ok = gn < p.n && gk < p.k;
      const cplx* src = ok ? b + (int64_t)gn * p.ldb + gk : b;
      cp_async16(sm + nrow * LD_KMAJOR + kcol, src, ok);
    }
  }
}

template <int OPA>
__device__ __forceinline__ cplx frag_a(const cplx* sm, int m, int k) {
  if (OPA == OP_N) return sm[m * LD_KMAJOR + k];
  cplx v = sm[k * LD_MMAJOR + m];
  return make_double2(v.x, -v.y);
}
template <int OPB>
__device__ __forceinline__ cplx frag_b(const cplx* sm, int k, int n) {
  if (OPB == OP_N) return sm[k * LD_MMAJOR + n];
  cplx v = sm[n * LD_KMAJOR + k];
  return make_double2(v.x, -v.y);
}

template <int OPA, int OPB>
__global__ void __launch_bounds__(THREADS, 2) zgemm_dmma_kernel(Params p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx* smem = reinterpret_cast<cplx*>(smem_raw);

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;
  const int wm0 = (warp >> 1) * 32, wn0 = (warp & 1) * 32;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int ktiles = (p.k + BK - 1) / BK;

  for (int64_t e = blockIdx.z; e < p.batch; e += gridDim.z) {
    if (p.active && !p.active[e]) continue;
    const cplx* a = p.a + e * p.sa;
    const cplx* b = p.b + e * p.sb;

    double acc_re[2][4][4], acc_im[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc_re[i][j][q] = acc_im[i][j][q] = 0.0;

#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
      if (s < ktiles) {
        cplx* sa = smem + s * 2 * TILE_ELEMS;
        load_a<OPA>(sa, p, a, m0, s * BK, tid);
        load_b<OPB>(sa + TILE_ELEMS, p, b, n0, s * BK, tid);
      }
      cp_async_commit();
    }

    for (int kt = 0; kt < ktiles; ++kt) {
      cp_async_wait<STAGES - 2>();
      __syncthreads();
      {
        int nk = kt + STAGES - 1;
        if (nk < ktiles) {
          cplx* sa = smem + (nk % STAGES) * 2 * TILE_ELEMS;
          load_a<OPA>(sa, p, a, m0, nk * BK, tid);
          load_b<OPB>(sa + TILE_ELEMS, p, b, n0, nk * BK, tid);
        }
        cp_async_commit();
      }
      const cplx* sa = smem + (kt % STAGES) * 2 * TILE_ELEMS;
      const cplx* sb = sa + TILE_ELEMS;
#pragma unroll
      for (int kk = 0; kk < BK; kk += 4) {
        cplx af[2][2], bf[4];
#pragma unroll
        for (int mi = 0; mi < 2; ++mi) {
          af[mi][0] = frag_a<OPA>(sa, wm0 + mi * 16 + g, kk + t);
          af[mi][1] = frag_a<OPA>(sa, wm0 + mi * 16 + g + 8, kk + t);
        }
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) bf[ni] = frag_b<OPB>(sb, kk + t, wn0 + ni * 8 + g);
        // first product of every accumulator, then the second (the order
        // within each accumulator is unchanged: Ar Br, -Ai Bi / Ar Bi, Ai Br)
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
    }
    cp_async_wait<0>();
    __syncthreads();

    // Epilogue: D = alpha acc + beta C + gamma C2
    cplx* d = p.d + e * p.sd;
    const cplx* c = p.c ? p.c + e * p.sc : nullptr;
    const cplx* c2 = p.c2 ? p.c2 + e * p.sc2 : nullptr;
#pragma unroll
    for (int mi = 0; mi < 2; ++mi) {
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          int row = m0 + wm0 + mi * 16 + g + ((q >> 1) << 3);
          int col = n0 + wn0 + ni * 8 + 2 * t + (q & 1);
          if (row < p.m && col < p.n) {
            cplx v = cmul(p.alpha, cmk(acc_re[mi][ni][q], acc_im[mi][ni][q]));
            if (c) v = cfma(p.beta, c[(int64_t)row * p.ldc + col], v);
            if (c2) v = cfma(p.gamma, c2[(int64_t)row * p.ldc2 + col], v);
            if (p.diag_shift && row == col) v = cadd(v, p.diag_shift[e]);
            d[(int64_t)row * p.ldd + col] = v;
          }
        }
      }
    }
  }
}

template <int OPA, int OPB>
void launch_t(const Params& p, cudaStream_t stream) {
  // opt-in to the large shared-memory carve-out (per device)
  qtx_opt_in_smem((const void*)zgemm_dmma_kernel<OPA, OPB>, SMEM_BYTES);
  dim3 grid(ceil_div_u(p.n, BN), ceil_div_u(p.m, BM), (unsigned)(p.batch < 65535 ? p.batch : 65535));
  zgemm_dmma_kernel<OPA, OPB><<<grid, THREADS, SMEM_BYTES, stream>>>(p);
}

}  // namespace

void launch_zgemm(const GemmCall& g, cudaStream_t stream) {
  if (g.m <= 0 || g.n <= 0 || g.batch <= 0) return;
  Params p;
  p.m = g.m; p.n = g.n; p.k = g.k; p.batch = g.batch;
  p.a = g.a.ptr; p.lda = g.a.ld; p.sa = g.a.stride;
  p.b = g.b.ptr; p.ldb = g.b.ld; p.sb = g.b.stride;
  p.c = g.c.ptr; p.ldc = g.c.ld; p.sc = g.c.stride; p.beta = g.beta;
  p.c2 = g.c2.ptr; p.ldc2 = g.c2.ld; p.sc2 = g.c2.stride; p.gamma = g.gamma;
  p.d = g.d.ptr; p.ldd = g.d.ld; p.sd = g.d.stride; p.alpha = g.alpha;
  p.active = g.active;
  p.diag_shift = g.diag_shift;
  if (g.op_a == OP_N && g.op_b == OP_N) launch_t<OP_N, OP_N>(p, stream);
  else if (g.op_a == OP_N && g.op_b == OP_C) launch_t<OP_N, OP_C>(p, stream);
  else if (g.op_a == OP_C && g.op_b == OP_N) launch_t<OP_C, OP_N>(p, stream);
  else launch_t<OP_C, OP_C>(p, stream);
  qtx_check_launch("zgemm_dmma_kernel");
}
