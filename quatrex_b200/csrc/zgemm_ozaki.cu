// Mixed-precision complex GEMM: FP64 operands split into signed 7-bit slices
// (Ozaki scheme) whose pairwise products run on the INT8 tensor cores
// (tcgen05.mma kind::i8) with exact INT32 accumulation in tensor memory.
//
// Splitting.  Row m of op(A) gets the exponent E_m with max_k max(|Re|, |Im|)
// < 2^E_m * 127/128; every part x of the row is written as
// x = 2^E_m sum_{s=1..S} q_s 128^-s + r, q_s = nearest integer of successive
// 128x remainders, |q_1| <= 127, |q_s| <= 64 for s >= 2, |r| <= 2^E_m 128^-S / 2.
// Columns of op(B) likewise with exponents F_n.  The products q_s(A) q_t(B) are
// exact in INT32 and so are their sums over K and over the slice pairs of one
// level L = s + t (at most 2 * 127 * 64 + (L - 3) * 64^2 per k for L >= 3,
// 127^2 for L = 2: below 2^31 for K <= 16384 and S <= 8).  The kernel keeps
// every pair with s + t <= S + 1 (the dropped pairs are below the slice
// truncation), one TMEM accumulator per level and part (Re, Im), and combines
// them once in FP64:
//   C_mn = 2^(E_m + F_n) sum_L 128^-L acc_L[m][n].
// Complex products: [Re | Im] = Ar [Br | Bi] + Ai [-Bi | Br].
//
// Layout.  The split kernels write each (tile, K-chunk) block in the exact
// shared-memory image the UMMA descriptors read (K-major, no swizzle, 8-row x
// 16-byte core matrices, K-adjacent cores 128 B apart, 8-row groups 256 B
// apart), so one pipeline stage is a single 1-D bulk copy per operand.
//
// Tile 128 x 32 outputs, K chunk 32, S <= 8 slices (8 by default): a stage
// holds 2 S 4 KiB of A and 4 S 1 KiB of B; two stages for S >= 7, three below.
// TMEM: level l holds [Re | Im] at columns [64 l, 64 l + 64) (all 512 columns
// at S = 8).  For a fixed A slice s, two MMAs (Ar^(s) against [Br | Bi],
// Ai^(s) against [-Bi | Br]) over all partner B slices (stored contiguously)
// fill the accumulators of levels s - 1 .. S - 1.
// Every mbarrier wait is bounded; a wait that gives up sets an error flag, the
// remaining work is skipped and the tensor memory is released before exit.
#include <algorithm>
#include <cstdlib>

#include <mutex>

#include "kernels.h"

namespace {

constexpr int TM = 128, TN = 32, KC = 32;
constexpr int MAX_S = 8;
constexpr int THREADS = 160;  // warps 0-3 drain, warp 4 loads and issues MMAs
constexpr int MAX_STAGES = 4;
constexpr int MAX_SMEM = 227 * 1024;  // dynamic shared memory a CTA may opt into
constexpr int BAR_BYTES = 256;        // barrier words behind the stages
constexpr uint32_t TMEM_COLS = 512;
constexpr unsigned long long WAIT_NS = 2000000000ull;  // give up a wait after 2 s

// set by any CTA whose pipeline wait gave up; read and cleared by mixed_check_error()
__device__ int g_mixed_wait_error = 0;

// A chunk block: parts Ar, Ai, each S slices of TM x KC bytes.
// B chunk block: two concatenations, each S slices of 2 TN x KC bytes:
//   cat 0, slice t: rows [0, TN) = Br^(t), rows [TN, 2 TN) = Bi^(t)
//   cat 1, slice t: rows [0, TN) = -Bi^(t), rows [TN, 2 TN) = Br^(t)
// so Ar^(s) x cat0 accumulates [Ar Br | Ar Bi] and Ai^(s) x cat1 accumulates
// [-Ai Bi | Ai Br] into the same [Re | Im] TMEM columns.
__host__ __device__ inline int a_block_bytes(int S) { return 2 * S * TM * KC; }
__host__ __device__ inline int b_block_bytes(int S) { return 2 * S * 2 * TN * KC; }

// byte offset of (row, k) inside one 8-row-group-tiled operand slice
__device__ __forceinline__ int core_off(int row, int k) {
  return (row >> 3) * 256 + (k >> 4) * 128 + (row & 7) * 16 + (k & 15);
}

// ---------------------------------------------------------------------------
// split kernel
// ---------------------------------------------------------------------------
// Two kernels split an operand into slices, one per memory layout.  Both cover
// a group of consecutive rows of one batch entry (rows of op(A), or columns of
// op(B)) and all of K, in chunks of KC k; the element (i, k) is
// base[i * si + k * sk], conjugated when `conj`.  Pass 1 reduces each row's
// exponent E (max < 2^E * 127/128, so that the first rounded slice stays in
// [-127, 127]); pass 2 re-reads the rows (L2-resident by then), writes the
// chunk's slices into shared memory in the UMMA image and copies the chunk out
// with 16-byte stores.  NPARTS = 2: the A operand (Ar, Ai); NPARTS = 4: the B
// operand (two concatenations, see b_block_bytes).
//
// Slice s is the nearest integer of 128 x (remainder of slice s - 1), taken
// with the 1.5 * 2^52 shift on the FP64 adder (exact for |v| < 2^51; the
// integer is the low word): |q_1| <= 127, |q_s| <= 64 after.
constexpr double SPLIT_RND = 6755399441055744.0;

// E of a row from its max |Re|, |Im|: 2^(E-1) <= max, max < 2^E * 127/128.
__device__ __forceinline__ int split_exponent(double mx) {
  int E = 0;
  if (mx > 0) {
    const double mant = frexp(mx, &E);
    if (mant >= 127.0 / 128.0) ++E;
  }
  return E;
}

// Rows adjacent in memory: a block takes 32 rows; warp w of a chunk takes rows
// 8 (w / 2) .. + 7 and k 16 (w % 2) .. + 15, lane l row l % 8 of those and the 4
// consecutive k from 4 (l / 8), so every load of a warp reads 4 runs of 8
// consecutive rows; the 4 slice bytes of a thread are packed into one 32-bit
// word per slice and part and stored conflict-free (32 rows = 1 KiB per slice
// and part).
constexpr int SPLIT_ROWS = 32;

template <int S, int NPARTS>
__global__ void __launch_bounds__(256) ozaki_split_rows_kernel(int R, int K, int64_t batch, const cplx* base, int64_t si,
                                                          int64_t sk, int64_t sb, int conj, int KT, int TR, int* expo,
                                                          signed char* out) {
  constexpr int NSEG = NPARTS * S;  // 1 KiB segments per chunk: A 2S, B 4S
  __shared__ __align__(16) uint32_t stage[NSEG * 256];
  __shared__ double wmax[8][8];
  __shared__ double rscale[SPLIT_ROWS];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int Rt = (R + TR - 1) / TR;
  const int64_t rblocks = (int64_t)Rt * (TR / SPLIT_ROWS);
  const int blk_bytes = (NPARTS == 2 ? 2 * S * TR * KC : 2 * S * 2 * TR * KC);
  const int rr = (warp >> 1) * 8 + (lane & 7);         // row within the block
  const int k0 = (warp & 1) * 16 + (lane >> 3) * 4;    // first of 4 k within the chunk
  const int woff = core_off(rr, k0) >> 2;              // word offset within a 1 KiB segment
  for (int64_t blk = blockIdx.x; blk < batch * rblocks; blk += gridDim.x) {
    const int64_t e = blk / rblocks;
    const int r0 = (int)(blk % rblocks) * SPLIT_ROWS;
    const int i = r0 + rr;
    const cplx* row = base + e * sb + (int64_t)i * si;
    // pass 1: row maxima
    double m = 0.0;
    if (i < R) {
      for (int kc = 0; kc < KT; ++kc) {
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          const int k = kc * KC + k0 + jj;
          if (k < K) {
            const cplx v = row[(int64_t)k * sk];
            m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
          }
        }
      }
    }
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, 8));
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, 16));
    if (lane < 8) wmax[warp][lane] = m;
    __syncthreads();
    if (tid < SPLIT_ROWS) {
      const int rh = tid >> 3, rl = tid & 7;
      const double mx = fmax(wmax[2 * rh][rl], wmax[2 * rh + 1][rl]);
      const int E = split_exponent(mx);
      if (r0 + tid < R) expo[e * R + r0 + tid] = E;
      rscale[tid] = ldexp(1.0, -E);
    }
    __syncthreads();
    const double scale = rscale[rr];
    // pass 2: slices, chunk by chunk
    const int it = r0 / TR, rin = r0 % TR;
    for (int kc = 0; kc < KT; ++kc) {
      uint32_t wr[S], wi[S], wn[S];
#pragma unroll
      for (int sl = 0; sl < S; ++sl) wr[sl] = wi[sl] = wn[sl] = 0;
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) {
        const int k = kc * KC + k0 + jj;
        const cplx v = (i < R && k < K) ? row[(int64_t)k * sk] : cmk(0, 0);
        double re = v.x * scale;
        double im = (conj ? -v.y : v.y) * scale;
#pragma unroll
        for (int sl = 0; sl < S; ++sl) {
          const double vr = re * 128.0, vi = im * 128.0;
          const double yr = vr + SPLIT_RND, yi = vi + SPLIT_RND;
          re = vr - (yr - SPLIT_RND);
          im = vi - (yi - SPLIT_RND);
          const int qr = __double2loint(yr), qi = __double2loint(yi);
          wr[sl] |= (uint32_t)(qr & 0xFF) << (8 * jj);
          wi[sl] |= (uint32_t)(qi & 0xFF) << (8 * jj);
          if (NPARTS == 4) wn[sl] |= (uint32_t)((-qi) & 0xFF) << (8 * jj);
        }
      }
#pragma unroll
      for (int sl = 0; sl < S; ++sl) {
        if (NPARTS == 2) {
          // A: Ar slices, then Ai slices
          stage[(0 * S + sl) * 256 + woff] = wr[sl];
          stage[(1 * S + sl) * 256 + woff] = wi[sl];
        } else {
          // B: cat 0 = [Br | Bi], cat 1 = [-Bi | Br]; segment 2 (c S + sl) + half
          stage[((0 * S + sl) * 2 + 0) * 256 + woff] = wr[sl];
          stage[((0 * S + sl) * 2 + 1) * 256 + woff] = wi[sl];
          stage[((1 * S + sl) * 2 + 0) * 256 + woff] = wn[sl];
          stage[((1 * S + sl) * 2 + 1) * 256 + woff] = wr[sl];
        }
      }
      __syncthreads();
      signed char* g = out + ((e * Rt + it) * (int64_t)KT + kc) * blk_bytes + (rin >> 3) * 256;
      for (int q = tid; q < NSEG * 64; q += 256) {
        const int seg = q >> 6, w16 = q & 63;
        const int64_t goff = (NPARTS == 2) ? (int64_t)seg * TR * KC
                                           : (int64_t)(seg >> 1) * 2 * TR * KC + (seg & 1) * (TR / 8) * 256;
        *reinterpret_cast<int4*>(g + goff + w16 * 16) = *reinterpret_cast<const int4*>(stage + seg * 256 + w16 * 4);
      }
      __syncthreads();
    }
  }
}

// k adjacent in memory: a block takes 16 rows; element q of a chunk (thread q
// and q + 256) is row q / 32, k q % 32, so every load of a warp reads 32
// consecutive k of one row; the slice bytes go to shared memory one by one.
constexpr int SPLIT_KROWS = 16;

template <int S, int NPARTS>
__global__ void __launch_bounds__(256) ozaki_split_k_kernel(int R, int K, int64_t batch, const cplx* base, int64_t si,
                                                            int64_t sk, int64_t sb, int conj, int KT, int TR,
                                                            int* expo, signed char* out) {
  constexpr int NSEG = NPARTS * S;  // 512-byte segments per chunk (16 rows)
  __shared__ __align__(16) signed char stage[NSEG * 512];
  __shared__ double rscale[SPLIT_KROWS];
  __shared__ double wmax[SPLIT_KROWS];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int Rt = (R + TR - 1) / TR;
  const int64_t rblocks = (int64_t)Rt * (TR / SPLIT_KROWS);
  const int blk_bytes = (NPARTS == 2 ? 2 * S * TR * KC : 2 * S * 2 * TR * KC);
  // a warp holds rows warp and warp + 8, one k per lane
  const int rr0 = warp, rr1 = warp + 8, kk = lane;
  for (int64_t blk = blockIdx.x; blk < batch * rblocks; blk += gridDim.x) {
    const int64_t e = blk / rblocks;
    const int r0 = (int)(blk % rblocks) * SPLIT_KROWS;
    const cplx* mat = base + e * sb;
    double m0 = 0.0, m1 = 0.0;
    for (int kc = 0; kc < KT; ++kc) {
      const int k = kc * KC + kk;
      if (k < K) {
        if (r0 + rr0 < R) {
          const cplx v = mat[(int64_t)(r0 + rr0) * si + (int64_t)k * sk];
          m0 = fmax(m0, fmax(fabs(v.x), fabs(v.y)));
        }
        if (r0 + rr1 < R) {
          const cplx v = mat[(int64_t)(r0 + rr1) * si + (int64_t)k * sk];
          m1 = fmax(m1, fmax(fabs(v.x), fabs(v.y)));
        }
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      m0 = fmax(m0, __shfl_xor_sync(0xffffffffu, m0, off));
      m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, off));
    }
    if (lane == 0) {
      wmax[rr0] = m0;
      wmax[rr1] = m1;
    }
    __syncthreads();
    if (tid < SPLIT_KROWS) {
      const int E = split_exponent(wmax[tid]);
      if (r0 + tid < R) expo[e * R + r0 + tid] = E;
      rscale[tid] = ldexp(1.0, -E);
    }
    __syncthreads();
    const int it = r0 / TR, rin = r0 % TR;
    for (int kc = 0; kc < KT; ++kc) {
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int rr = j ? rr1 : rr0;
        const int i = r0 + rr, k = kc * KC + kk;
        const cplx v = (i < R && k < K) ? mat[(int64_t)i * si + (int64_t)k * sk] : cmk(0, 0);
        double re = v.x * rscale[rr];
        double im = (conj ? -v.y : v.y) * rscale[rr];
        const int off = core_off(rr, kk);
#pragma unroll
        for (int sl = 0; sl < S; ++sl) {
          const double vr = re * 128.0, vi = im * 128.0;
          const double yr = vr + SPLIT_RND, yi = vi + SPLIT_RND;
          re = vr - (yr - SPLIT_RND);
          im = vi - (yi - SPLIT_RND);
          const int qr = __double2loint(yr), qi = __double2loint(yi);
          if (NPARTS == 2) {
            stage[(0 * S + sl) * 512 + off] = (signed char)qr;
            stage[(1 * S + sl) * 512 + off] = (signed char)qi;
          } else {
            stage[((0 * S + sl) * 2 + 0) * 512 + off] = (signed char)qr;
            stage[((0 * S + sl) * 2 + 1) * 512 + off] = (signed char)qi;
            stage[((1 * S + sl) * 2 + 0) * 512 + off] = (signed char)(-qi);
            stage[((1 * S + sl) * 2 + 1) * 512 + off] = (signed char)qr;
          }
        }
      }
      __syncthreads();
      signed char* g = out + ((e * Rt + it) * (int64_t)KT + kc) * blk_bytes + (rin >> 3) * 256;
      for (int q = tid; q < NSEG * 32; q += 256) {
        const int seg = q >> 5, w16 = q & 31;
        const int64_t goff = (NPARTS == 2) ? (int64_t)seg * TR * KC
                                           : (int64_t)(seg >> 1) * 2 * TR * KC + (seg & 1) * (TR / 8) * 256;
        *reinterpret_cast<int4*>(g + goff + w16 * 16) = *reinterpret_cast<const int4*>(stage + seg * 512 + w16 * 16);
      }
      __syncthreads();
    }
  }
}

template <int NPARTS>
void launch_split(int S, cudaStream_t stream, int R, int K, int64_t batch, const cplx* base, int64_t si, int64_t sk,
                  int64_t sb, int conj, bool rows_adjacent, int KT, int TR, int* expo, signed char* out) {
  const int rows = rows_adjacent ? SPLIT_ROWS : SPLIT_KROWS;
  const int64_t rblocks = (int64_t)((R + TR - 1) / TR) * (TR / rows);
  const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(batch * rblocks, 148 * 16));
#define QTX_SPLIT_CASE(SS)                                                                                      \
  case SS:                                                                                                     \
    if (rows_adjacent)                                                                                         \
      ozaki_split_rows_kernel<SS, NPARTS><<<grid, 256, 0, stream>>>(R, K, batch, base, si, sk, sb, conj, KT, TR, \
                                                                    expo, out);                                \
    else                                                                                                       \
      ozaki_split_k_kernel<SS, NPARTS><<<grid, 256, 0, stream>>>(R, K, batch, base, si, sk, sb, conj, KT, TR,    \
                                                                 expo, out);                                   \
    break;
  switch (S) {
    QTX_SPLIT_CASE(2)
    QTX_SPLIT_CASE(3)
    QTX_SPLIT_CASE(4)
    QTX_SPLIT_CASE(5)
    QTX_SPLIT_CASE(6)
    QTX_SPLIT_CASE(7)
    QTX_SPLIT_CASE(8)
    default:
      throw QtxError(QTX_E_INVAL, "mixed-precision GEMM: slice count outside 2..8");
  }
#undef QTX_SPLIT_CASE
  qtx_check_launch("ozaki_split_kernel");
}

// ---------------------------------------------------------------------------
// tcgen05 helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Exact int32 -> double on the FP64 adder: the bit pattern 0x43300000:(v + 2^31)
// is 2^52 + 2^31 + v.
__device__ __forceinline__ double i32_to_f64(int v) {
  return __hiloint2double(0x43300000, v ^ (int)0x80000000) - 4503601774854144.0;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Wait on a phase parity for at most WAIT_NS, or until *abort is set; returns
// false if it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, const volatile int* abort = nullptr) {
  const uint32_t addr = smem_u32(bar);
  const unsigned long long t0 = global_ns();
  for (unsigned it = 0;; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if ((it & 255) == 255) {
      if (abort && *abort) return false;
      if (global_ns() - t0 > WAIT_NS) return false;
    }
  }
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void bulk_prefetch_l2(const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ uint64_t smem_desc(const void* p) {
  // K-major, no swizzle: LBO = 128 B (K-adjacent core matrices), SBO = 256 B
  // (adjacent 8-row groups), version 1 (bits 46-47), layout type 0.
  uint64_t addr = (smem_u32(p) >> 4) & 0x3FFF;
  uint64_t lbo = (128 >> 4) & 0x3FFF;
  uint64_t sbo = (256 >> 4) & 0x3FFF;
  return addr | (lbo << 16) | (sbo << 32) | (1ull << 46);
}

__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, int (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,"
      "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
        "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

struct OzParams {
  int M, N, K, S, KT, Mt, Nt;
  int64_t batch;
  const signed char* as;
  const signed char* bs;
  const int* ea;
  const int* eb;
  const cplx* c; int64_t ldc, sc; cplx beta;
  const cplx* c2; int64_t ldc2, sc2; cplx gamma;
  cplx* d; int64_t ldd, sd; cplx alpha;
  const int* active;
  const cplx* diag_shift;
  int* error_flag;
  int a_shared, b_shared;  // operand sliced once for every batch entry
  int nst;                 // pipeline stages (2..MAX_STAGES), as many as fit in shared memory
};

// Persistent: one CTA per SM loops over output tiles (n-tile fastest, so
// co-resident CTAs share the A block in L2).  Warp 4 lane 0 streams the chunk
// blocks (two-stage ring, continuing across tiles) and issues the MMAs; warps
// 0-3 drain the accumulators of a finished tile (warp w reads TMEM lanes
// 32w..32w+31), release the tensor memory with tmem_empty and then write the
// FP64 results while the next tile's MMAs already run.
__global__ void __launch_bounds__(THREADS, 1) ozaki_gemm_kernel(OzParams p) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const int S = p.S;
  const int abytes = a_block_bytes(S), bbytes = b_block_bytes(S);
  const int stage_bytes = ((abytes + bbytes + 1023) / 1024) * 1024;
  unsigned char* stage0 = smem_raw;
  const int NST = p.nst;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + NST * stage_bytes);
  uint64_t* empty = full + MAX_STAGES;
  uint64_t* tmem_full = empty + MAX_STAGES;
  uint64_t* tmem_empty = tmem_full + 1;
  uint64_t* all_done = tmem_empty + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(all_done + 1);
  int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t tiles_per_e = (int64_t)p.Mt * p.Nt;
  const int64_t ntiles = p.batch * tiles_per_e;

  if (tid == 0) {
    for (int q = 0; q < NST; ++q) {
      mbar_init(&full[q], 1);
      mbar_init(&empty[q], 1);
    }
    mbar_init(tmem_full, 1);
    mbar_init(tmem_empty, 128);
    mbar_init(all_done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  volatile int* abort_v = abort_flag;
  // kind::i8 instruction descriptor: D = S32 (bits 4-5), A = B = signed 8-bit
  // (bits 7-9, 10-12), both K-major, M = 128 (bits 24-28); N (bits 17-22) per MMA
  const uint32_t idesc_base = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TM >> 4) << 24);

  if (warp == 4) {
    if (lane == 0) {
      bool ok = true;
      int64_t issued = 0, consumed = 0;  // chunk loads issued / waited for (global chunk counter)
      const int64_t my_tiles = (ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x;
      const int64_t total = my_tiles * p.KT;
      auto chunk_src = [&](int64_t c, const signed char*& a, const signed char*& b) {
        const int64_t tile = blockIdx.x + (c / p.KT) * (int64_t)gridDim.x;
        const int kc = (int)(c % p.KT);
        const int64_t e = tile / tiles_per_e;
        const int rem = (int)(tile % tiles_per_e);
        const int mt = rem / p.Nt, nt = rem % p.Nt;
        const int64_t ea_i = p.a_shared ? 0 : e, eb_i = p.b_shared ? 0 : e;
        a = p.as + (((ea_i * p.Mt + mt) * (int64_t)p.KT) + kc) * abytes;
        b = p.bs + (((eb_i * p.Nt + nt) * (int64_t)p.KT) + kc) * bbytes;
      };
      auto load = [&](int64_t c) {
        const signed char *a, *b;
        chunk_src(c, a, b);
        const int q = (int)(c % NST);
        unsigned char* st = stage0 + q * stage_bytes;
        mbar_expect_tx(&full[q], (uint32_t)(abytes + bbytes));
        bulk_g2s(st, a, (uint32_t)abytes, &full[q]);
        bulk_g2s(st + abytes, b, (uint32_t)bbytes, &full[q]);
        issued = c + 1;
      };
      auto prefetch = [&](int64_t c) {
        if (c >= total) return;
        const signed char *a, *b;
        chunk_src(c, a, b);
        bulk_prefetch_l2(a, (uint32_t)abytes);
        bulk_prefetch_l2(b, (uint32_t)bbytes);
      };
      // every stage filled up front, the next few chunk blocks on their way into L2
      for (int64_t c = NST; c <= NST + 2; ++c) prefetch(c);
      for (int64_t c = 0; c < NST && c < total; ++c) load(c);
      for (int64_t c = 0; c < total && ok; ++c) {
        const int st = (int)(c % NST);
        const int64_t j = c / p.KT;  // local tile index
        const int kc = (int)(c % p.KT);
        ok = mbar_wait(&full[st], (uint32_t)((c / NST) & 1), abort_v);
        if (!ok) break;
        consumed = c + 1;
        if (kc == 0 && j >= 1) {
          // the accumulators of the previous tile have been read out
          ok = mbar_wait(tmem_empty, (uint32_t)((j - 1) & 1), abort_v);
          if (!ok) break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const unsigned char* abase = stage0 + st * stage_bytes;
        const unsigned char* bbase = abase + abytes;
        // For slice s of A the partner slices t = 1..S+1-s of B are contiguous in
        // shared memory and their levels l = s+t-2 = s-1..S-1 are contiguous
        // [Re | Im] TMEM column blocks of width 2 TN, so Ar^(s) x cat0 and
        // Ai^(s) x cat1 over N = 2 TN (S+1-s) cover every pair of slice s
        // (issued in pieces of at most 256 columns).
        for (int sa = 1; sa <= S; ++sa) {
          const uint32_t first = (kc == 0 && sa == 1) ? 0u : 1u;
          const uint64_t ar = smem_desc(abase + (0 * S + sa - 1) * TM * KC);
          const uint64_t ai = smem_desc(abase + (1 * S + sa - 1) * TM * KC);
          const int ncols = 2 * TN * (S + 1 - sa);
          for (int c0 = 0; c0 < ncols; c0 += 256) {
            const uint32_t n = (uint32_t)min(256, ncols - c0);
            const uint32_t idesc_s = idesc_base | ((n >> 3) << 17);
            const uint32_t d = tmem + (uint32_t)((sa - 1) * 2 * TN + c0);
            // B rows [c0, c0 + n) of the stacked slices start c0 rows into the block
            const int boff = (c0 / 8) * 256;
            const uint64_t b0 = smem_desc(bbase + 0 * S * 2 * TN * KC + boff);
            const uint64_t b1 = smem_desc(bbase + 1 * S * 2 * TN * KC + boff);
            umma_i8(d, ar, b0, idesc_s, first);
            umma_i8(d, ai, b1, idesc_s, 1u);
          }
        }
        umma_commit(&empty[st]);
        if (kc == p.KT - 1) umma_commit(tmem_full);
        // Refill the stage of chunk c - 1 with chunk c - 1 + NST once its MMAs
        // are done.  The MMAs of chunk c are already queued behind them, so the
        // tensor pipe stays busy while this thread waits and copies.
        const int64_t cn = c - 1 + NST;
        if (c >= 1 && cn < total) {
          ok = mbar_wait(&empty[(c - 1) % NST], (uint32_t)(((c - 1) / NST) & 1), abort_v);
          if (!ok) break;
          load(cn);
          prefetch(cn + 3);
        }
      }
      if (!ok) {
        *abort_v = 1;
        atomicExch(&g_mixed_wait_error, 1);
        // let the bulk copies already issued land before the CTA can exit
        for (int64_t c = consumed; c < issued; ++c) mbar_wait(&full[c % NST], (uint32_t)((c / NST) & 1));
      }
      // completes once every MMA issued above has finished
      umma_commit(all_done);
      mbar_wait(all_done, 0);
    }
    __syncwarp();
  } else {
    // ---- drain warps 0-3
    const int64_t my_tiles = (ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x;
    for (int64_t j = 0; j < my_tiles; ++j) {
      const int64_t tile = blockIdx.x + j * (int64_t)gridDim.x;
      const int64_t e = tile / tiles_per_e;
      const int rem = (int)(tile % tiles_per_e);
      const int mt = rem / p.Nt, nt = rem % p.Nt;
      const bool ok = mbar_wait(tmem_full, (uint32_t)(j & 1), abort_v);
      if (!ok) {
        if (lane == 0) atomicExch(&g_mixed_wait_error, 1);
        *abort_v = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      double acc_re[TN], acc_im[TN];
#pragma unroll
      for (int jj = 0; jj < TN; ++jj) acc_re[jj] = acc_im[jj] = 0.0;
      for (int l = 0; l < S; ++l) {
        const double scale = ldexp(1.0, -7 * (l + 2));
        int v[32];
        tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(l * 2) * TN, v);
#pragma unroll
        for (int jj = 0; jj < TN; ++jj) acc_re[jj] = fma(i32_to_f64(v[jj]), scale, acc_re[jj]);
        tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(l * 2 + 1) * TN, v);
#pragma unroll
        for (int jj = 0; jj < TN; ++jj) acc_im[jj] = fma(i32_to_f64(v[jj]), scale, acc_im[jj]);
      }
      // accumulators read: the next tile's MMAs may overwrite them
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(tmem_empty)) : "memory");
      if (p.active && !p.active[e]) continue;
      const int row = mt * TM + warp * 32 + lane;
      if (row < p.M) {
        const int ea = p.ea[(p.a_shared ? 0 : e) * p.M + row];
        cplx* d = p.d + e * p.sd + (int64_t)row * p.ldd;
        const cplx* c = p.c ? p.c + e * p.sc + (int64_t)row * p.ldc : nullptr;
        const cplx* c2 = p.c2 ? p.c2 + e * p.sc2 + (int64_t)row * p.ldc2 : nullptr;
#pragma unroll
        for (int jj = 0; jj < TN; ++jj) {
          const int col = nt * TN + jj;
          if (col < p.N) {
            const int ex = ea + p.eb[(p.b_shared ? 0 : e) * p.N + col];
            cplx v;
            if (ex >= -1022 && ex <= 1023) {
              // 2^ex from its bit pattern: one multiply, the same rounding as ldexp
              const double sc = __longlong_as_double((long long)(ex + 1023) << 52);
              v = cmk(acc_re[jj] * sc, acc_im[jj] * sc);
            } else {
              v = cmk(ldexp(acc_re[jj], ex), ldexp(acc_im[jj], ex));
            }
            v = cmul(p.alpha, v);
            if (c) v = cfma(p.beta, c[col], v);
            if (c2) v = cfma(p.gamma, c2[col], v);
            if (p.diag_shift && row == col) v = cadd(v, p.diag_shift[e]);
            d[col] = v;
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

// Slices per operand.  8 by default: a product is then accurate to ~1e-15
// relative (FP64 class) and the transport observables of the nb = 64, b = 256
// device stay within 1e-10 of the FP64 form; with 7 slices the products are
// ~1e-14 and the density error reaches ~1e-8 on that device.
// QTX_OZAKI_SLICES overrides it (2..8).
int ozaki_slices() {
  static int s = [] {
    const char* env = getenv("QTX_OZAKI_SLICES");
    int v = env ? atoi(env) : 8;
    return v < 2 ? 2 : (v > MAX_S ? MAX_S : v);
  }();
  return s;
}

}  // namespace

bool mixed_supported(const GemmCall& g) { return g.k > 0 && g.k <= 16384; }

size_t mixed_workspace_bytes(int m, int n, int k, int64_t a_batch, int64_t b_batch) {
  const int S = ozaki_slices();
  const int KT = (k + KC - 1) / KC;
  const int Mt = (m + TM - 1) / TM, Nt = (n + TN - 1) / TN;
  return (size_t)a_batch * Mt * KT * a_block_bytes(S) + (size_t)b_batch * Nt * KT * b_block_bytes(S) +
         sizeof(int) * (size_t)(a_batch * m + b_batch * n) + 1024;
}

void mixed_check_error(cudaStream_t stream) {
  int flag = 0;
  QTX_CUDA_TRY(cudaMemcpyFromSymbolAsync(&flag, g_mixed_wait_error, sizeof(int), 0, cudaMemcpyDeviceToHost, stream));
  QTX_CUDA_TRY(cudaStreamSynchronize(stream));
  if (flag) {
    const int zero = 0;
    QTX_CUDA_TRY(cudaMemcpyToSymbolAsync(g_mixed_wait_error, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, stream));
    QTX_CUDA_TRY(cudaStreamSynchronize(stream));
    throw QtxError(QTX_E_TIMEOUT, "mixed-precision GEMM: a pipeline wait gave up (results invalid)");
  }
}

void launch_zgemm_mixed(const GemmCall& g, cudaStream_t stream) {
  if (g.m <= 0 || g.n <= 0 || g.batch <= 0) return;
  const int S = ozaki_slices();
  const int KT = (g.k + KC - 1) / KC;
  const int Mt = (g.m + TM - 1) / TM, Nt = (g.n + TN - 1) / TN;
  // an operand with batch stride 0 is the same matrix for every entry: slice it once
  const int64_t a_batch = g.a.stride == 0 ? 1 : g.batch;
  const int64_t b_batch = g.b.stride == 0 ? 1 : g.batch;
  const size_t abytes = (size_t)a_batch * Mt * KT * a_block_bytes(S);
  const size_t bbytes = (size_t)b_batch * Nt * KT * b_block_bytes(S);
  const size_t ebytes = sizeof(int) * (size_t)(a_batch * g.m + b_batch * g.n) + sizeof(int);
  unsigned char* buf = static_cast<unsigned char*>(qtx_malloc_async(abytes + bbytes + ebytes + 512, stream));
  if (!buf) {
    throw QtxError(QTX_E_NOMEM, "mixed-precision GEMM: slice buffer allocation failed");
  }
  signed char* as = reinterpret_cast<signed char*>(buf);
  signed char* bs = as + abytes;
  int* ea = reinterpret_cast<int*>(bs + bbytes);
  int* eb = ea + a_batch * g.m;
  int* eflag = eb + b_batch * g.n;
  {
    // op(A)[m][k]: op N -> a[m * lda + k] (k adjacent); op C -> conj(a[k * lda + m]) (m adjacent)
    const bool a_n = g.op_a == OP_N;
    const int64_t asi = a_n ? g.a.ld : 1, ask = a_n ? 1 : g.a.ld;
    // op(B)[k][n]: op N -> b[k * ldb + n] (n adjacent); op C -> conj(b[n * ldb + k]) (k adjacent)
    const bool b_n = g.op_b == OP_N;
    const int64_t bsi = b_n ? 1 : g.b.ld, bsk = b_n ? g.b.ld : 1;
    // rows of op(A) are adjacent in memory for op C, rows of op(B)^T (columns of op(B)) for op N
    launch_split<2>(S, stream, g.m, g.k, a_batch, g.a.ptr, asi, ask, g.a.stride, a_n ? 0 : 1, !a_n, KT, TM, ea, as);
    launch_split<4>(S, stream, g.n, g.k, b_batch, g.b.ptr, bsi, bsk, g.b.stride, b_n ? 0 : 1, b_n, KT, TN, eb, bs);
  }
  OzParams p;
  p.M = g.m; p.N = g.n; p.K = g.k; p.S = S; p.KT = KT; p.Mt = Mt; p.Nt = Nt; p.batch = g.batch;
  p.as = as; p.bs = bs; p.ea = ea; p.eb = eb;
  p.c = g.c.ptr; p.ldc = g.c.ld; p.sc = g.c.stride; p.beta = g.beta;
  p.c2 = g.c2.ptr; p.ldc2 = g.c2.ld; p.sc2 = g.c2.stride; p.gamma = g.gamma;
  p.d = g.d.ptr; p.ldd = g.d.ld; p.sd = g.d.stride; p.alpha = g.alpha;
  p.active = g.active; p.diag_shift = g.diag_shift; p.error_flag = eflag;
  p.a_shared = a_batch == 1 && g.batch > 1;
  p.b_shared = b_batch == 1 && g.batch > 1;
  const int stage_bytes = ((a_block_bytes(S) + b_block_bytes(S) + 1023) / 1024) * 1024;
  // as many stages as fit next to the barrier words (S = 7: 2, S <= 6: 3)
  p.nst = std::min<int>(MAX_STAGES, (MAX_SMEM - BAR_BYTES) / stage_bytes);
  const size_t smem = (size_t)p.nst * stage_bytes + BAR_BYTES;
  qtx_opt_in_smem((const void*)ozaki_gemm_kernel, smem);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t ntiles = g.batch * (int64_t)Mt * Nt;
  const unsigned grid = (unsigned)std::min<int64_t>(ntiles, sms);
  ozaki_gemm_kernel<<<grid, THREADS, smem, stream>>>(p);
  qtx_check_launch("ozaki_gemm_kernel");
  cudaFreeAsync(buf, stream);
}
