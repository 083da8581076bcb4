// Kernels of the spectral open-boundary condition: Beyn's contour-integral
// solution of the lead's quadratic eigenvalue problem
//     (a_ji / w + a_ii + a_ij w) v = 0
// and the surface Green's function built from the modes that propagate or
// decay into the lead.
//
// Upstream: qttools.nevp.Beyn (src/qttools/nevp/beyn.py:14-379), the contour
// operator of src/qttools/kernels/operator.py:122-179 and
// qttools.boundary_conditions.obc.Spectral
// (src/qttools/boundary_conditions/obc/spectral.py:15-526).  The O(n^3) work
// -- one n x n inverse per quadrature point and energy, the moment products,
// the mode products and the surface recursion -- runs on the DMMA GEMM and the
// batched inverse; these kernels are the bandwidth-bound glue between them:
//   contour_operator_kernel   T(z) for every (energy, quadrature point)
//   contour_moment_kernel     q0, q1 = weighted sums of the inverses
//   mode_filter_kernel        residual, group velocity and decay of each mode
//   masked_modes_kernel       selected modes, scaled by 1 / w
#include <cmath>

#include "kernels.h"

namespace {

constexpr int TB = 256;
constexpr double TWO_PI = 6.283185307179586476925286766559;

unsigned grid_for(int64_t work) {
  int64_t g = (work + TB - 1) / TB;
  return (unsigned)(g < 65535 * 16 ? g : 65535 * 16);
}

// Quadrature point q of 2 nq: q < nq on the outer circle, else the inner one
// (phases exp(2 pi i (q' + 1.5) / nq), q' = q mod nq; beyn.py:203-209).
__device__ __forceinline__ cplx contour_point(int q, int nq, double r_o, double r_i) {
  const int qq = q < nq ? q : q - nq;
  const double r = q < nq ? r_o : r_i;
  double s, c;
  sincos(TWO_PI * ((qq + 1) + 0.5) / nq, &s, &c);
  return cmk(r * c, r * s);
}

// out[(e * 2nq + q)][r][c] = a_ji / z + a_ii + a_ij z  (operator.py:155-157)
__global__ void contour_operator_kernel(int n, int64_t batch, int nq, double r_o, double r_i, const cplx* a_ii,
                                        int64_t s_ii, const cplx* a_ij, int64_t s_ij, const cplx* a_ji, int64_t s_ji,
                                        cplx* out) {
  const int64_t nn = (int64_t)n * n;
  const int64_t total = batch * 2 * nq * nn;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t rc = t % nn;
    const int64_t eq = t / nn;
    const int q = (int)(eq % (2 * nq));
    const int64_t e = eq / (2 * nq);
    const cplx z = contour_point(q, nq, r_o, r_i);
    const cplx zi = crecip(z);
    cplx v = a_ii[e * s_ii + rc];
    v = cfma(zi, a_ji[e * s_ji + rc], v);
    v = cfma(z, a_ij[e * s_ij + rc], v);
    out[t] = v;
  }
}

// q0[e] = sum_q c0_q inv[e][q], q1[e] = sum_q c1_q inv[e][q] with
// c0 = w z_o, c1 = w z_o^2 on the outer circle and -w z_i, -w z_i^2 on the
// inner one (beyn.py:228-237).
__global__ void contour_moment_kernel(int n, int64_t batch, int nq, double r_o, double r_i, const cplx* inv, cplx* q0,
                                      int64_t s_q0, cplx* q1, int64_t s_q1) {
  const int64_t nn = (int64_t)n * n;
  const double w = 1.0 / nq;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < batch * nn;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = t / nn, rc = t % nn;
    cplx acc0 = cmk(0, 0), acc1 = cmk(0, 0);
    for (int q = 0; q < 2 * nq; ++q) {
      const cplx z = contour_point(q, nq, r_o, r_i);
      const double sgn = q < nq ? w : -w;
      const cplx c0 = cscale(z, sgn);
      const cplx c1 = cmul(c0, z);
      const cplx x = inv[(e * 2 * nq + q) * nn + rc];
      acc0 = cfma(c0, x, acc0);
      acc1 = cfma(c1, x, acc1);
    }
    q0[e * s_q0 + rc] = acc0;
    q1[e * s_q1 + rc] = acc1;
  }
}

// Columns of vs (batch, n, m) scaled to unit 2-norm in place
// (spectral.py:355-358); one warp per (energy, column).
__global__ void normalize_columns_kernel(int n, int m, int64_t batch, cplx* vs) {
  const int64_t warp_id = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp_id >= batch * m) return;
  const int64_t e = warp_id / m;
  const int k = (int)(warp_id % m);
  cplx* v = vs + e * (int64_t)n * m + k;
  double ss = 0;
  for (int r = lane; r < n; r += 32) ss += v[(int64_t)r * m].x * v[(int64_t)r * m].x + v[(int64_t)r * m].y * v[(int64_t)r * m].y;
  for (int off = 16; off > 0; off >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, off);
  const double inv = 1.0 / sqrt(ss);  // a zero column becomes NaN, as upstream's division does
  for (int r = lane; r < n; r += 32) v[(int64_t)r * m] = cscale(v[(int64_t)r * m], inv);
}

// Mode classification of spectral.py:196-322 for one (energy, mode) per warp,
// given R_x = a_x V (x = ji, ii, ij; each (batch, n, m)) and unit columns V.
__global__ void mode_filter_kernel(int n, int m, int64_t batch, const cplx* ws, const cplx* vs, const cplx* r_ji,
                                   const cplx* r_ii, const cplx* r_ij, double min_decay, double max_decay,
                                   double min_propagation, double residual_tolerance, int residual_normalization,
                                   double eta_decay, int* mask) {
  const int64_t warp_id = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp_id >= batch * m) return;
  const int64_t e = warp_id / m;
  const int k = (int)(warp_id % m);
  const cplx w = ws[e * m + k];
  const int64_t base = e * (int64_t)n * m + k;
  // w = 0 (a padded or vanishing eigenvalue): never a reflected mode (its
  // residual and group velocity are not finite)
  if (w.x == 0.0 && w.y == 0.0) {
    if (lane == 0) mask[e * m + k] = 0;
    return;
  }
  const cplx wi = crecip(w);
  double res2 = 0;
  cplx d_ji = cmk(0, 0), d_ij = cmk(0, 0);
  for (int r = lane; r < n; r += 32) {
    const int64_t o = base + (int64_t)r * m;
    const cplx v = vs[o];
    cplx p = r_ii[o];
    p = cfma(wi, r_ji[o], p);
    p = cfma(w, r_ij[o], p);
    res2 += p.x * p.x + p.y * p.y;
    d_ji = cfma(cconj(v), r_ji[o], d_ji);
    d_ij = cfma(cconj(v), r_ij[o], d_ij);
  }
  for (int off = 16; off > 0; off >>= 1) {
    res2 += __shfl_xor_sync(0xffffffffu, res2, off);
    d_ji.x += __shfl_xor_sync(0xffffffffu, d_ji.x, off);
    d_ji.y += __shfl_xor_sync(0xffffffffu, d_ji.y, off);
    d_ij.x += __shfl_xor_sync(0xffffffffu, d_ij.x, off);
    d_ij.y += __shfl_xor_sync(0xffffffffu, d_ij.y, off);
  }
  if (lane != 0) return;
  const double absw = hypot(w.x, w.y);
  double residual = sqrt(res2);  // the columns have unit norm
  if (residual_normalization) residual /= absw;
  // dE/dk = -[(-i) (v^H a_ji v) w^-1 + (i) (v^H a_ij v) w]   (spectral.py:184-192)
  const cplx t_ji = cmul(d_ji, wi), t_ij = cmul(d_ij, w);
  cplx dedk = cmk(-(t_ji.y - t_ij.y), (t_ji.x - t_ij.x));  // i (t_ji - t_ij)
  if (!isfinite(dedk.x)) dedk.x = 0;
  if (!isfinite(dedk.y)) dedk.y = 0;
  // k = -i log w: Im k = -log |w|
  double im_k = -log(absw);
  if (!isfinite(im_k)) im_k = 0;
  const double speed = fabs(dedk.x) / (fabs(dedk.y) + 2.220446049250313e-16);
  const bool propagating = fabs(im_k) < min_decay && min_propagation < speed && dedk.x < 0;
  bool decaying = im_k < -min_decay;
  decaying = decaying || (min_propagation >= speed && im_k < -eta_decay);
  decaying = decaying && im_k > -max_decay;
  mask[e * m + k] = ((propagating || decaying) && residual < residual_tolerance) ? 1 : 0;
}

// vm = V diag(mask), vw = V diag(mask / w), and G += diag(1 - mask) on the
// Gram matrix (batch, m, m) so that its unselected block is the identity.
__global__ void masked_modes_kernel(int n, int m, int64_t batch, const cplx* ws, const cplx* vs, const int* mask,
                                    cplx* vm, cplx* vw) {
  const int64_t total = batch * (int64_t)n * m;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(t % m);
    const int64_t e = t / ((int64_t)n * m);
    const bool on = mask[e * m + k] != 0;
    const cplx v = on ? vs[t] : cmk(0, 0);
    vm[t] = v;
    vw[t] = on ? cmul(v, crecip(ws[e * m + k])) : cmk(0, 0);
  }
}

__global__ void gram_identity_kernel(int m, int64_t batch, const int* mask, cplx* g) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < batch * m; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = t / m;
    const int k = (int)(t % m);
    if (!mask[t]) g[e * (int64_t)m * m + (int64_t)k * m + k].x += 1.0;
  }
}

}  // namespace

void launch_contour_operator(int n, int64_t batch, int nq, double r_o, double r_i, MatView a_ii, MatView a_ij,
                             MatView a_ji, cplx* out, cudaStream_t stream) {
  const int64_t total = batch * 2 * nq * (int64_t)n * n;
  if (total <= 0) return;
  contour_operator_kernel<<<grid_for(total), TB, 0, stream>>>(n, batch, nq, r_o, r_i, a_ii.ptr, a_ii.stride,
                                                               a_ij.ptr, a_ij.stride, a_ji.ptr, a_ji.stride, out);
  qtx_check_launch("contour_operator_kernel");
}

void launch_contour_moments(int n, int64_t batch, int nq, double r_o, double r_i, const cplx* inv, MutView q0,
                            MutView q1, cudaStream_t stream) {
  const int64_t total = batch * (int64_t)n * n;
  if (total <= 0) return;
  contour_moment_kernel<<<grid_for(total), TB, 0, stream>>>(n, batch, nq, r_o, r_i, inv, q0.ptr, q0.stride, q1.ptr,
                                                             q1.stride);
  qtx_check_launch("contour_moment_kernel");
}

void launch_normalize_columns(int n, int m, int64_t batch, cplx* vs, cudaStream_t stream) {
  const int64_t warps = batch * m;
  if (warps <= 0) return;
  normalize_columns_kernel<<<grid_for(warps * 32), TB, 0, stream>>>(n, m, batch, vs);
  qtx_check_launch("normalize_columns_kernel");
}

void launch_mode_filter(int n, int m, int64_t batch, const cplx* ws, const cplx* vs, const cplx* r_ji,
                        const cplx* r_ii, const cplx* r_ij, const SpectralFilter& f, int* mask, cudaStream_t stream) {
  const int64_t warps = batch * m;
  if (warps <= 0) return;
  mode_filter_kernel<<<grid_for(warps * 32), TB, 0, stream>>>(n, m, batch, ws, vs, r_ji, r_ii, r_ij, f.min_decay,
                                                               f.max_decay, f.min_propagation, f.residual_tolerance,
                                                               f.residual_normalization, f.eta_decay, mask);
  qtx_check_launch("mode_filter_kernel");
}

void launch_masked_modes(int n, int m, int64_t batch, const cplx* ws, const cplx* vs, const int* mask, cplx* vm,
                         cplx* vw, cudaStream_t stream) {
  const int64_t total = batch * (int64_t)n * m;
  if (total <= 0) return;
  masked_modes_kernel<<<grid_for(total), TB, 0, stream>>>(n, m, batch, ws, vs, mask, vm, vw);
  qtx_check_launch("masked_modes_kernel");
}

void launch_gram_identity(int m, int64_t batch, const int* mask, cplx* g, cudaStream_t stream) {
  if (batch * m <= 0) return;
  gram_identity_kernel<<<grid_for(batch * m), TB, 0, stream>>>(m, batch, mask, g);
  qtx_check_launch("gram_identity_kernel");
}
