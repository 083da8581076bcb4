// Host-side launchers of the device kernels of libqtxrgf (all enqueue on `stream`).
#pragma once

#include "common.cuh"

// A strided batch of row-major complex matrices: element (e, r, c) at
// ptr[e * stride + r * ld + c].  stride 0 broadcasts one matrix over the batch.
struct MatView {
  const cplx* ptr = nullptr;
  int64_t ld = 0;
  int64_t stride = 0;
};
struct MutView {
  cplx* ptr = nullptr;
  int64_t ld = 0;
  int64_t stride = 0;
  operator MatView() const { return MatView{ptr, ld, stride}; }
};

enum Op : int { OP_N = 0, OP_C = 1 };

// D = alpha op(A) op(B) + beta C + gamma C2   (C, C2 optional: ptr == nullptr)
// op(A) is m x k, op(B) is k x n.  `active` (device, [batch], optional) skips
// batch entries whose flag is 0.  D may alias C or C2 but not A or B.
struct GemmCall {
  int m = 0, n = 0, k = 0;
  int64_t batch = 0;
  MatView a; int op_a = OP_N;
  MatView b; int op_b = OP_N;
  MatView c; cplx beta = {0, 0};
  MatView c2; cplx gamma = {0, 0};
  MutView d; cplx alpha = {1, 0};
  const int* active = nullptr;
  // optional per-batch-entry diagonal shift: D[r][r] += diag_shift[e] (e.g. (E + i eta) I)
  const cplx* diag_shift = nullptr;
};
void launch_zgemm(const GemmCall& g, cudaStream_t stream);

// Mixed-precision variant of the same contract: FP64 operands split into
// 7-bit integer slices whose products run on tcgen05 kind::i8 with exact
// INT32 accumulation (Ozaki scheme); see zgemm_ozaki.cu.
void launch_zgemm_mixed(const GemmCall& g, cudaStream_t stream);
bool mixed_supported(const GemmCall& g);
// Device bytes of the slice buffers of one mixed GEMM (m x n x k, batch entries
// per operand; an operand with batch stride 0 counts once).
size_t mixed_workspace_bytes(int m, int n, int k, int64_t a_batch, int64_t b_batch);
// Throws QTX_E_TIMEOUT (and clears the flag) if a mixed GEMM since the last
// check gave up a pipeline wait.  Synchronises the stream.
void mixed_check_error(cudaStream_t stream);

// Batched in-place-capable Gauss-Jordan inverse with partial pivoting:
// X = A^-1 for n x n matrices.  info[e] (device, optional) receives the
// 1-based column of the first exactly-zero pivot and is left untouched when
// there is none (callers zero it once and may read it after several
// launches).  X may alias A.  Batches smaller than the GPU take a split path
// whose per-panel scratch comes from the stream-ordered pool; with
// may_allocate = false the one-CTA-per-matrix kernel runs at every size.
void launch_zinv(int n, int64_t batch, MatView a, MutView x, int* info, const int* active,
                 cudaStream_t stream, bool may_allocate = true);
// Scratch the split path of launch_zinv takes for one call (0 when the batch
// takes the one-CTA-per-matrix kernel).
size_t zinv_workspace_bytes(int n, int64_t batch);

// out = s + gamma_s * s2 + w^H - w  (n x n), in place allowed for out == s.
void launch_skew_combine(int n, int64_t batch, MatView s, MatView w, MutView out, cudaStream_t stream);
// x = x - x^H in place (n x n).
void launch_sub_herm_inplace(int n, int64_t batch, MutView x, cudaStream_t stream);
// out = alpha * x + beta * y (rows x cols); y optional; entries with active[e] == 0 untouched.
void launch_axpby(int rows, int cols, int64_t batch, cplx alpha, MatView x, cplx beta, MatView y, MutView out,
                  cudaStream_t stream, const int* active = nullptr);
// shift[e] = (energies[e] + i eta)
void launch_energy_shift(int64_t batch, const double* energies, double eta, cplx* shift, cudaStream_t stream);

// Scatter / gather between dense (batch, rows, cols) blocks and a DSDBSparse
// data slice (entry q of the block at data[e * stride + q], local index
// index[q] = r * cols + c, or row-major dense when index == nullptr).
// mode: 0 = copy, 1 = 0.5 (X - X^H) (square), 2 = -X^H (out is cols x rows of x^H)
void launch_block_scatter(int rows, int cols, int64_t batch, MatView x, int mode, cplx* data, int64_t stride,
                          int64_t nnz, const int32_t* index, cudaStream_t stream);
void launch_block_gather(int rows, int cols, int64_t batch, const cplx* data, int64_t stride, int64_t nnz,
                         const int32_t* index, MutView out, cudaStream_t stream);

// tr[e] (+)= sum_rc x[r][c] * y[c][r] * scale  (trace of x y); x rows x cols, y cols x rows.
// accumulate: add into tr instead of overwriting.
void launch_trace_product(int rows, int cols, int64_t batch, MatView x, MatView y, cplx scale, cplx* tr,
                          bool accumulate, cudaStream_t stream);
// tr[e] = sum_rc x[r][c] * conj(y[r][c])   (Tr[x y^H])
void launch_trace_product_h(int rows, int cols, int64_t batch, MatView x, MatView y, cplx* tr,
                            cudaStream_t stream);
// Sancho-Rubio convergence: delta[e] = || |alpha| + |beta| ||_F / 2 ; then
// active[e] = active[e] && delta >= tol; iterations[e] += active-before.
void launch_sr_norm_update(int n, int64_t batch, MatView alpha, MatView beta, double tol, int* active,
                           int* iterations, int* num_active, cudaStream_t stream);
// A_ii(E) = (E + i eta) I - H  for energies[batch]; out (batch, n, n).
void launch_assemble_diag(int n, int64_t batch, const cplx* h, const double* energies, double eta, MutView out,
                          cudaStream_t stream);
// out = -H^H for a single matrix (n x n).
void launch_neg_herm(int n, const cplx* h, cplx* out, cudaStream_t stream);
// gamma = i (s - s^H); sl = i f gamma; sg = i (f - 1) gamma with f = occ[e]
void launch_obc_lesser_greater(int n, int64_t batch, MatView sigma_r, const double* occ, MutView sl, MutView sg,
                               MutView gamma, cudaStream_t stream);
// occ[e] = 1 / (1 + exp((E_e - mu) / kT))
void launch_fermi(int64_t batch, const double* energies, double mu, double kt, double* occ, cudaStream_t stream);
void launch_fill_int(int* p, int64_t count, int value, cudaStream_t stream);
// dst[t * dst_stride] = src[t * src_stride], t < count.  The solver's small
// fills and copies run as kernels, not cudaMemset / cudaMemcpy: those go to a
// copy engine and wait there behind any large download a caller has in
// flight on another stream.
void launch_copy_int(int* dst, int64_t dst_stride, const int* src, int64_t src_stride, int64_t count,
                     cudaStream_t stream);
// abs_res[e] = ||x_ref - x||_F, rel_res[e] = abs_res[e] / ||x_ref||_F (contiguous n x n matrices)
void launch_residual_norm(int n, int64_t batch, MatView x_ref, MatView x, double* abs_res, double* rel_res,
                          cudaStream_t stream);
void launch_real_part(int64_t count, const cplx* src, double* dst, cudaStream_t stream);
// mapped_out (device alias of mapped page-locked host memory, 3 ints):
// [0] = 1 + index of the first nonzero src entry or 0, [1] = that entry,
// [2] = src[0].  The host reads it after synchronising the stream.
void launch_flag_reduce(const int* src, int64_t n, int* mapped_out, cudaStream_t stream);
// out = alpha op(x) + beta op(y) (rows x cols each; y optional: ptr == nullptr),
// op = OP_N or OP_C.  out must not overlap x or y when an operand is transposed.
void launch_block_combine(int rows, int cols, int64_t batch, cplx alpha, MatView x, int op_x, cplx beta, MatView y,
                          int op_y, MutView out, cudaStream_t stream);
// flags[k] = 1 if block slice k of a DSDBSparse data stack holds any nonzero
// entry in any of `rows` data rows (flags zeroed by the caller).  slices
// (device int64 [2 * num_slices]): (offset, nnz) of each slice in a row;
// num_slices <= 65535.
void launch_block_nonzero(int num_slices, const int64_t* slices, const cplx* data, int64_t stride, int64_t rows,
                          int* flags, cudaStream_t stream);
// Lesser / greater blocks from the two contact-source responses XL, XR
// (n x n, per batch entry e):  Y< = f_L XL + s f_R XR,  Y> = (f_L - 1) XL + s (f_R - 1) XR
// with f = occ_l[e], occ_r[e] and s = sign_r; sym: write 0.5 (Y - Y^H), else Y.
// out_l / out_g (row-major n x n at out + e * stride) may be null.
void launch_keldysh_combine(int n, int64_t batch, MatView xl, MatView xr, const double* occ_l, const double* occ_r,
                            double sign_r, bool sym, cplx* out_l, int64_t stride_l, cplx* out_g, int64_t stride_g,
                            cudaStream_t stream);
// out[e * out_stride + out_col] = -(1/n) sum_r Im g[r][r]   (per-block density of states of G^R)
void launch_block_dos(int n, int64_t batch, MatView g, double* out, int64_t out_stride, int out_col,
                      cudaStream_t stream);
// out[e * out_stride + out_col] = sum_rc H[r][c] (-conj Y[r][c]) - Y[r][c] conj H[r][c] with Y the lesser
// combination of (xl, xr) as in launch_keldysh_combine: the layer current across the interface whose
// coupling block is H (one matrix for the whole batch) and whose G^< upper block is Y.
void launch_layer_current(int n, int64_t batch, MatView xl, MatView xr, const double* occ_l, const double* occ_r,
                          double sign_r, const cplx* coupling, cplx* out, int64_t out_stride, int out_col,
                          cudaStream_t stream);
// density[e * out_stride + out_col] = sum_r Im Y<_rr, hole[...] = -sum_r Im Y>_rr (either may be null)
void launch_keldysh_density(int n, int64_t batch, MatView xl, MatView xr, const double* occ_l, const double* occ_r,
                            double* density, double* hole, int64_t out_stride, int out_col, cudaStream_t stream);

// One generator-form problem of a grouped transport solve, as the persistent
// kernel reads it (rgf_grouped.cu).  Pairs item0 .. item0 + num_energies - 1 of
// the launch's work list are this problem's energies.
struct GroupedProblem {
  int nb = 0, b = 0;
  int64_t num_energies = 0, item0 = 0;
  const cplx* h_diag = nullptr;   // (nb, b, b)
  const cplx* h_upper = nullptr;  // (nb - 1, b, b)
  const double* energies = nullptr;
  double eta = 0, mu_left = 0, mu_right = 0, kt = 0, sr_tol = 0;
  int sr_max_iterations = 0;
  cplx *gr_diag = nullptr, *gr_upper = nullptr, *gr_lower = nullptr;
  cplx *gl_diag = nullptr, *gl_upper = nullptr, *gg_diag = nullptr, *gg_upper = nullptr;
  double *density = nullptr, *hole_density = nullptr, *transmission = nullptr;
  cplx *current_left = nullptr, *current_right = nullptr;
  int* sr_iterations = nullptr;
  double* dos = nullptr;
  cplx* layer_current = nullptr;
};
// Largest block size of the grouped solve.
constexpr int GROUPED_MAX_B = 64;
// CTAs of the persistent launch for `items` pairs of block size b (never more
// than fit on the device at once), and the work-space elements of one CTA.
int grouped_grid(int b, int64_t items);
int64_t grouped_ws_elems(int max_nb, int b);
// flags (device ints [1 + count], zeroed by the caller): bit 0 a zero pivot in
// a sweep inverse, bit 1 a Sancho-Rubio iteration that did not converge;
// flags[0] for the whole launch, flags[1 + q] for problem q.
void launch_transport_grouped(int b, const GroupedProblem* problems, int count, int64_t items,
                              unsigned long long* counter, int* flags, cplx* ws, int64_t ws_elems, int max_nb, int grid,
                              cudaStream_t stream);

// ---- spectral open-boundary condition (spectral.cu) -----------------------
// Mode-classification thresholds of qttools' Spectral OBC
// (src/qttools/boundary_conditions/obc/spectral.py:63-94).
struct SpectralFilter {
  double min_decay = 1e-3, max_decay = 6.9, min_propagation = 0.01, residual_tolerance = 1e-3, eta_decay = 1e-14;
  int residual_normalization = 1;
};
// out (batch * 2 nq, n, n) contiguous: a_ji / z + a_ii + a_ij z at the nq
// points of the outer circle, then the nq of the inner one.
void launch_contour_operator(int n, int64_t batch, int nq, double r_o, double r_i, MatView a_ii, MatView a_ij,
                             MatView a_ji, cplx* out, cudaStream_t stream);
// q0, q1 (batch, n, n) from the inverses (batch * 2 nq, n, n) of the operator.
void launch_contour_moments(int n, int64_t batch, int nq, double r_o, double r_i, const cplx* inv, MutView q0,
                            MutView q1, cudaStream_t stream);
// Unit 2-norm columns of vs (batch, n, m), in place.
void launch_normalize_columns(int n, int m, int64_t batch, cplx* vs, cudaStream_t stream);
// mask (batch, m) of the reflected modes, from ws (batch, m), unit-column vs
// (batch, n, m) and r_x = a_x vs (x = ji, ii, ij).
void launch_mode_filter(int n, int m, int64_t batch, const cplx* ws, const cplx* vs, const cplx* r_ji,
                        const cplx* r_ii, const cplx* r_ij, const SpectralFilter& f, int* mask, cudaStream_t stream);
// vm = vs diag(mask), vw = vs diag(mask / w)   (batch, n, m)
void launch_masked_modes(int n, int m, int64_t batch, const cplx* ws, const cplx* vs, const int* mask, cplx* vm,
                         cplx* vw, cudaStream_t stream);
// g[e] += diag(1 - mask[e])   (batch, m, m)
void launch_gram_identity(int m, int64_t batch, const int* mask, cplx* g, cudaStream_t stream);
