/*
 * qtx_rgf.h -- C ABI of libqtxrgf.so, the B200 (sm_100a) recursive Green's
 * function (RGF) solver for block-tridiagonal systems
 *     A(E) = (E + i eta) S - H - Sigma^R_OBC(E)
 * batched over the energy (stack) axis.
 *
 * Every entry point is a drop-in for one call of the upstream qttools /
 * quatrex Python API (paths relative to the upstream repository):
 *
 *   qtx_selected_inv    <- qttools.greens_function_solver.RGF.selected_inv
 *                          (src/qttools/greens_function_solver/rgf.py:25-113,
 *                           abstract signature solver.py:34-60)
 *   qtx_selected_solve  <- qttools.greens_function_solver.RGF.selected_solve
 *                          (src/qttools/greens_function_solver/rgf.py:115-414,
 *                           abstract signature solver.py:62-113)
 *   qtx_sancho_rubio    <- qttools.boundary_conditions.obc.SanchoRubio.__call__
 *                          (src/qttools/boundary_conditions/obc/sancho_rubio.py:33-86)
 *   qtx_inv             <- qttools.kernels.linalg.inv
 *                          (src/qttools/kernels/linalg/inv.py:24-40)
 *   qtx_obc_assemble    <- the contact part of ElectronSolver._compute_obc
 *                          (src/quatrex/electron/solver.py:318-337, 372-386)
 *   qtx_transport_solve <- ElectronSolver.solve for a device whose leads
 *                          repeat its end cells: A(E) assembly
 *                          (src/quatrex/electron/solver.py:388-410), both
 *                          contacts (:305-386), selected_solve (:533-541) and
 *                          the observables (src/quatrex/core/observables.py:57-189)
 *
 * Conventions
 *  - complex numbers are interleaved (re, im) doubles, layout-identical to
 *    numpy.complex128 / torch.complex128; every matrix is row-major.
 *  - A block-tridiagonal matrix is stored in the DSDBSparse layout of qttools
 *    (src/qttools/datastructures/dsdbsparse.py:109-247): one data row of nnz
 *    entries per stack element; the entries of block (i, j) form one
 *    contiguous slice of that row (src/qttools/datastructures/dsdbcoo.py:285-319).
 *    qtx_btd_desc describes, for each of the 3*nb-2 blocks, where its slice
 *    starts and how its entries map into the dense block.
 *  - All data pointers are DEVICE pointers unless QTX_FLAG_HOST_BUFFERS is set
 *    (qtx_selected_inv / qtx_selected_solve): then the data rows, the OBC
 *    blocks and the current are HOST pointers (the block_index arrays of a
 *    qtx_btd_desc stay device pointers) and the library streams the stack
 *    through the device in energy batches: two device staging sets, a copy
 *    thread moving the caller's (pageable) rows through a ring of page-locked
 *    slots (512 MiB per context, taken from a process-wide pool at the first
 *    such call and kept) while the solver runs; the call returns when every
 *    output is back in host memory.
 *  - Nothing is synchronous unless stated: work is enqueued on `stream`.
 *  - No exception crosses the ABI; every call returns a qtx_status and the
 *    context keeps a text message (qtx_last_error).
 */
#ifndef QTX_RGF_H_
#define QTX_RGF_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int qtx_status;
#define QTX_OK 0
#define QTX_E_INVAL 1          /* invalid argument */
#define QTX_E_NOMEM 2          /* device memory exhausted / over the admission budget */
#define QTX_E_SINGULAR 3       /* exact zero pivot in a diagonal-block inverse */
#define QTX_E_NOT_CONVERGED 4  /* Sancho-Rubio reached max_iterations (results still written) */
#define QTX_E_TIMEOUT 5        /* a bounded device-side wait gave up */
#define QTX_E_CUDA 6           /* CUDA runtime error */
#define QTX_E_UNSUPPORTED 7    /* option not implemented */

/* precision of the bulk block products */
#define QTX_PREC_FP64 0        /* complex128 throughout */
#define QTX_PREC_MIXED 1       /* bulk Schur/Keldysh products of the sweep as 7-bit integer slice
                                  products on the INT8 tensor cores (tcgen05 kind::i8, exact INT32
                                  accumulation, FP64 combine); block inverses and Sancho-Rubio in FP64 */

/* flags of qtx_selected_solve */
#define QTX_FLAG_RETURN_RETARDED 0x1u  /* write diagonal X^R blocks to xr (rgf.py:304-305, 403-404) */
#define QTX_FLAG_RETURN_CURRENT 0x2u   /* Meir-Wingreen layer current (rgf.py:381-400) */
#define QTX_FLAG_SYMMETRIC_OUT 0x4u    /* outputs store the upper triangle only (rgf.py:351, 373) */
#define QTX_FLAG_HOST_BUFFERS 0x8u     /* every data pointer is host memory */
#define QTX_FLAG_RETARDED_OFFDIAG 0x10u /* also write X^R off-diagonal blocks into xr */
#define QTX_FLAG_GRAPH 0x20u           /* qtx_transport_solve: capture the sweep of a single-batch call as a
                                          CUDA graph, cache it per (shapes, buffers, precision) and replay it */

typedef struct qtx_ctx qtx_ctx;
typedef struct CUstream_st* qtx_stream; /* == cudaStream_t; NULL = legacy default stream */

/* Block map of a block-tridiagonal DSDBSparse matrix.  Block (i, j), |i-j|<=1,
 * has index k = 2*i + j (order (0,0),(0,1),(1,0),(1,1),(1,2),(2,1),...). */
typedef struct qtx_btd_desc {
  int32_t num_blocks;                 /* nb */
  const int32_t* block_sizes;         /* host [nb] */
  const int64_t* block_offset;        /* host [3nb-2]: first entry of block k in a data row; -1 = empty block */
  const int64_t* block_nnz;           /* host [3nb-2]: entries of block k */
  const int32_t* const* block_index;  /* host [3nb-2] of DEVICE pointers: local linear index r*cols+c of
                                         each entry of block k; NULL entry = block is dense row-major.
                                         The array itself may be NULL (all blocks dense). */
  int64_t stack_size;                 /* number of stack elements (energies), stack flattened */
  int64_t stack_stride;               /* complex elements between consecutive data rows (>= nnz) */
} qtx_btd_desc;

/* Boundary blocks: per diagonal block i, NULL or a pointer to a contiguous
 * (stack_size, b_i, b_i) complex array (OBCBlocks, solver.py:12-28). */
typedef struct qtx_obc {
  const void* const* retarded;  /* host [nb] of pointers, or NULL */
  const void* const* lesser;    /* host [nb] of pointers, or NULL */
  const void* const* greater;   /* host [nb] of pointers, or NULL */
} qtx_obc;

qtx_status qtx_ctx_create(int device, qtx_ctx** out);
qtx_status qtx_ctx_destroy(qtx_ctx* ctx);
const char* qtx_last_error(const qtx_ctx* ctx);
/* Device bytes the context may keep for workspaces (0 = no limit). */
qtx_status qtx_ctx_set_memory_limit(qtx_ctx* ctx, size_t bytes);
/* Release cached workspaces. */
qtx_status qtx_ctx_trim(qtx_ctx* ctx);
/* Library version string. */
const char* qtx_version(void);

/* Batched inverse of (batch, n, n) complex matrices; x may alias a.
 * <- qttools.kernels.linalg.inv (src/qttools/kernels/linalg/inv.py:24-40). */
qtx_status qtx_inv(qtx_ctx* ctx, int32_t n, int64_t batch, const void* a, int64_t stride_a, void* x,
                   int64_t stride_x, qtx_stream stream);

/* Batched complex GEMM D = alpha op(A) op(B) + beta C, all row-major with
 * per-matrix strides; op = 0 (none) or 1 (conjugate transpose).  Exposed for
 * the tests and the autotuner; the solver uses it internally. */
qtx_status qtx_zgemm(qtx_ctx* ctx, int32_t m, int32_t n, int32_t k, int64_t batch, double alpha_re,
                     double alpha_im, const void* a, int64_t lda, int64_t stride_a, int32_t op_a,
                     const void* b, int64_t ldb, int64_t stride_b, int32_t op_b, double beta_re,
                     double beta_im, const void* c, int64_t ldc, int64_t stride_c, void* d, int64_t ldd,
                     int64_t stride_d, int32_t precision, qtx_stream stream);

/* Batched block combination out = alpha op(x) + beta op(y), op = 0 (none) or
 * 1 (conjugate transpose; op(x) is rows x cols, x itself cols x rows); y may
 * be NULL.  The element-wise glue of the partitioned solver (RGFDist), whose
 * block products run through qtx_zgemm and inverses through qtx_inv.  No
 * reference counterpart as a call: upstream forms these sums with NumPy /
 * CuPy array expressions (src/qttools/greens_function_solver/_serinv.py). */
qtx_status qtx_block_combine(qtx_ctx* ctx, int32_t rows, int32_t cols, int64_t batch, double alpha_re,
                             double alpha_im, const void* x, int64_t ldx, int64_t stride_x, int32_t op_x,
                             double beta_re, double beta_im, const void* y, int64_t ldy, int64_t stride_y,
                             int32_t op_y, void* out, int64_t ldo, int64_t stride_out, qtx_stream stream);

/* Selected inversion: out receives X = A^-1 on the BTD pattern of out_desc.
 * obc_retarded: NULL or host [nb] of device pointers subtracted from A_ii.
 * <- RGF.selected_inv(a, obc_blocks, out) (rgf.py:25-113). */
qtx_status qtx_selected_inv(qtx_ctx* ctx, const qtx_btd_desc* a_desc, const void* a,
                            const void* const* obc_retarded, const qtx_btd_desc* out_desc, void* out,
                            int64_t max_batch_size, int32_t precision, uint32_t flags, qtx_stream stream);

/* Selected solve: X^< = A^-1 Sigma^< A^-H, X^> likewise, and (flags) diagonal
 * X^R and the layer current (stack_size, nb-1) complex.
 * <- RGF.selected_solve(a, sigma_lesser, sigma_greater, obc_blocks, out,
 *    return_retarded, return_current) (rgf.py:115-414).  OBC lesser/greater
 * blocks are ADDED to the diagonal Sigma blocks and the retarded ones
 * subtracted from A, as in rgf.py:207-255. */
qtx_status qtx_selected_solve(qtx_ctx* ctx, const qtx_btd_desc* a_desc, const void* a,
                              const qtx_btd_desc* sl_desc, const void* sigma_lesser,
                              const qtx_btd_desc* sg_desc, const void* sigma_greater, const qtx_obc* obc,
                              const qtx_btd_desc* xl_desc, void* xl, const qtx_btd_desc* xg_desc, void* xg,
                              const qtx_btd_desc* xr_desc, void* xr, void* current, int64_t max_batch_size,
                              int32_t precision, uint32_t flags, qtx_stream stream);

/* Sancho-Rubio surface Green's function x = inv(a_ii - a_ji x a_ij) for a
 * batch of (n, n) blocks; each input has its own batch stride (0 = shared).
 * iterations (device, [batch], may be NULL) receives the iteration count of
 * each batch entry; converged entries stop iterating (per-entry masks).
 * Returns QTX_E_NOT_CONVERGED (after writing x) when an entry reached
 * max_iterations (sancho_rubio.py:81-82 warns in that case), QTX_E_SINGULAR
 * when a decimation block was exactly singular.  batch = 0 is a no-op.
 * <- SanchoRubio(max_iterations, convergence_tol)(a_ii, a_ij, a_ji, contact). */
qtx_status qtx_sancho_rubio(qtx_ctx* ctx, int32_t n, int64_t batch, const void* a_ii, int64_t stride_ii,
                            const void* a_ij, int64_t stride_ij, const void* a_ji, int64_t stride_ji,
                            double convergence_tol, int32_t max_iterations, void* x, int32_t* iterations,
                            qtx_stream stream);

/* Sancho-Rubio that allocates nothing -- no counterpart in the upstream code.
 * For callers that cannot let a library allocate device memory (an
 * application allocator that owns all device memory, a plugin host that
 * forbids library allocations, a latency-critical loop where cudaMalloc /
 * cudaFree would synchronise the device).  Same contract as qtx_sancho_rubio
 * (x, iterations and the QTX_E_NOT_CONVERGED status), without a context: the
 * work space is one fixed 16 MiB device array inside the library, held by
 * every GPU that loads it until the process exits.  A call needs about
 * 9 * 16 * n^2 * batch bytes of it; larger requests return QTX_E_INVAL with the
 * reason in `err` (optional caller buffer of err_len bytes).  An exactly
 * singular decimation block returns QTX_E_SINGULAR.  Every call looks up the
 * array's address on the current device.  All calls share the array: calls
 * that overlap on the GPU race, so serialise them.  The call synchronises
 * `stream` after every iteration (convergence checks through pageable host
 * memory), so it cannot run inside a stream capture. */
qtx_status qtx_sancho_rubio_noalloc(int32_t n, int64_t batch, const void* a_ii, int64_t stride_ii,
                                    const void* a_ij, int64_t stride_ij, const void* a_ji, int64_t stride_ji,
                                    double convergence_tol, int32_t max_iterations, void* x, int32_t* iterations,
                                    qtx_stream stream, char* err, int32_t err_len);

/* One fixed-point step of the surface Green's function and its residuals:
 * x_ref = inv(a_ii - a_ji x a_ij), abs_res = ||x_ref - x||_F,
 * rel_res = abs_res / ||x_ref||_F per batch entry (device arrays, may be NULL).
 * <- OBCSystem._fixed_point_step / _get_residuals
 *    (src/qttools/boundary_conditions/obc/obc.py:105-130, 156-202). */
qtx_status qtx_obc_fixed_point(qtx_ctx* ctx, int32_t n, int64_t batch, const void* a_ii, int64_t stride_ii,
                               const void* a_ij, int64_t stride_ij, const void* a_ji, int64_t stride_ji,
                               const void* x, void* x_ref, double* abs_res, double* rel_res, qtx_stream stream);

/* Spectral open-boundary condition (QuaTrEx's default OBC) in two device
 * steps around a small dense eigenproblem that the caller solves:
 *
 * 1. qtx_beyn_moments: Beyn's contour moments of the lead's quadratic
 *    eigenvalue problem (a_ji / w + a_ii + a_ij w) v = 0, for every energy
 *    p0 = q0 y and p1 = q1 y (batch, n, m0) with
 *    q0 = sum_q (z_o T(z_o)^-1 - z_i T(z_i)^-1) / N, q1 likewise with z^2,
 *    T(z) = a_ji / z + a_ii + a_ij z, z on circles of radius r_o and r_i at
 *    phases exp(2 pi i (q + 1.5) / N), q = 0..N-1 (N = num_quad_points), and
 *    y (batch, n, m0) the caller's probe block.  QTX_E_SINGULAR when a
 *    quadrature point hits an eigenvalue exactly.
 *    <- Beyn._contour_integrate / _one_sided (src/qttools/nevp/beyn.py:187-330)
 *       with the contour operator of src/qttools/kernels/operator.py:122-179.
 * 2. (caller) the SVD projection and the m0 x m0 eigenproblem
 *    (beyn.py:99-144, 241-289) give eigenvalues ws (batch, m0) and
 *    eigenvectors vs (batch, n, m0); padding entries have ws = 0.
 * 3. qtx_spectral_surface: normalises the columns of vs in place, classifies
 *    the modes (propagating with Re dE/dk < 0 or decaying into the lead, with
 *    residual below the tolerance; mask (device int32 (batch, m0), may be
 *    NULL) receives the choice), builds x a_ij = V_r diag(1/w_r) (V_r^H V_r)^-1
 *    V_r^H over the chosen modes, x = inv(a_ii + a_ji x a_ij) and then
 *    num_ref_iterations fixed-point steps x = inv(a_ii - a_ji x a_ij).
 *    <- Spectral._find_reflected_modes, _compute_x_ii and __call__
 *       (src/qttools/boundary_conditions/obc/spectral.py:196-526),
 *       block_sections = 1. */
typedef struct qtx_spectral_params {
  double min_decay, max_decay, min_propagation, residual_tolerance, eta_decay;
  int32_t residual_normalization;
  int32_t num_ref_iterations;
} qtx_spectral_params;

qtx_status qtx_beyn_moments(qtx_ctx* ctx, int32_t n, int64_t batch, const void* a_ii, int64_t stride_ii,
                            const void* a_ij, int64_t stride_ij, const void* a_ji, int64_t stride_ji, double r_o,
                            double r_i, int32_t num_quad_points, const void* y, int32_t m0, void* p0, void* p1,
                            qtx_stream stream);
qtx_status qtx_spectral_surface(qtx_ctx* ctx, int32_t n, int64_t batch, const void* a_ii, int64_t stride_ii,
                                const void* a_ij, int64_t stride_ij, const void* a_ji, int64_t stride_ji,
                                const void* ws, void* vs, int32_t m0, const qtx_spectral_params* params,
                                int32_t* mask, void* x, qtx_stream stream);

/* Contact self-energies from a surface Green's function g (batch, n, n):
 * sigma_r = m_ji g m_ij, gamma = i (sigma_r - sigma_r^H),
 * sigma_l = i f gamma, sigma_g = i (f - 1) gamma with f = occupancy[batch]
 * (src/quatrex/electron/solver.py:318-337). m_ij/m_ji may have stride 0. */
qtx_status qtx_obc_assemble(qtx_ctx* ctx, int32_t n, int64_t batch, const void* g, const void* m_ji,
                            int64_t stride_ji, const void* m_ij, int64_t stride_ij, const double* occupancy,
                            void* sigma_r, void* sigma_l, void* sigma_g, qtx_stream stream);

/* Generator-form transport solve of a device with constant block size b.
 * H is energy independent and resident on the device; A(E) = (E + i eta) I - H
 * is built per energy batch on the device, both contacts come from
 * Sancho-Rubio, and the selected solve writes the requested outputs.  Output
 * pointers may be NULL (not stored).  Block arrays are dense and contiguous:
 * diagonal outputs (num_energies, nb, b, b), off-diagonal (num_energies, nb-1, b, b). */
typedef struct qtx_transport_problem {
  int32_t num_blocks;
  int32_t block_size;
  int64_t num_energies;
  const void* h_diag;       /* (nb, b, b) */
  const void* h_upper;      /* (nb-1, b, b): H[i, i+1]; H[i+1, i] = H[i, i+1]^H */
  const double* energies;   /* (num_energies) device; may be NULL when num_energies = 0 (a no-op call) */
  double eta, mu_left, mu_right, kt;
  double sr_tol;
  int32_t sr_max_iterations;
  int64_t max_batch_size;   /* energies per device batch */
} qtx_transport_problem;

typedef struct qtx_transport_outputs {
  void* gr_diag; void* gr_upper; void* gr_lower;   /* G^R */
  void* gl_diag; void* gl_upper;                   /* G^< (lower = -upper^H) */
  void* gg_diag; void* gg_upper;                   /* G^> */
  double* density;       /* (num_energies, nb): sum over each block of Im diag G^< */
  double* hole_density;  /* (num_energies, nb): sum over each block of -Im diag G^> */
  double* transmission;  /* (num_energies): Tr[Gamma_L G^R_0N Gamma_R G^R_0N^H] */
  void* current_left;    /* (num_energies) complex contact current (observables.py:151-157) */
  void* current_right;   /* (num_energies) complex */
  int32_t* sr_iterations; /* (num_energies, 2) */
  double* dos;           /* (num_energies, nb): mean over each block of -Im diag G^R, the density of
                            states ElectronSolver._filter_peaks builds (src/quatrex/electron/solver.py:428-434) */
  void* layer_current;   /* (num_energies, nb-1) complex: observables.device_current with the Hamiltonian,
                            sum(H_ij * G^<_ji^T - G^<_ij * H_ji^T) per interface (src/quatrex/core/observables.py:192-237) */
} qtx_transport_outputs;

qtx_status qtx_transport_solve(qtx_ctx* ctx, const qtx_transport_problem* p, const qtx_transport_outputs* o,
                               int32_t precision, uint32_t flags, qtx_stream stream);

/* Grouped transport solve (the batching form's persistent launch): every
 * energy of `count` generator-form problems that share one block size
 * b <= 64 (each its own number of blocks, H, energy grid, contacts and
 * outputs, as for qtx_transport_solve) in ONE persistent kernel launch.  Each
 * CTA takes the next (problem, energy) pair and runs its whole solve
 * (Sancho-Rubio of both leads, contact self-energies, forward and backward
 * sweeps, observables); pairs are handed out longest problem first.
 * max_batch_size is ignored.  precision must be QTX_PREC_FP64 (the INT8
 * split products only pay off at b >= 512).  Synchronous (returns when the
 * outputs are written).  statuses (host, count entries, may be NULL) receives
 * each problem's own status: QTX_OK, QTX_E_NOT_CONVERGED (a lead's
 * Sancho-Rubio iteration hit sr_max_iterations; outputs written) or
 * QTX_E_SINGULAR (an exactly singular diagonal block; that problem's outputs
 * hold inf/NaN).  The return value is the worst of them (QTX_E_SINGULAR before
 * QTX_E_NOT_CONVERGED), or QTX_E_UNSUPPORTED for b > 64, QTX_E_INVAL for mixed
 * block sizes or a bad problem. */
qtx_status qtx_transport_solve_grouped(qtx_ctx* ctx, int32_t count, const qtx_transport_problem* problems,
                                       const qtx_transport_outputs* outputs, int32_t precision, uint32_t flags,
                                       qtx_status* statuses, qtx_stream stream);

/* Device bytes one qtx_transport_solve_grouped call allocates (descriptors
 * and one work space per resident CTA); H and the outputs are the caller's.
 * 0 for an unsupported block size. */
size_t qtx_transport_grouped_footprint(int32_t count, const int32_t* num_blocks, const int64_t* num_energies,
                                       int32_t block_size);

/* Block-sorting permutation of a COO pattern on the device (DSDBCOO
 * construction, <- compute_block_sort_index,
 * src/qttools/kernels/datastructure/cupy/dsdbcoo.py:234-298): rows, cols
 * (device int64, nnz entries, global indices) are assigned to the blocks of
 * block_sizes (host [num_blocks]); sort_index (device int64, nnz) receives the
 * stable permutation that orders the entries by block row, then block column
 * (original order kept within a block), block_nnz (host int64 [nb * nb],
 * row-major over (i, j)) the entries of each block.  An index outside the
 * matrix gives QTX_E_INVAL.  num_blocks <= 4096.  Synchronous. */
qtx_status qtx_block_sort_index(qtx_ctx* ctx, int64_t nnz, const int64_t* rows, const int64_t* cols,
                                int32_t num_blocks, const int32_t* block_sizes, int64_t* sort_index,
                                int64_t* block_nnz, qtx_stream stream);

/* System matrix on DSDBSparse data rows, all operands in one entry order:
 * a[e, q] = (E_e + i eta) S_q - V_r [q on the diagonal, r its row] - Sigma[e, q] - H_q
 * (<- ElectronSolver._assemble_system_matrix, src/quatrex/electron/solver.py:388-410,
 * with _btd_subtract :26-51).  rows, cols: device int64 [nnz] (global indices
 * of the entries); overlap: device [nnz] or NULL for S = I; potential: device
 * double [N] or NULL; hamiltonian: device [nnz]; sigma: device
 * (num_energies, stride_sigma) or NULL; a: device (num_energies, stride_a). */
qtx_status qtx_assemble_system(qtx_ctx* ctx, int64_t nnz, int64_t num_energies, const double* energies,
                               double eta, const int64_t* rows, const int64_t* cols, const void* overlap,
                               const double* potential, const void* hamiltonian, const void* sigma,
                               int64_t stride_sigma, void* a, int64_t stride_a, qtx_stream stream);

/* Device bytes one qtx_transport_solve call allocates for itself (recursion
 * state, couplings, Sancho-Rubio and, for QTX_PREC_MIXED, the slice buffers)
 * when it processes `energies_per_call` energies at a time; H and the outputs
 * are the caller's and not included.  Used for admission control. */
size_t qtx_transport_footprint(int32_t num_blocks, int32_t block_size, int64_t energies_per_call,
                               int32_t precision);

/* ---------------------------------------------------------------------------
 * Continuous-batching transport server (the serving form; no reference
 * counterpart: the reference solves one request at a time).
 *
 * `slots` worker threads, each with its own context and CUDA stream, take
 * requests in arrival order.  The oldest waiting request is admitted as soon
 * as a slot is free and its footprint (qtx_transport_footprint) fits in
 * `memory_budget` next to the running requests, so requests that arrive while
 * others run overlap with them on the device.  With group_max_block_size > 0,
 * a worker that admits an FP64 request of block size b <= group_max_block_size
 * (<= 64) also takes every waiting FP64 request of the same b that fits the
 * budget, and solves them together in one qtx_transport_solve_grouped launch;
 * each still completes with its own status.  A request whose footprint
 * exceeds the whole budget is refused at submission (QTX_E_NOMEM).  The
 * problem's device arrays (H, energies) and the outputs belong to the caller
 * and must stay valid until the request has completed.
 * ------------------------------------------------------------------------- */
typedef struct qtx_server qtx_server;

typedef struct qtx_server_config {
  int32_t device;
  int32_t slots;          /* concurrent requests (>= 1) */
  size_t memory_budget;   /* device bytes the running requests may hold; 0 = half of the free memory */
  int32_t group_max_block_size;  /* 0: every request alone; else group requests of b <= this (max 64) */
} qtx_server_config;

typedef struct qtx_server_stats {
  int64_t submitted, completed, failed, queued, running, peak_running;
  int64_t solves;             /* energies of the completed requests */
  size_t memory_in_use;       /* footprint of the running requests */
  double p50_latency_s, p99_latency_s, mean_latency_s;  /* completion - submission */
  int64_t grouped_launches;   /* qtx_transport_solve_grouped launches */
  int64_t grouped_requests;   /* requests solved in them */
} qtx_server_stats;

qtx_status qtx_server_create(const qtx_server_config* cfg, qtx_server** out);
/* Finishes every request already submitted, then stops the workers. */
qtx_status qtx_server_destroy(qtx_server* srv);
/* Enqueue one request (precision and flags as for qtx_transport_solve, except
 * that QTX_FLAG_GRAPH is ignored: every request has its own buffers; the
 * problem's max_batch_size sets the energies per device call). */
qtx_status qtx_server_submit(qtx_server* srv, const qtx_transport_problem* p, const qtx_transport_outputs* o,
                             int32_t precision, uint32_t flags, int64_t* request_id);
/* Wait up to timeout_ms (< 0: no limit) for request `request_id`.  Returns
 * QTX_E_TIMEOUT if it has not completed, QTX_E_INVAL for an unknown or already
 * collected id, else QTX_OK with the request's own status, latency and error
 * text (err may be NULL); the request is collected. */
qtx_status qtx_server_wait(qtx_server* srv, int64_t request_id, int64_t timeout_ms, qtx_status* request_status,
                           double* latency_s, char* err, int32_t err_len);
/* As qtx_server_wait, for whichever uncollected request completes first. */
qtx_status qtx_server_wait_any(qtx_server* srv, int64_t timeout_ms, int64_t* request_id, qtx_status* request_status,
                               double* latency_s, char* err, int32_t err_len);
qtx_status qtx_server_get_stats(qtx_server* srv, qtx_server_stats* stats);

/* Number of captured-sweep replays issued by this context (QTX_FLAG_GRAPH). */
int64_t qtx_graph_replays(const qtx_ctx* ctx);
/* Drop every captured sweep the context holds; their work spaces are freed in
 * stream order on `stream` after their last use, without a device-wide
 * synchronisation (safe while other threads capture or run).  No reference
 * counterpart: the reference captures no graphs. */
qtx_status qtx_ctx_release_graphs(qtx_ctx* ctx, qtx_stream stream);

/* Number of kernel launches this context has issued (for launch accounting). */
int64_t qtx_launch_count(const qtx_ctx* ctx);

/* Launch timing (the counterpart of qttools.profiling.Profiler,
 * src/qttools/profiling/profiler.py:187-429, which times code regions): when
 * enabled, every complex-GEMM (kind 0) and block-inverse (kind 1) launch of
 * this context is bracketed by CUDA events on its stream.  Enabling or
 * disabling resets the totals.  The report synchronises on the recorded events
 * and returns the summed device time, the algorithmic flops (8 m n k per
 * complex product, 8 n^3 per inverse) and the number of launches. */
qtx_status qtx_ctx_set_timing(qtx_ctx* ctx, int enable);
qtx_status qtx_ctx_timing_report(qtx_ctx* ctx, int32_t kind, double* total_ms, double* total_flops,
                                 int64_t* launches);

#ifdef __cplusplus
}
#endif
#endif /* QTX_RGF_H_ */
