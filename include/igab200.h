/*
 * igab200.h -- C ABI of the B200 (sm_100a) matrix-free weighted-quadrature
 * library `libigab200.so`.
 *
 * Every entry point takes plain device pointers, sizes and a CUDA stream
 * (passed as `void*`), returns an `iga_status`, never aborts and never
 * allocates device memory: callers own every buffer (inputs, outputs and the
 * scratch work arrays some calls ask for).  Calls are stream-ordered.
 *
 * The reference (igaops) is pure Python, so it has no FFI of its own; each
 * entry point below names the reference function whose arithmetic it
 * replaces.  Paths are relative to the igaops repository root.
 */
#ifndef IGAB200_H
#define IGAB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int iga_status;
#define IGA_OK 0
#define IGA_ERR_INVALID_ARG 1  /* bad size, pointer, alignment or choice   */
#define IGA_ERR_UNSUPPORTED 2  /* valid, but no kernel for this case       */
#define IGA_ERR_CUDA 3         /* a CUDA runtime call failed              */
#define IGA_ERR_NOT_CONVERGED 4
#define IGA_ERR_BREAKDOWN 5
#define IGA_ERR_NONFINITE 6
#define IGA_ERR_GEOMETRY 7     /* det J <= 0 at some quadrature point      */
#define IGA_ERR_TIMEOUT 8      /* a bounded device-side wait gave up       */

/* element types */
#define IGA_F64 0
#define IGA_F32 1
#define IGA_BF16 2

/* operator kinds of the fused matrix-free matvec */
#define IGA_OP_MASS 0     /* compute_mf_scalar_u_v          */
#define IGA_OP_STIFF 1    /* compute_mf_scalar_gradu_gradv  */
#define IGA_OP_GRADU_V 2  /* compute_mf_scalar_gradu_v      */
#define IGA_OP_U_GRADV 3  /* compute_mf_scalar_u_gradv      */

typedef void* iga_stream; /* a cudaStream_t; NULL = legacy default stream */

/* A banded matrix of `rows` x `cols`: row r holds the entries of columns
 * start[r] .. start[r]+width-1 in vals[r*width .. r*width+width-1]
 * (zero-padded).  start[] must be non-decreasing.  This is the device form of
 * the CSR 1D factors `q.basis[k]` / `q.weights[k]` (and their transposes). */
typedef struct {
  int32_t rows, cols, width, reserved;
  const int32_t* start; /* device, [rows] */
  const void* vals;     /* device, [rows*width], element type of the call */
} iga_band;

/* One 1D factor of a Kronecker product: a band or a strided dense matrix
 * (element (r,c) at dense[r*ld_row + c*ld_col]; swap the strides for M^T). */
typedef struct {
  int32_t kind; /* 0 = band, 1 = dense */
  int32_t rows, cols, reserved;
  int64_t ld_row, ld_col;
  iga_band band;
  const void* dense;
} iga_factor;

/* --------------------------------------------------------------------- */
/* library                                                                */
/* --------------------------------------------------------------------- */

/* ABI revision of this header. */
int iga_abi_version(void);

/* Message of the last failed call on this host thread ("" if none). */
const char* iga_last_error(void);

/* --------------------------------------------------------------------- */
/* L-mode (n-mode) products                                              */
/* --------------------------------------------------------------------- */

/* One n-mode product on a tensor viewed as (outer, cols, inner):
 *   y[o, r, i] = sum_c M[r, c] x[o, c, i]   (accumulate: y += ...).
 * Replaces MatrixFree.tensor_matrix_product
 * (src/igaops/operators/utils/matrix_free.py:39-75). */
iga_status iga_mode_product(int dtype, const iga_factor* M, int64_t outer,
                            int64_t inner, const void* x, void* y,
                            int accumulate, iga_stream stream);

/* y = (M_d (x) ... (x) M_1) x for `ncols` right-hand sides stored with the
 * column index fastest (the layout of a C-order (N, ncols) array).
 * factors[0] is M_1 (fastest direction).  work0/work1 must each hold the
 * largest intermediate tensor (max over k of prod(rows_{<=k}) *
 * prod(cols_{>k}) * ncols elements).  Replaces MatrixFree.apply
 * (src/igaops/operators/utils/matrix_free.py:77-119). */
iga_status iga_lmode_apply(int dtype, int ndim, const iga_factor* factors,
                           int64_t ncols, const void* x, void* y, void* work0,
                           void* work1, iga_stream stream);

/* out[q*ncols + k] (+)= coef[q*coef_stride] * u[q*ncols + k]; the pointwise
 * "broadcast" einsum of src/igaops/operators/bsplines_ops.py:311,341-343. */
iga_status iga_pointwise_scale(int dtype, int64_t nq, int64_t ncols,
                               const void* coef, int64_t coef_stride,
                               const void* u, void* out, int accumulate,
                               iga_stream stream);

/* y = alpha*x + beta*y over n elements (beta == 0: y = alpha*x).  The
 * accumulation `array_out += ...` of src/igaops/operators/bsplines_ops.py:350
 * and the vector updates of the Krylov solvers. */
iga_status iga_axpby(int dtype, int64_t n, double alpha, const void* x,
                     double beta, void* y, iga_stream stream);

/* --------------------------------------------------------------------- */
/* Fused matrix-free weighted-quadrature matvec                           */
/* --------------------------------------------------------------------- */

/* Plan of one fused operator on one patch (2D or 3D tensor mesh).
 * Per direction d the plan holds three banded views of the 1D factors, all
 * built from the quadrature rule q_d of the patch:
 *   trial[d]  : B0_d (nq x n) band; trial_d1[d] = B1_d values, same band;
 *   testT[d]  : W0_d^T (nq x n) band; testT_d1[d] = W1_d^T values, same band;
 *   testR[d]  : W0_d (n x nq) band;  testR_d1[d] = W1_d values, same band;
 * where W0 = q.weights[0] (= weights[1]) and W1 = q.weights[2] (= [3]).
 * The band starts of trial[d] and testT[d] must advance by at most one row
 * per quadrature point (smooth the jump at the last point, as the Python
 * layer does); the 3D kernel moves its plane windows once per point.
 * Packed coefficients follow `tile_off` (see iga_mf_pack). */
typedef struct {
  int32_t ndim;       /* 2 or 3                                          */
  int32_t op;         /* IGA_OP_*                                        */
  int32_t spacetime;  /* 1: last direction is time (time_ders given)    */
  int32_t time_test;  /* time derivative order of the test side (0/1)   */
  int32_t time_trial; /* time derivative order of the trial side (0/1)  */
  int32_t sym;        /* IGA_OP_STIFF: coefficients packed symmetric    */
  int32_t width;      /* common band width of trial / testT (<= 8)      */
  int32_t rwidth;     /* band width of testR                            */
  int32_t n[3], nq[3];
  int32_t face[2];    /* quadrature tile face (FX, FY; FY = 1 in 2D)    */
  int32_t nseg;       /* segments of the streamed (last) direction      */
  int32_t nstream;    /* packed coefficient streams                     */
  int32_t src_row[9]; /* leading index of the reference coefficient array
                         read by each stream (see iga_mf_pack)           */
  int32_t cmax[2];    /* max trial ctrl range of a tile in dirs 1, 2    */
  int32_t dmax[2];    /* max test ctrl range of a tile in dirs 1, 2     */
  const int64_t* tile_off; /* device: element offset of each tile      */
  iga_band trial[3];
  const void* trial_d1[3];
  iga_band testT[3];
  const void* testT_d1[3];
  iga_band testR[3];
  const void* testR_d1[3];
  int32_t* status;    /* device int32 error word (IGA_ERR_TIMEOUT)      */
  const void* step_table; /* device: per-point rows of the streamed direction
                             (iga_mf_table), element type of the matvec    */
  int32_t wait_test;      /* 0 in normal use.  Test hook of the 3D kernel's
                             bounded waits: nonzero withholds the first
                             coefficient copy of every CTA, so that its first
                             wait runs out (after about 1 ms) and the launch
                             reports IGA_ERR_TIMEOUT in *status after draining
                             the copies that were issued                     */
} iga_mf_plan;

/* Layout of the packed coefficient buffer of `plan` for element type
 * `dtype`: total elements, and (if tile_off_host is not NULL) the element
 * offset of each quadrature tile, tiles1*tiles2 entries (tiles1 in 2D), to be
 * copied to the device array plan->tile_off. */
iga_status iga_mf_layout(const iga_mf_plan* plan, int dtype, int64_t* elems,
                         int64_t* tile_off_host);

/* Step table of the streamed (last) direction: one row per quadrature
 * point holding its trial band values (B0, B1), test band values (W0^T,
 * W1^T) and the two band starts, padded to 16 bytes.  With table == NULL
 * only *elems is returned; otherwise the rows are written to `table`
 * (caller-owned, *elems elements of `dtype`).  plan->step_table must point
 * to it before iga_mf_matvec. */
iga_status iga_mf_table(const iga_mf_plan* plan, int dtype, int64_t* elems,
                        void* table, iga_stream stream);

/* Packs reference-layout coefficients into the streamed tile layout.
 * `coefs` is the array the reference takes: (Nq,) for mass, (d, d, Nq) for
 * stiffness, (d, Nq) for the advection terms, with element (s, q) at
 * coefs[s*ld + q] (s = flattened leading index); dtype_in is IGA_F64 or
 * IGA_F32, dtype_out the element type of the matvec. */
iga_status iga_mf_pack(const iga_mf_plan* plan, int dtype_in, const void* coefs,
                       int64_t ld, int dtype_out, void* packed,
                       iga_stream stream);

/* y = A x for the operator of `plan`, ncols right-hand sides stored column
 * after column (x[k*N + i]).  Replaces BsplineOperations.compute_mf_scalar_*
 * (src/igaops/operators/bsplines_ops.py:290-429). */
iga_status iga_mf_matvec(const iga_mf_plan* plan, int dtype, const void* packed,
                         int64_t ncols, const void* x, void* y,
                         iga_stream stream);

/* Tensor-core (FP64) 3D matvec: plan of one operator on one patch, built by
 * igaops_b200/tile3d.py.  Tiles of 16 x 8 x 16 quadrature points; per
 * direction and tile a geometry record (16 int32: first point, points,
 * first trial / test control point, trial / test extents, trial / test
 * window offsets of the two 8-point groups, groups, prefix and weight of the
 * packed-unit count) and a fragment table (512 doubles: [group][B0, B1,
 * W0^T, W1^T][k-step][lane], the 8 x 8 window blocks in tensor-core operand
 * order).  Covers the stiffness operator with symmetric coefficients and the
 * mass operator, FP64, band widths <= 5, no space-time derivatives. */
typedef struct {
  int32_t op;          /* IGA_OP_MASS or IGA_OP_STIFF */
  int32_t nstream;     /* 1 (mass) or 6 (C00, C01, C02, C11, C12, C22) */
  int32_t n[3];        /* control points per direction */
  int32_t nq[3];       /* quadrature points per direction */
  int32_t ntile[3];    /* tiles per direction */
  int32_t wsum[3];     /* sums of the per-tile unit weights per direction */
  int32_t src_row[6];  /* leading index of each stream in the coefficient array */
  const int32_t* geom; /* device: (ntile[0] + ntile[1] + ntile[2]) x 16 */
  const double* frag;  /* device: (ntile[0] + ntile[1] + ntile[2]) x 512 */
  int32_t* status;     /* device: first error of a launch (IGA_ERR_TIMEOUT) */
} iga_mft_plan;

/* Packs reference-layout coefficients ((Nq,) mass, (3, 3, Nq) stiffness with
 * element (s, q) at coefs[s*ld + q]) into the plan's coefficient units:
 * wsum[0]*wsum[1]*wsum[2] units of 2*nstream*32 doubles, each the 8 (q1, q2)
 * rows x 8 q3 points of one tile block in the order the kernel reads them,
 * zero where the tile has no point. */
iga_status iga_mft_pack(const iga_mft_plan* plan, int dtype_in, const void* coefs,
                        int64_t ld, double* packed, int64_t packed_elems,
                        iga_stream stream);

/* Dynamic shared memory of the plan's kernel (bytes). */
iga_status iga_mft_smem_bytes(const iga_mft_plan* plan, int64_t* bytes);

/* y = A x (FP64) with the plan's packed coefficients; ncols right-hand sides
 * stored column after column.  Replaces
 * BsplineOperations.compute_mf_scalar_gradu_gradv / compute_mf_scalar_u_v
 * (src/igaops/operators/bsplines_ops.py:290-355) for the operators the plan
 * covers. */
iga_status iga_mft_matvec(const iga_mft_plan* plan, const double* packed, int64_t ncols,
                          const double* x, double* y, iga_stream stream);

/* --------------------------------------------------------------------- */
/* Solve level                                                            */
/* --------------------------------------------------------------------- */

/* A user operator for the solve entry points: y = op(x), x and y device
 * vectors of n FP64 entries, work issued on `stream`; returns IGA_OK or an
 * error status, which ends the solve with that status. */
typedef iga_status (*iga_apply_fn)(void* user, const double* x, double* y, iga_stream stream);

/* Device workspace (elements of FP64) of iga_gmres_solve for n unknowns and
 * maxiters iterations: (2 maxiters + 3) n plus a few reduction partials. */
iga_status iga_gmres_workspace(int64_t n, int maxiters, int64_t* elems);

/* x = A^{-1} b by unrestarted flexible GMRES, right preconditioned by P
 * (NULL: none), the Krylov vectors in `work` (device, caller-owned,
 * iga_gmres_workspace elements).  Replaces LinearSolver.solve(Afun, b, Pfun)
 * with linear_type="gmres" (src/igaops/solvers/linear_solver.py:149-257,
 * 438-525): two Gram-Schmidt passes per step, the Dirichlet DOFs `dirichlet`
 * (device, ndirichlet int64 indices; the reference's cleandod) zeroed in b
 * and in every input and output of A and P, stop at relative residual <
 * tolerance or absolute residual < 1e-14 (the reference's increment
 * criterion is not applied).  b and x are device vectors; x starts at zero.
 * residual_history (host, maxiters + 1 doubles, or NULL) receives the
 * relative residuals from iteration 0, *iterations the steps taken.
 * Returns IGA_OK (converged), IGA_ERR_NOT_CONVERGED (x is the last
 * iterate -- the reference's success=False), IGA_ERR_BREAKDOWN,
 * IGA_ERR_NONFINITE (a NaN / Inf in b or in an operator output) or the
 * status of a failing callback. */
iga_status iga_gmres_solve(int64_t n, const double* b, double* x, double tolerance,
                           int maxiters, iga_apply_fn A, iga_apply_fn P, void* user,
                           const int64_t* dirichlet, int64_t ndirichlet, double* work,
                           int64_t work_elems, double* residual_history, int* iterations,
                           iga_stream stream);

/* --------------------------------------------------------------------- */
/* Fast-diagonalisation preconditioner                                    */
/* --------------------------------------------------------------------- */

/* y = P^{-1} x with P^{-1} = (U_d (x)..(x) U_1) diag(inv_lambda)
 * (U_d (x)..(x) U_1)^T on the free box {lo_k <= i_k < lo_k + m_k} of the
 * control-point tensor (direction 1 fastest, n[k] points per direction) and
 * zero outside it.  U[k] is the dense m_k x m_k eigenvector matrix of
 * direction k (row-major), inv_lambda has prod(m) entries (direction 1
 * fastest); x, y hold ncols columns with the column index fastest.  work0 and
 * work1 hold prod(m)*ncols elements each.  dtype IGA_F64 or IGA_F32.
 * Replaces SpaceFD.apply (src/igaops/fastdiag/utils/space_precond.py:273-320). */
iga_status iga_fd_apply(int dtype, int ndim, const int32_t* n, const int32_t* lo,
                        const int32_t* m, const void* const* U,
                        const void* inv_lambda, int64_t ncols, const void* x,
                        void* y, void* work0, void* work1, iga_stream stream);

/* Copy between a full tensor x (extents n, direction 1 fastest, ncols
 * columns fastest) and the dense box [lo, lo+m) of it: scatter = 0 gathers
 * the box into dst, scatter = 1 writes src into the box of dst (the rest of
 * dst untouched).  The free-node selection of space_precond.py:273-320. */
iga_status iga_box_copy(int dtype, int ndim, const int32_t* n, const int32_t* lo,
                        const int32_t* m, int64_t ncols, const void* src, void* dst,
                        int scatter, iga_stream stream);

/* Arrowhead solve of the space-time FD (src/igaops/fastdiag/utils/
 * operations.py:5-93) in place on a complex tensor stored as re / im, time
 * index i (0..mt-1) slowest, spatial eigen-index j (0..ms-1) fastest:
 * H_ij = dt_i + lam_j (dt complex, (re, im) pairs), border b (mt-1 complex
 * pairs), Schur complement formed on the fly. */
iga_status iga_arrowhead_solve(int dtype, int mt, int64_t ms, const double* dt,
                               const double* b, const double* lam, void* re, void* im,
                               iga_stream stream);

/* Space-time FD apply (SpTimeFD.apply / apply_transpose,
 * src/igaops/fastdiag/utils/time_arrow.py:112-192): sdim space directions
 * plus time (last, slowest); n/lo/m hold sdim+1 entries (time: lo = 1,
 * m = nt - 1); U[d] the m_d x m_d space eigenvectors; ut_re / ut_im the
 * time eigenvectors (m_t x m_t, row-major); dt = adv * arrowhead diagonal,
 * bfac = adv * g (apply) or -conj(adv * g) (transpose), complex pairs; lam
 * the combined space eigenvalues (prod m_space).  y is zero off the free box.
 * work0..2: prod(m) elements each. */
iga_status iga_fd_sptime_apply(int dtype, int sdim, const int32_t* n, const int32_t* lo,
                               const int32_t* m, const void* const* U, const void* ut_re,
                               const void* ut_im, const double* dt, const double* bfac,
                               const double* lam, int transpose, const void* x, void* y,
                               void* work0, void* work1, void* work2, iga_stream stream);

/* Space-time FD in the QZ ("legacy") form (SpTimeFD.apply / apply_transpose
 * of src/igaops/fastdiag/utils/time_legacy.py:61-170, selected by
 * SingleFD.compute_time_schurdecomposition(..., use_arrowhead=False),
 * src/igaops/fastdiag/preconditioner.py:66-86): same box and space passes as
 * iga_fd_sptime_apply; in time Q^H, then per spatial eigen-index j the
 * triangular solve with adv*S + lam[j]*T, then Z (apply) -- or Z^T, the
 * transposed solve and conj(Q) (transpose).  q_*, z_*: real / imaginary
 * parts of Q and Z (m_t x m_t, row-major, element type of the call); S, Tm:
 * the complex Schur forms as (re, im) pairs, row-major. */
iga_status iga_fd_sptime_qz_apply(int dtype, int sdim, const int32_t* n, const int32_t* lo,
                                  const int32_t* m, const void* const* U, const void* q_re,
                                  const void* q_im, const void* z_re, const void* z_im,
                                  const double* S, const double* Tm, double adv,
                                  const double* lam, int transpose, const void* x, void* y,
                                  void* work0, void* work1, void* work2, iga_stream stream);

/* --------------------------------------------------------------------- */
/* Krylov primitives                                                      */
/* --------------------------------------------------------------------- */

/* Scratch size of iga_gram: number of partial blocks and FP64 elements. */
iga_status iga_gram_workspace(int64_t n, int m1, int m2, int cplx, int* nblk,
                              int64_t* elems);

/* out[j1*m2 + j2] = sum_i conj(A_j1[i]) B_j2[i] (FP64 accumulation, fixed
 * reduction order); A_j = A + j*lda, B_j = B + j*ldb (elements; complex
 * values are (re, im) pairs and count as one element).  `partial` is the
 * caller's scratch of iga_gram_workspace size.  The dot products and
 * Gram-Schmidt projections of src/igaops/solvers/linear_solver.py:481-490 and
 * src/igaops/solvers/deflated/helpers.py:46-55,118-130 and the overlaps of
 * src/igaops/solvers/deflated/gcrodr.py:266-273,327-340. */
iga_status iga_gram(int dtype, int cplx, int64_t n, int m1, const void* A,
                    int64_t lda, int m2, const void* B, int64_t ldb, double* out,
                    double* partial, int nblk, iga_stream stream);

/* iga_gram for callers that cannot allocate device memory -- for example a
 * host program that links only this C ABI and owns no device allocator, or
 * code that must not call cudaMalloc because that would synchronize the
 * device mid-pipeline.  No counterpart in the reference (whose dot products
 * are numpy calls).  Same arguments and result as iga_gram minus the
 * scratch: the partial sums live in a 512 KiB array (65536 doubles) built
 * into the library (held on every GPU that loads it until exit).  Limit:
 * m1*m2 <= 4096 pairs, as for iga_gram; larger requests return
 * IGA_ERR_INVALID_ARG.  The array also bounds the reduction blocks of one
 * call to 65536 / (m1*m2, twice that for complex), so wide requests run with
 * fewer blocks than iga_gram_workspace would give them.  The first call on
 * each device looks up the array's device address (cudaGetSymbolAddress with
 * that device current), so make that first call before any stream capture;
 * the address is kept for the life of the device's context and looked up
 * again when another context is current (e.g. after cudaDeviceReset).  All
 * calls share the array: calls that overlap on the GPU (e.g. on two streams
 * at once) race.  Nothing is allocated, freed or cleared. */
iga_status iga_gram_noalloc(int dtype, int cplx, int64_t n, int m1,
                            const void* A, int64_t lda, int m2, const void* B,
                            int64_t ldb, double* out, iga_stream stream);

/* out_k = beta*out_k + alpha * sum_j coef[j*kout + k] A_j for k < kout
 * (coef on the device, FP64 or complex FP64).  Gram-Schmidt updates, x = Z y
 * and basis rotations (linear_solver.py:484-503, gcrodr.py:271,291,329,
 * 344-362). */
iga_status iga_combine(int dtype, int cplx, int64_t n, int m_in, const void* A,
                       int64_t lda, int kout, const double* coef, double alpha,
                       double beta, void* out, int64_t ldo, iga_stream stream);

/* x *= s[0] (invert = 1: x /= s[0]; invert = 2: x /= sqrt(s[0]), the
 * normalisation by a squared norm that a Gram call left on the device, with a
 * zero norm giving x = 0) with s on the device. */
iga_status iga_scale_dev(int dtype, int cplx, int64_t n, void* x, const double* s,
                         int invert, iga_stream stream);

/* x[idx[i]] = 0 (the Dirichlet mask of linear_solver.py:119-124). */
iga_status iga_mask_zero(int dtype, int64_t nidx, const int64_t* idx, void* x,
                         iga_stream stream);

/* dst = (dtype_out) src, FP64 <-> FP32. */
iga_status iga_convert(int dtype_in, int dtype_out, int64_t n, const void* src,
                       void* dst, iga_stream stream);

/* complex (interleaved) <-> real / imaginary planes (GCRO-DR applies real
 * operators to complex vectors part by part, gcrodr.py:147-162). */
iga_status iga_complex_split(int64_t n, const double* z, double* re, double* im,
                             iga_stream stream);
iga_status iga_complex_merge(int64_t n, const double* re, const double* im,
                             double* z, iga_stream stream);

/* BF16 elements of each work buffer of iga_fd_apply_tc for free extents m[3]. */
iga_status iga_fd_tc_workspace(const int32_t* m, int64_t* elems);

/* 3D FD apply with the mode products on the tensor cores (tcgen05, BF16
 * operands, FP32 accumulation in tensor memory).  Bfwd[d] / Bbwd[d] are the
 * images of U_d^T / U_d padded to Kp = Np = 16*ceil(m_d/16) and laid out in
 * 8x8 core matrices (core (g, kc) of rows 8g.. and columns 8kc.. at element
 * offset (kc*Np/8 + g)*64, rows of 8 contiguous elements); inv_lambda is FP32
 * (prod(m), direction 1 fastest); x, y are full FP32/FP64 vectors (io_dtype),
 * y zero outside the free box; work0/work1 hold iga_fd_tc_workspace BF16
 * elements each and are zeroed once by the caller before the first call.
 * *status (device) receives IGA_ERR_TIMEOUT if a bounded wait gave up.
 * Accuracy is that of BF16 (about 1e-2 relative); FGMRES refines it.
 * Replaces SpaceFD.apply (space_precond.py:273-320) inside preconditioners. */
iga_status iga_fd_apply_tc(int io_dtype, const int32_t* n, const int32_t* lo,
                           const int32_t* m, const void* const* Bfwd,
                           const void* const* Bbwd, const float* inv_lambda,
                           const void* x, void* y, void* work0, void* work1,
                           int32_t* status, iga_stream stream);

/* --------------------------------------------------------------------- */
/* Weighted-quadrature rules (host computation)                           */
/* --------------------------------------------------------------------- */

/* Weight rows of a weighted-quadrature rule, computed on the host (no
 * device work): for each row i, W[i] = Z[i] * v_i with v_i the minimum-norm
 * least-squares solution of (A diag(Z[i])) v = B[i] (complete orthogonal
 * decomposition; pivots below rcond * the largest dropped) -- the solution
 * of the rule construction's optimisation problem, which the reference
 * approximates by LSQR (src/igaops/quadrature/utils/operations.py:107-143).  A: nt x npts, Z and W: nrows x npts, B: nrows x nt, all
 * row-major FP64 host arrays. */
iga_status iga_wq_min_norm_rows(int nrows, int nt, int npts, const double* A,
                                const double* Z, const double* B, double rcond,
                                double* W);

/* Non-zero B-spline basis functions of degree `degree` on the knot vector
 * U (nknots knots) and their derivatives up to order nders at npts points
 * x (host computation; Piegl & Tiller A2.1 / A2.3, the basis evaluation
 * of src/igaops/quadrature/utils/operations.py:53-105 through geomdl's
 * helpers): span[i] = the knot span of x[i] (the last s in [p, n-1] with
 * U[s] <= x[i]); ders[(k * (p + 1) + j) * npts + i] = the k-th derivative of
 * basis function span[i] - p + j at x[i]. */
iga_status iga_bspline_basis(int degree, int nknots, const double* U, int64_t npts,
                             const double* x, int nders, int32_t* span, double* ders);

/* Points per element of a weighted-quadrature rule (the point-count tables
 * of src/igaops/quadrature/utils/wq_helpers.py:11-82,221-259).
 * test_range / targ_range: (first, last) element covered with positive
 * measure by each test / target basis function (2 ints each).  counts[e] =
 * 1 + the largest number of (test, target) pairs of one test function whose
 * shared element interval is element e; *feasible = 1 when every
 * multi-element range then holds enough points for the pairs inside it,
 * else 0 (the counts are a lower bound for the integer program). */
iga_status iga_wq_point_counts(int ne, int ntest, const int32_t* test_range, int ntarg,
                               const int32_t* targ_range, int32_t* counts,
                               int32_t* feasible);

/* --------------------------------------------------------------------- */
/* Many patches in one launch                                             */
/* --------------------------------------------------------------------- */
/* Independent patches solved together keep their vectors in one flat array:
 * patch p owns elements [offsets[p], offsets[p] + N_p).  No counterpart in
 * the reference, which handles one patch per call; each call below runs the
 * arithmetic of the single-patch entry point it names for every patch. */

/* Bytes of the device table of a multi-patch fused matvec. */
iga_status iga_mf_batch_table_bytes(int dtype, int npatch, int64_t* bytes);

/* Fill the device table (256-byte aligned, synchronous copies) of a
 * multi-patch fused matvec over plans[0..npatch-1] (3D, no time direction,
 * same op, symmetry, band width and face; each with its packed coefficients
 * and step table as for iga_mf_matvec).  Returns the CTA count of the launch
 * and its dynamic shared memory. */
iga_status iga_mf_batch_prepare(const iga_mf_plan* plans, int npatch, int dtype,
                                const void* const* packed, const int64_t* offsets,
                                void* table, int32_t* total_ctas, int64_t* smem_bytes);

/* y = A_p x on every patch of the table in one launch (the arithmetic of
 * iga_mf_matvec per patch).  zero_y: clear y[0 .. ntot) first (give 0 when
 * an earlier launch of the same flat y already did).  skip (device, npatch,
 * or NULL): patches with skip[p] >= 0 are not computed (their y stays as
 * cleared) -- a batched solver passes its per-patch convergence step; p is
 * the patch's position in THIS table (a solver that splits its patches over
 * several tables by band width gathers each table's flags). */
iga_status iga_mf_batch_matvec(const iga_mf_plan* plan0, int dtype, int npatch,
                               const void* table, int32_t total_ctas,
                               int64_t smem_bytes, const void* x, void* y,
                               int64_t ntot, int zero_y, const int32_t* skip,
                               iga_stream stream);

/* Bytes of the device table of a multi-patch tensor-core FD apply. */
iga_status iga_fd_tc_batch_table_bytes(int npatch, int64_t* bytes);

/* Fill the table of a multi-patch iga_fd_apply_tc: per patch p, n/lo/m at
 * [3p..3p+2], the B images Bfwd/Bbwd at [3p..3p+2], inv_lambda[p],
 * work0[p] / work1[p] (zeroed once, iga_fd_tc_workspace elements each) and
 * offsets[p].  Returns the grid of each of the six products (grid[6]) and
 * the dynamic shared memory. */
iga_status iga_fd_tc_batch_prepare(int npatch, const int32_t* n, const int32_t* lo,
                                   const int32_t* m, const void* const* Bfwd,
                                   const void* const* Bbwd,
                                   const float* const* inv_lambda,
                                   void* const* work0, void* const* work1,
                                   const int64_t* offsets, int io_dtype,
                                   int32_t* status, void* table, int32_t* grid,
                                   int64_t* smem);

/* y = P_p^{-1} x for every patch (six launches in all; y[0 .. ntot) is
 * cleared first); skip as for iga_mf_batch_matvec. */
iga_status iga_fd_tc_batch_apply(int io_dtype, int npatch, const void* table,
                                 const int32_t* grid, int64_t smem, const void* x,
                                 void* y, int64_t ntot, const int32_t* skip,
                                 iga_stream stream);

/* Segmented Krylov primitives: offs (device, npatch+1) bound the patches;
 * blk0 (device, npatch+1) numbers the blocks of at most iga_seg_chunk()
 * elements each patch is split into (nblk = blk0[npatch]). */
int iga_seg_chunk(void);

/* out[p*ldo + j] = sum_{i in p} A_j[i] x[i], j < m <= 32, FP64 accumulation,
 * fixed reduction order; partial: nblk*m doubles of scratch. */
iga_status iga_seg_gram(int dtype, int npatch, const int64_t* offs, const int32_t* blk0,
                        int nblk, int m, const void* A, int64_t lda, const void* x,
                        double* partial, double* out, int64_t ldo, iga_stream stream);

/* out[i] = beta*out[i] + alpha * sum_j coef[p*ldc + j] A_j[i] for i in p. */
iga_status iga_seg_combine(int dtype, int npatch, const int64_t* offs, const int32_t* blk0,
                           int nblk, int m, const void* A, int64_t lda, const double* coef,
                           int64_t ldc, double alpha, double beta, void* out,
                           iga_stream stream);

/* x[i] *= f(s[p*lds]) for i in p; mode 0: f = s, 1: 1/s, 2: 1/sqrt(s) (0 for s <= 0). */
iga_status iga_seg_scale(int dtype, int npatch, const int64_t* offs, const int32_t* blk0,
                         int nblk, void* x, const double* s, int64_t lds, int mode,
                         iga_stream stream);

/* Per-patch Givens form of the GMRES least squares
 * (src/igaops/solvers/linear_solver.py:492-497).  H: npatch x m x (m+1),
 * column j of patch p at H[p*m*(m+1) + j*(m+1)]: rows 0..j the first
 * Gram-Schmidt projections, row j+1 the squared norm of the new vector.
 * init: g = (sqrt(beta2_p), 0, ...), conv = -1.  step j: adds the second
 * projections h2[p*ldh2 + i], rotates, residual resid[p] = |g[j+1]|, and sets
 * conv[p] = j at the first step with resid < tol * ref[p]; from then on
 * resid[p] keeps that step's residual.  trisolve: y =
 * R^{-1} g over the first conv[p]+1 (else k) columns, zero beyond. */
iga_status iga_seg_givens_init(int npatch, int m, const double* beta2, double* g,
                               int32_t* conv, double* resid, iga_stream stream);
iga_status iga_seg_givens_step(int npatch, int m, int j, double* H, const double* h2,
                               int64_t ldh2, double* cs, double* sn, double* g,
                               const double* ref, double tol, int32_t* conv,
                               double* resid, iga_stream stream);
iga_status iga_seg_trisolve(int npatch, int m, int k, const double* H, const double* g,
                            const int32_t* conv, double* y, iga_stream stream);

/* --------------------------------------------------------------------- */
/* Geometry at quadrature points                                          */
/* --------------------------------------------------------------------- */

/* From the Jacobian jac (ncoord, ndim, nq) (d x_m / d xi_j, as returned by
 * eval_jacobien) computes, per quadrature point, G = J^T J,
 * det_out = sqrt(det G), invjac_out = G^{-1} J^T (ndim, ncoord, nq) and
 * coef_out = det_out * J^+ J^{+T} (ndim, ndim, nq), the stiffness
 * coefficients; any output may be NULL.  *status (device) is OR-ed with 1
 * where |det G| < 1e-14 and with 2 where det J <= 0 (or NaN).  Replaces
 * Operations.inverse_rectangular_matrix / eval_inverse_and_determinant
 * (src/igaops/geometry/mixin/operations.py:73-159). */
iga_status iga_geometry_pointwise(int ndim, int ncoord, int64_t nq,
                                  const double* jac, double* det_out,
                                  double* invjac_out, double* coef_out,
                                  int32_t* status, iga_stream stream);

/* --------------------------------------------------------------------- */
/* Rational (NURBS) operators                                             */
/* --------------------------------------------------------------------- */

/* Per-point coefficient streams of NurbsOperations.compute_mf_scalar_<op>
 * (src/igaops/operators/nurbs_ops.py:320-463; weight projections :14-62).
 * wq (nq) is the interpolated NURBS weight W at the quadrature points, dwq
 * (>= sp rows, row stride nq) its parametric gradient; w = 1/W,
 * z_k = dwq_k w^2.  coef is (nq) for IGA_OP_MASS, (sp, sp, nq) for
 * IGA_OP_STIFF, (sp, nq) for IGA_OP_GRADU_V / IGA_OP_U_GRADV.
 *   out_main = coef * w^2                      (same shape as coef)
 *   out_uv   = sum_ij C_ij z_i z_j   (STIFF)  |  sum_i c_i z_i w  (GRADU_V, U_GRADV)
 *   out_ug[j] = sum_i C_ij z_i w,  out_gu[i] = sum_j C_ij z_j w  (STIFF, (sp, nq))
 * Unused outputs may be NULL.  *status (device) is OR-ed with 1 where W == 0. */
iga_status iga_nurbs_coefficients(int op, int sp, int64_t nq, const double* coef,
                                  const double* wq, const double* dwq,
                                  double* out_main, double* out_uv,
                                  double* out_ug, double* out_gu,
                                  int32_t* status, iga_stream stream);

#ifdef __cplusplus
}
#endif

#endif /* IGAB200_H */
