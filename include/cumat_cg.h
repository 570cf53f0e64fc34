/*
 * cumat_cg.h — C ABI of the sm_100a batched sparse conjugate-gradient library.
 *
 * This is the drop-in boundary for cuMat's batched sparse iterative-solve path.
 * The reference (shamanDevel/cuMat) is a header-only C++ template library with
 * no FFI; each entry point below names the reference interface it replaces
 * (paths relative to the reference repository). The C++ facade in
 * include/cuMat/ re-exposes those names on top of this ABI.
 *
 * Conventions
 *  - Every function returns a cmcg_status; 0 is success. On failure a message
 *    is kept per host thread and returned by cmcg_last_error_string(). No C++
 *    exception crosses this boundary (the reference throws cuda_error /
 *    std::invalid_argument, cuMat/src/Errors.h:17-30, Macros.h:158-165).
 *  - Handles are library-owned and destroyed explicitly. A pattern is shared by
 *    the matrices created on it (reference: SparseMatrix shares its
 *    SparsityPattern, cuMat/src/SparseMatrix.h:42).
 *  - One CUDA stream per context (reference: one stream per host thread,
 *    cuMat/src/Context.h:204-214). Work is enqueued on that stream; calls on a
 *    context are not re-entrant.
 *  - Vector and value pointers passed to compute entry points are DEVICE
 *    pointers unless the name or an `is_device` flag says otherwise. Index
 *    arrays are int32 (reference StorageIndex = int,
 *    cuMat/src/SparseMatrixBase.h:98).
 *  - Batches: a matrix holds `batches` value sets on one pattern, stored
 *    batch-major ([batch][nnz] for CSR, [batch][slot][row] for ELLPACK), like
 *    the reference's data matrix (SparseMatrix.h:71). Vectors are [batch][n].
 *    A one-batch matrix or vector broadcasts against the other operand.
 */
#ifndef CUMAT_CG_H
#define CUMAT_CG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t cmcg_status;
enum {
    CMCG_OK = 0,
    CMCG_ERR_INVALID_ARGUMENT = 1,
    CMCG_ERR_CUDA = 2,
    CMCG_ERR_OUT_OF_MEMORY = 3,
    CMCG_ERR_NOT_SUPPORTED = 4,
    CMCG_ERR_INTERNAL = 5
};

/* element types */
enum { CMCG_F32 = 0, CMCG_F64 = 1, CMCG_BF16 = 2 };
/* storage formats (reference SparseFlags, cuMat/src/Constants.h; BSR, block
 * CSR, has no reference SparseFlags value: the reference stores blocks as a
 * block scalar type in a CSR pattern) */
enum { CMCG_CSR = 0, CMCG_ELLPACK = 1, CMCG_CSC = 2, CMCG_BSR = 3 };
/* preconditioners (reference ConjugateGradient.h:218-265) */
enum { CMCG_PRECOND_IDENTITY = 0, CMCG_PRECOND_JACOBI = 1 };
/* assignment modes of a product (reference AssignmentMode ASSIGN / ADD / SUB) */
enum { CMCG_ASSIGN = 0, CMCG_ADD = 1, CMCG_SUB = 2 };
/* per-system outcome of a solve */
enum {
    CMCG_SOLVE_CONVERGED = 0,   /* |r|^2 < tol^2 |b|^2 */
    CMCG_SOLVE_MAX_ITER = 1,    /* iteration limit reached */
    CMCG_SOLVE_ZERO_RHS = 2,    /* |b|^2 < tol^2: x = 0, no iteration */
    CMCG_SOLVE_BREAKDOWN = 3,   /* p.Ap <= 0 or r.z <= 0 (matrix not SPD) */
    CMCG_SOLVE_NON_FINITE = 4   /* NaN / Inf met in a scalar of the iteration */
};
/* solver execution paths (cmcg_cg_set_path) */
enum {
    CMCG_PATH_AUTO = 0,
    CMCG_PATH_PERSISTENT = 1,         /* one CTA per system, whole loop in one launch; FP32
                                         vectors of systems up to 16384 rows live in shared memory */
    CMCG_PATH_GRID = 2,               /* grid-wide fused kernels per iteration, CUDA graph */
    CMCG_PATH_PERSISTENT_GLOBAL = 3   /* persistent, vectors in global memory (comparison) */
};
/* mixed-precision methods (cmcg_cg_set_refinement) */
enum {
    CMCG_REFINE_RELIABLE = 0,   /* FP32 CG with FP64 residual replacement ("reliable updates") */
    CMCG_REFINE_RESTART = 1     /* classical refinement: restart FP32 CG on each FP64 residual */
};

typedef struct cmcg_ctx_s* cmcg_ctx;
typedef struct cmcg_pattern_s* cmcg_pattern;
typedef struct cmcg_matrix_s* cmcg_matrix;
typedef struct cmcg_solver_s* cmcg_solver;

/* ---- runtime ------------------------------------------------------------ */

/* Last error message of this host thread ("" when none). */
const char* cmcg_last_error_string(void);
/* ABI version, major * 10000 + minor * 100 + patch. */
int32_t cmcg_version(void);
/* Number of kernel launches this library issued on this host thread
 * (reference test hook: CUMAT_PROFILING counters, cuMat/src/Profiling.h:23-145). */
int64_t cmcg_launch_count(void);

/* Context = device + stream (reference Context, cuMat/src/Context.h:132-214).
 * stream == NULL creates a private non-blocking stream; any cudaStream_t,
 * cudaStreamLegacy ((void*)1) included, is used as given. */
cmcg_status cmcg_ctx_create(int32_t device, void* stream, cmcg_ctx* out);
cmcg_status cmcg_ctx_destroy(cmcg_ctx ctx);
cmcg_status cmcg_ctx_synchronize(cmcg_ctx ctx);

/* Device memory for callers that do not link a CUDA runtime themselves (the
 * C++ facade's dense vectors). Reference: Context::mallocDevice / freeDevice
 * (cuMat/src/Context.h:271-286) and Matrix::copyFromHost / copyToHost
 * (cuMat/src/Matrix.h:847-858). cmcg_device_free waits for the context's
 * queued work; cmcg_memcpy returns after host<->device copies completed and
 * queues device-to-device copies on the context stream. */
enum { CMCG_HOST_TO_DEVICE = 0, CMCG_DEVICE_TO_HOST = 1, CMCG_DEVICE_TO_DEVICE = 2 };
cmcg_status cmcg_device_alloc(cmcg_ctx ctx, int64_t bytes, void** out);
cmcg_status cmcg_device_free(cmcg_ctx ctx, void* p);
cmcg_status cmcg_memcpy(cmcg_ctx ctx, void* dst, const void* src, int64_t bytes, int32_t kind);
cmcg_status cmcg_memset_zero(cmcg_ctx ctx, void* dst, int64_t bytes);
cmcg_status cmcg_ctx_stream(cmcg_ctx ctx, void** stream);
/* Log hook (no reference counterpart; the reference has no logging): the
 * library reports what it decided and what went wrong (the kernel a product
 * or reduction tuned to, the execution path and CTA tiers of a solve, systems
 * re-solved with FP32 values, failures with their message) through
 * callback(level, message, user) with level 0 = error, 1 = info, 2 = detail,
 * for every message at or below max_level. NULL removes the callback.
 * CUMAT_LOG=<level> in the environment logs to stderr instead when no
 * callback is set. Solves, products and reductions are also marked as NVTX
 * ranges ("cmcg_cg_solve", ...) for Nsight timelines. */
typedef void (*cmcg_log_fn)(int32_t level, const char* message, void* user);
cmcg_status cmcg_set_log_callback(cmcg_log_fn callback, int32_t max_level, void* user);

/* Synchronises and returns (then clears) the context's device error bits:
 * bit 0 = a bulk-copy (mbarrier) wait ran out, bit 1 = a grid-barrier wait of
 * the cooperative solver ran out. Every device-side wait is bounded (no
 * reference counterpart; the reference has no device-side waits). */
cmcg_status cmcg_ctx_device_errors(cmcg_ctx ctx, int32_t* flags);

/* ---- sparsity patterns --------------------------------------------------- */

/* CSR pattern (reference SparsityPattern<CSR>, cuMat/src/SparseMatrixBase.h:89-147:
 * JA = row_ptr (rows+1), IA = col_idx (nnz)). Validated on the host: rows, cols
 * > 0; row_ptr[0] == 0, non-decreasing, row_ptr[rows] == nnz; 0 <= col < cols.
 * Index arrays are host pointers unless is_device != 0. */
cmcg_status cmcg_pattern_create_csr(cmcg_ctx ctx, int32_t rows, int32_t cols, int64_t nnz,
                                    const int32_t* row_ptr, const int32_t* col_idx, int32_t is_device,
                                    cmcg_pattern* out);
/* ELLPACK pattern (reference SparsityPattern<ELLPACK>, SparseMatrixBase.h:149-206):
 * indices is rows x nnz_per_row, column-major, -1 marks padding. Validated:
 * 0 < nnz_per_row <= cols, every index in [-1, cols). */
cmcg_status cmcg_pattern_create_ell(cmcg_ctx ctx, int32_t rows, int32_t cols, int32_t nnz_per_row,
                                    const int32_t* indices, int32_t is_device, cmcg_pattern* out);
/* CSC pattern (reference SparsityPattern<CSC>, SparseMatrixBase.h:29-87:
 * JA = col_ptr (cols+1), IA = row_idx (nnz)). Validated like CSR with rows and
 * columns exchanged. Values of matrices on it are given and returned in CSC
 * (column) order; products, solves and reductions run on the equivalent CSR
 * pattern, whose value order is a permutation of the caller's. */
cmcg_status cmcg_pattern_create_csc(cmcg_ctx ctx, int32_t rows, int32_t cols, int64_t nnz, const int32_t* col_ptr,
                                    const int32_t* row_idx, int32_t is_device, cmcg_pattern* out);
/* Block CSR pattern of block_rows x block_cols blocks of block_size x
 * block_size (2 .. 8) entries: row_ptr (block_rows+1) and col_idx (nnz_blocks)
 * index blocks. The reference's blocked solver (a block scalar type such as a
 * row-major float3x3 in a CSR pattern with float3 vectors,
 * tests/TestBlockedConjugateGradient.cu:10-237, ConjugateGradient.h:47-61).
 * Values are block_size^2 per block, row-major, in block order; vectors hold
 * block_size entries per block row. The pattern is block_rows * block_size
 * square rows for every other call; each block row expands to block_size
 * scalar rows, so products, CG (Jacobi = inverse of the scalar diagonal, the
 * reference's ExtractDiagonalFunctor + cwiseInverseCheck) and the
 * mixed-precision solves apply unchanged. */
cmcg_status cmcg_pattern_create_bsr(cmcg_ctx ctx, int32_t block_rows, int32_t block_cols, int32_t block_size,
                                    int64_t nnz_blocks, const int32_t* row_ptr, const int32_t* col_idx,
                                    int32_t is_device, cmcg_pattern* out);
/* Partitions a square pattern into n_sys independent diagonal blocks
 * (system i owns rows and columns [row_off[i], row_off[i+1])). Fails if an
 * entry couples two systems. No reference counterpart (the reference needs one
 * shared pattern per batch, cuMat/src/SparseProductEvaluation.h:113-114). */
cmcg_status cmcg_pattern_set_systems(cmcg_pattern p, int64_t n_sys, const int64_t* row_off);
/* rows, cols, nnz (stored scalar entries incl. ELL padding), format (as
 * created: CSR, ELLPACK, CSC or BSR), n_sys, width (ELL; BSR: block size). */
cmcg_status cmcg_pattern_info(cmcg_pattern p, int32_t* rows, int32_t* cols, int64_t* nnz, int32_t* format,
                              int64_t* n_sys, int32_t* width);
/* Copies the pattern's index arrays, as given at creation, to host memory
 * (row_ptr/col_idx; CSC col_ptr/row_idx; BSR block row_ptr/col_idx; or the
 * column-major ELL indices in row_ptr_or_idx, col_idx unused). */
cmcg_status cmcg_pattern_download(cmcg_pattern p, int32_t* row_ptr_or_idx, int32_t* col_idx);
cmcg_status cmcg_pattern_destroy(cmcg_pattern p);

/* ---- matrices -------------------------------------------------------------- */

/* Matrix of `batches` value sets of type dtype on pattern p
 * (reference SparseMatrix<Scalar, Batches, Flags>, cuMat/src/SparseMatrix.h:48-414).
 * Values start at zero. */
cmcg_status cmcg_matrix_create(cmcg_pattern p, int32_t dtype, int32_t batches, cmcg_matrix* out);
/* Uploads values, batch-major, converting from src_dtype (F32 / F64 / BF16; to
 * BF16 rounds to nearest even). ELL padding values are stored as given but
 * never read by a product (reference: unspecified, tests/TestSparseMatrix.cu:356-366).
 * (reference getData().copyFromHost, cuMat/src/Matrix.h:826-858) */
cmcg_status cmcg_matrix_set_values(cmcg_matrix m, int32_t src_dtype, const void* values, int32_t is_device);
/* Downloads values in the matrix dtype, batch-major, to host memory. */
cmcg_status cmcg_matrix_get_values(cmcg_matrix m, void* host_values);
/* dtype, batches. */
cmcg_status cmcg_matrix_info(cmcg_matrix m, int32_t* dtype, int32_t* batches);
cmcg_status cmcg_matrix_destroy(cmcg_matrix m);

/* ---- products and reductions ---------------------------------------------- */

/* y (mode)= A * x for every batch (reference operator*(SparseMatrix, vector),
 * cuMat/src/ProductOp.h:519-524, evaluated by ProductAssignment,
 * cuMat/src/SparseProductEvaluation.h:95-139 (CSR) and :232-276 (ELLPACK)).
 * x: [x_batches][cols] of vec_dtype (F32 or F64), y: [out_batches][rows].
 * out_batches = max(matrix batches, x_batches); a one-batch side broadcasts.
 * Rows without entries give 0. Device pointers. */
cmcg_status cmcg_spmv(cmcg_matrix A, int32_t vec_dtype, const void* x, int32_t x_batches, void* y,
                      int32_t mode);

/* y (mode)= A^T * x for every batch (no reference product: the reference's
 * product kernels leave transposed operands as a TODO,
 * SparseProductEvaluation.h:94). x: [x_batches][rows], y: [out_batches][cols].
 * CSR-equivalent patterns (CSR, CSC, BSR) only: thread per column of A over
 * the pattern's transpose (built once per pattern), values read through the
 * transpose's entry map; no atomics, deterministic. */
cmcg_status cmcg_spmv_transposed(cmcg_matrix A, int32_t vec_dtype, const void* x, int32_t x_batches, void* y,
                                 int32_t mode);

/* Dense <-> sparse on the pattern (reference: assignment of a sparse matrix
 * to a dense one and of a dense expression to a sparse matrix, evaluated
 * coefficient-wise on the pattern: SparseEvaluation.h:15-34, tests
 * TestSparseMatrix.cu:10-384). dense: device, [batches][rows][cols] when
 * row_major, else [batches][cols][rows], of the matrix dtype. to_dense writes
 * zeros off the pattern; from_dense takes the dense values at the pattern's
 * entries (a sparse view of the dense matrix). */
cmcg_status cmcg_matrix_to_dense(cmcg_matrix A, void* dense, int32_t row_major);
cmcg_status cmcg_matrix_from_dense(cmcg_matrix A, const void* dense, int32_t row_major);

/* out[b] = sum_i x[b][i] * y[b][i] for b < out_batches (reference
 * MatrixBase::dot, cuMat/src/ReductionOpsPlugin.inl:279-298); a one-batch
 * operand broadcasts. Sums in the vector type (F32 / F64) with warp shuffles
 * and one deterministic grid-level combine. out: device, out_batches values. */
cmcg_status cmcg_dot(cmcg_ctx ctx, int32_t dtype, int64_t n, const void* x, int32_t x_batches, const void* y,
                     int32_t y_batches, void* out);
/* out[b] = sum_i x[b][i]^2 (reference squaredNorm, ReductionOpsPlugin.inl:300-315). */
cmcg_status cmcg_squared_norm(cmcg_ctx ctx, int32_t dtype, int64_t n, const void* x, int32_t batches, void* out);
/* Same result as cmcg_dot, but this entry point allocates nothing: no cudaMalloc,
 * cudaFree or allocating library call. It has no counterpart in the reference.
 * It is for callers that may not let a library allocate device memory, for
 * instance because their own pool or framework allocator owns the device
 * memory, or because allocation and the synchronisation it can bring are not
 * allowed inside their loop. Its scratch is a fixed device array of about
 * 36 KB that every GPU loading this library holds until the process exits;
 * at most 1024 batches per call (more is rejected with CMCG_ERR_INVALID_ARGUMENT).
 * The first call on a device looks up the array's address with that device
 * current, so make that first call before any stream capture. All calls on a
 * device share the array: calls that overlap on the GPU (other streams,
 * other threads) race and must be serialised by the caller. */
cmcg_status cmcg_dot_noalloc(cmcg_ctx ctx, int32_t dtype, int64_t n, const void* x, int32_t x_batches, const void* y,
                             int32_t y_batches, void* out);

/* Reduction of a dense batched matrix along any set of axes (reference: the
 * sum / prod / minCoeff / maxCoeff reductions over rows, columns and batches,
 * cuMat/src/ReductionOps.h, ReductionOpsPlugin.inl, with the algorithm
 * selection of ReductionAlgorithmSelection.h:40-112). in: device,
 * [batches][cols][rows] (rows fastest, the reference's ColumnMajor), dtype F32
 * or F64; axes: a mask of CMCG_AXIS_ROW | CMCG_AXIS_COLUMN | CMCG_AXIS_BATCH
 * (0 copies); out: device, the kept axes in the same order. The kernel
 * (thread, warp or CTA per output, or outputs split over several CTAs) is
 * picked per shape by timing on first use and kept in memory and in the
 * tuning cache file; each kernel combines in a fixed order, so results are
 * deterministic for a given choice (MIN / MAX for any). */
enum { CMCG_REDUCE_SUM = 0, CMCG_REDUCE_PROD = 1, CMCG_REDUCE_MIN = 2, CMCG_REDUCE_MAX = 3 };
enum { CMCG_AXIS_ROW = 1, CMCG_AXIS_COLUMN = 2, CMCG_AXIS_BATCH = 4 };
cmcg_status cmcg_reduce(cmcg_ctx ctx, int32_t dtype, int32_t op, int64_t rows, int64_t cols, int64_t batches,
                        int32_t axes, const void* in, void* out);

/* out (mode)= sum_t coeffs[t] * v_t over n_terms <= 16 vectors, for every
 * batch, in one streaming pass (reference: the cwise evaluation of
 * `v0 * f0 + v1 * f1 + ...`, cuMat/src/CwiseOp.h:66-85, timed by
 * benchmarks/linear_combination/Implementation_cuMat.cu:52-66). vectors: host
 * array of n_terms device pointers, vector t holding v_batches[t] batches of n
 * elements (1 broadcasts, else out_batches); coeffs: host array; out: device
 * [out_batches][n]; dtype F32 or F64. Terms are added in order. */
cmcg_status cmcg_lincomb(cmcg_ctx ctx, int32_t dtype, int64_t n, int32_t n_terms, const double* coeffs,
                         const void* const* vectors, const int32_t* v_batches, void* out, int32_t out_batches,
                         int32_t mode);

/* out[k] = alpha * u[row(k)] * v[col(k)] for every stored entry k of batch b
 * (u: [u_batches][rows], v: [v_batches][cols], out: [out_batches][nnz] in the
 * matrix layout). The sparse outer product evaluated on a pattern (reference
 * SparseProductEvaluation.h:16-37 + SparseEvaluation.h:15-34), used as the
 * dL/dA kernel of the adjoint. vec_dtype F32 or F64; out has the same type.
 * ELL padding slots get 0. */
cmcg_status cmcg_sddmm(cmcg_matrix pattern_of, int32_t vec_dtype, double alpha, const void* u, int32_t u_batches,
                       const void* v, int32_t v_batches, void* out, int32_t out_batches);

/* ---- conjugate gradient ------------------------------------------------------ */

/* Creates a CG solver on a square matrix (reference
 * ConjugateGradient<SMatrix, Preconditioner>(A), cuMat/src/ConjugateGradient.h:96-112,
 * IterativeSolverBase.h:36-41). Jacobi extracts 1 / a_ii per batch (1 where the
 * diagonal is zero or absent: cwiseInverseCheck, UnaryOps.h:177). Defaults:
 * tolerance = epsilon of the matrix value type (IterativeSolverBase.h:131),
 * max iterations = 2 * (rows of the largest system) (IterativeSolverBase.h:83-86). */
cmcg_status cmcg_cg_create(cmcg_matrix A, int32_t precond, cmcg_solver* out);
cmcg_status cmcg_cg_destroy(cmcg_solver s);
/* reference setTolerance / setMaxIterations (IterativeSolverBase.h:64-95);
 * max_iter < 0 restores the default. */
cmcg_status cmcg_cg_set_tolerance(cmcg_solver s, double tol);
cmcg_status cmcg_cg_set_max_iterations(cmcg_solver s, int64_t max_iter);
cmcg_status cmcg_cg_get_settings(cmcg_solver s, double* tol, int64_t* max_iter);
/* Execution path (default AUTO). */
cmcg_status cmcg_cg_set_path(cmcg_solver s, int32_t path);
/* Mixed-precision method of cmcg_cg_solve_refined (default RELIABLE): the
 * FP32 recursive residual is replaced by the FP64 one whenever its norm has
 * dropped by delta since the last replacement. delta 0 (the default) picks
 * 0.01 for FP32 inner values (the recurrence then stays within about
 * eps_f32 / delta of the true residual) and 0.1 for BF16 inner values.
 * No reference counterpart. */
cmcg_status cmcg_cg_set_refinement(cmcg_solver s, int32_t method, double delta);
/* Solves A x = b for every (batch, system) with vec_dtype F32 or F64 vectors
 * (reference solve / solveWithGuess, SolverBase.h:33-37, IterativeSolverBase.h:118-124;
 * algorithm ConjugateGradient.h:123-206). guess may be NULL (zero guess).
 * b, guess, x: device [batches][n]; batches = max(matrix batches, b_batches).
 * Every system stops on its own convergence (the reference iterates all
 * batches until all converge). */
cmcg_status cmcg_cg_solve(cmcg_solver s, int32_t vec_dtype, const void* b, int32_t b_batches, const void* guess,
                          void* x);
/* Same with host buffers: uploads b (and guess), solves, downloads x. */
cmcg_status cmcg_cg_solve_host(cmcg_solver s, int32_t vec_dtype, const void* b_host, int32_t b_batches,
                               const void* guess_host, void* x_host);
/* reference iterations() / error() (IterativeSolverBase.h:97-111): the largest
 * iteration count and the largest sqrt(|r|^2 / |b|^2) over all systems of the
 * last solve. Synchronises the context stream. */
cmcg_status cmcg_cg_iterations(cmcg_solver s, int64_t* iterations);
cmcg_status cmcg_cg_error(cmcg_solver s, double* error);
/* Per-system results of the last solve, [batches * n_sys] in batch-major
 * order, host memory; any pointer may be NULL. For a refined solve, iters
 * counts inner iterations and outer receives the refinement steps. */
cmcg_status cmcg_cg_system_stats(cmcg_solver s, int32_t* iters, double* err, int32_t* status, int32_t* outer);

/* Mixed precision with FP64 iterative refinement (no reference counterpart):
 * b and x are FP64 [batches][n]. Outer loop in FP64: r = b - A x with the
 * matrix values as stored in `A_outer` (F32 or F64) evaluated in FP64; inner
 * solve A d = r with this solver's matrix (F32 or BF16 values, FP32 vectors,
 * tolerance = this solver's tolerance relative to |r|), x += d; stop when
 * |b - A x| < outer_tol |b| or after max_outer steps. A_outer may be NULL
 * (use the solver's matrix; it must then be F32 or F64). */
cmcg_status cmcg_cg_solve_refined(cmcg_solver s, cmcg_matrix A_outer, const double* b, int32_t b_batches,
                                  double* x, double outer_tol, int32_t max_outer);

/* BF16 inner values (no reference counterpart): rounding the Jacobi-scaled
 * values to BF16 perturbs them by up to 2^-9 relative, which stops the
 * refinement from contracting once that times the condition number nears 1.
 * cmcg_cg_solve_refined therefore checks every system after a BF16 solve and
 * solves the ones that did not converge again with FP32 values (those of
 * A_outer, rounded to FP32 when it is FP64), keeping their results; this
 * synchronises the context stream once per BF16 solve. Set
 * CUMAT_CG_BF16_FALLBACK=0 before creating the solver to keep the BF16
 * statuses. flags (may be NULL): per instance of the last solve, 1 where it
 * was re-solved with FP32 values; count: how many. */
cmcg_status cmcg_cg_fallbacks(cmcg_solver s, int32_t* flags, int64_t* count);

/* Adjoint of x = A^{-1} b for a loss L(x) (no reference counterpart):
 * solves A^T lambda = gx with this solver (A symmetric, so A lambda = gx;
 * FP64 refined to outer_tol with the solver's matrix), then writes
 * gb = lambda and gA[k] = -lambda[row(k)] * x[col(k)] on the pattern.
 * x: the forward solution (FP64, checkpointed by the caller; no iterate is
 * stored). All FP64 device [batches][n]; gA [batches][nnz] FP64 in the matrix
 * layout (may be NULL). */
cmcg_status cmcg_cg_adjoint(cmcg_solver s, cmcg_matrix A_outer, const double* x, const double* gx, int32_t batches,
                            double* gb, double* gA, double outer_tol, int32_t max_outer);

#ifdef __cplusplus
}
#endif

#endif /* CUMAT_CG_H */
