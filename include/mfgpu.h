/* mfgpu.h -- C ABI of libmfgpu.so, a B200 (sm_100a) multifrontal sparse LU.
 *
 * libmfgpu replaces the numeric multifrontal factorization and the triangular
 * solves of PureUMFPACK.jl behind the reference's own entry points:
 *
 *   splu(A; method=:multifrontal, scale, check)   src/interface.jl:93-120
 *   multifrontal_lu(A; q, tol, check)            src/multifrontal.jl:146-358
 *   PureUMFPACK.solve(F::PureLU, b; refine)       src/interface.jl:170-177
 *   F \ b                                         src/interface.jl:179, src/solve.jl:66-79
 *
 * and keeps UMFPACK's convention  (F.Rs .* A)[F.p, F.q] == F.L * F.U.
 *
 * Conventions
 *   - Every index array is int64 and 1-based, exactly the buffers of a Julia
 *     SparseMatrixCSC{Float64,Int64} / Vector{Int64}; values are double.
 *   - Functions return MFGPU_OK (0) on success, a positive column number k for
 *     a zero pivot at factor column k when `check` is set (the reference's
 *     SingularException(k)), or a negative MFGPU_ERR_* code.
 *   - The caller allocates every output buffer; sizes come from the *_sizes
 *     queries.  The library owns its device memory, one context per handle;
 *     handles are independent and may be used from different host threads
 *     (one thread per handle at a time).  No torch types cross this ABI.
 */
#ifndef MFGPU_H
#define MFGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  MFGPU_OK = 0,
  MFGPU_ERR_ARGUMENT = -1,      /* bad pointer, size or permutation (ArgumentError) */
  MFGPU_ERR_CUDA = -2,          /* CUDA runtime error; see mfgpu_last_error */
  MFGPU_ERR_NOMEM = -3,         /* device allocation failed */
  MFGPU_ERR_STATE = -4,         /* call order: factor before analyze, solve before factor */
  MFGPU_ERR_TIMEOUT = -5,       /* a bounded device wait ran out */
  MFGPU_ERR_DIMENSION = -6,     /* non-square matrix (DimensionMismatch) */
  MFGPU_ERR_INTERNAL = -7,
  MFGPU_ERR_NO_DEVICE = -8      /* no CUDA device / wrong architecture */
};

enum { MFGPU_SCALE_NONE = 0, MFGPU_SCALE_SUM = 1, MFGPU_SCALE_MAX = 2 }; /* src/scaling.jl:11 */

enum {
  MFGPU_PRECISION_FP64 = 0,  /* all-FP64 fronts: the plain form */
  MFGPU_PRECISION_MIXED = 1  /* FP32 fronts, FP64 refinement */
};

/* ------------------------------------------------------------------------
 * Host-side ordering and symbolic analysis (no GPU needed).  The Julia host
 * keeps its own code for these; they are here for hosts without it and give
 * identical output.
 * ---------------------------------------------------------------------- */

/* row_scaling(A, kind) -> Rs (src/scaling.jl:92-115). */
int mfgpu_row_scaling(int64_t n, const int64_t* colptr, const int64_t* rowval, const double* nzval, int32_t kind,
                      double* rs);

/* row_scaling of a Float32 matrix in Float32 arithmetic (src/scaling.jl:92-115
 * with R = real(Tv) = Float32). */
int mfgpu_row_scaling_f32(int64_t n, const int64_t* colptr, const int64_t* rowval, const float* nzval,
                          int32_t kind, float* rs);

/* row_scaling of a ComplexF64 matrix (src/scaling.jl:92-115 with
 * R = real(Tv) = Float64): values as interleaved (re, im) doubles, Julia's
 * ComplexF64 layout; |z| = hypot(re, im); Float64 Rs (the Rs that
 * mfgpu_factor_c64 takes). */
int mfgpu_row_scaling_c64(int64_t n, const int64_t* colptr, const int64_t* rowval, const double* nzval_ri,
                          int32_t kind, double* rs);

/* amd_order_sym(A; dense) (src/amd.jl:141-148): perm of 1:n. */
int mfgpu_amd_order(int64_t n, const int64_t* colptr, const int64_t* rowval, double dense, int64_t* perm);

/* colamd_order(A; dense) (src/amd.jl:183-188): AMD on the A'A column graph. */
int mfgpu_colamd_order(int64_t m, int64_t n, const int64_t* colptr, const int64_t* rowval, double dense,
                       int64_t* perm);

typedef struct mfgpu_symbolic mfgpu_symbolic;

/* symbolic_mf(A; q) (src/symbolic.jl:211-226); q may be NULL (AMD). */
int mfgpu_symbolic_create(int64_t n, const int64_t* colptr, const int64_t* rowval, const int64_t* q,
                          mfgpu_symbolic** out);
void mfgpu_symbolic_destroy(mfgpu_symbolic* sym);
/* Symbolic analysis of nsys independent systems (1-based CSC each) as one
 * block-diagonal forest: every system ordered (MFGPU_ORDER_AMD or
 * MFGPU_ORDER_COLAMD, dense = 10) and analysed by symbolic_mf on its own,
 * on all host cores, then concatenated -- the same object as symbolic_mf of
 * the block-diagonal matrix with the concatenated orders.  The batch API
 * analyses through it. */
int mfgpu_symbolic_create_batch(int64_t nsys, const int64_t* n, const int64_t* const* colptr,
                                const int64_t* const* rowval, int32_t ordering, mfgpu_symbolic** out);
/* Opt-in relaxed amalgamation of the supernodes (no counterpart in the
 * reference, which keeps fundamental supernodes, src/symbolic.jl:178-179): a
 * supernode ending right before its parent merges into it when the merged
 * supernode stays small or stores few extra zeros.  Fewer, larger fronts; the
 * factors then store explicit zeros, so their structure is no longer the
 * reference's. */
int mfgpu_symbolic_relax(mfgpu_symbolic* sym);
/* out4 = {n, nsuper, length(upd_idx), length(child_idx)} */
int mfgpu_symbolic_sizes(const mfgpu_symbolic* sym, int64_t* out4);
/* SymbolicMF fields (src/symbolic.jl:203-209), flattened, any pointer may be
 * NULL.  qf(n), parent(n; 0 = root), colcount(n) = length(colstruct[j]),
 * sstart(nsuper+1), upd_ptr/upd_idx = colstruct[last column of each
 * supernode], child_ptr/child_idx = childsupers. */
int mfgpu_symbolic_get(const mfgpu_symbolic* sym, int64_t* qf, int64_t* parent, int64_t* colcount, int64_t* sstart,
                       int64_t* upd_ptr, int64_t* upd_idx, int64_t* child_ptr, int64_t* child_idx);
/* predicted_fill(S) (src/symbolic.jl:230-237). */
int64_t mfgpu_symbolic_predicted_fill(const mfgpu_symbolic* sym);
/* _factor_colptrs (src/multifrontal.jl:73-104): Lcolptr, Ucolptr (n+1 each). */
int mfgpu_factor_colptrs(const mfgpu_symbolic* sym, int64_t* lcolptr, int64_t* ucolptr);
const char* mfgpu_host_last_error(void);

/* ------------------------------------------------------------------------
 * GPU numeric factorization and solves.
 * ---------------------------------------------------------------------- */

typedef struct mfgpu_ctx mfgpu_ctx;

/* mfgpu_options.flags */
enum {
  MFGPU_FLAG_NO_TENSOR_CORES = 1,  /* FP32 fronts: CUDA-core FP32 GEMMs instead of tcgen05 */
  MFGPU_FLAG_PERSISTENT_SOLVE = 2, /* solves: one cooperative persistent launch per pass (slower than the
                                      default per-step launches on every measured case; kept for comparison) */
  MFGPU_FLAG_TF32_SPLIT = 4,       /* tensor-core GEMMs of FP32 fronts as 3xTF32 (two-part split, about 2^-21)
                                      instead of BF16x3 (three-part split, FP32 accuracy) */
  MFGPU_FLAG_STEP_SOLVE = 8,       /* solves: one launch per step (the default) */
  MFGPU_FLAG_LEAN_FRONTS = 16,     /* front memory reused by lifetime with a compact panel pool, whatever the
                                      size (default: only when all fronts would not fit in 45% of the device) */
  MFGPU_FLAG_NO_FRONT_MERGE = 32   /* factor every supernode as its own front.  Default: chains of supernodes
                                      (a child ending right before its parent) that stay small or store few
                                      zeros together are factored as one front, with the pivot search kept
                                      inside each original supernode's pivot rows and the factor's structure
                                      unchanged; this saves contribution-block hand-overs and tree levels */
};

typedef struct {
  int32_t device;     /* CUDA device ordinal */
  int32_t precision;  /* MFGPU_PRECISION_* */
  int32_t flags;      /* MFGPU_FLAG_* bits, 0 = defaults */
  int32_t reserved;
} mfgpu_options;

int mfgpu_create(const mfgpu_options* opts, mfgpu_ctx** out);
void mfgpu_destroy(mfgpu_ctx* h);
const char* mfgpu_last_error(const mfgpu_ctx* h);
/* Work is issued on this stream (a cudaStream_t; NULL = the handle's own). */
int mfgpu_set_stream(mfgpu_ctx* h, void* cuda_stream);
int mfgpu_set_precision(mfgpu_ctx* h, int32_t precision);
/* Mixed form: after the FP32 factorization the element growth
 * max|U| / max|Rs .* A| is measured; above `limit` (default 1e4) the matrix
 * is refactored in FP64 and solved with the FP64 factors (stats_json reports
 * "growth" and "refactored_fp64").  No counterpart in the reference, which
 * factors in the input precision only. */
int mfgpu_set_growth_limit(mfgpu_ctx* h, double limit);
/* Bound (seconds, > 0 and <= 3600; default 4) on every device-side wait of
 * this handle's kernels: the tensor-core GEMMs' mbarrier waits and the
 * persistent solve's grid barriers.  A wait that runs out ends its kernel
 * cleanly (issued tensor-core work drained, tensor memory freed) and the call
 * returns MFGPU_ERR_TIMEOUT; the handle stays usable (a factorization that
 * timed out leaves no factors: factor again).  The reference's counterpart is
 * a status, not a trap (src/multifrontal.jl:250-252). */
int mfgpu_set_wait_limit(mfgpu_ctx* h, double seconds);
/* Test hook for the bounded waits (no counterpart in the reference): with
 * on != 0 the handle's tensor-core GEMMs first wait on a barrier that nothing
 * arrives at, and CTA 0 of a persistent solve never arrives at its grid
 * barrier, so those waits run out after the wait limit and the calls return
 * MFGPU_ERR_TIMEOUT; on = 0 restores normal operation.  No fault is raised:
 * the waits end by the kernels' own clocks. */
int mfgpu_test_stall(mfgpu_ctx* h, int32_t on);

/* Pattern analysis for the numeric phase, from the reference's own symbolic
 * result: A's pattern (colptr, rowval, n x n), SymbolicMF.qf, .parent,
 * .sstart, and the update set of every supernode, i.e. colstruct[sstart[s+1]-1]
 * flattened into upd_ptr (nsuper+1) / upd_idx.  Replaces the pattern-only part
 * of multifrontal_lu (src/multifrontal.jl:152-196).
 * The arrays are checked before use (a partition of 1:n, monotone upd_ptr,
 * sorted update rows below their supernode that lie in the parent's front,
 * parent an elimination tree, qf a permutation, A's pattern inside the
 * fronts); an inconsistent set returns MFGPU_ERR_ARGUMENT.  Any failed
 * analysis leaves the handle unanalyzed (factor and solve then return
 * MFGPU_ERR_STATE) and ends a batch analysis. */
int mfgpu_analyze(mfgpu_ctx* h, int64_t n, const int64_t* colptr, const int64_t* rowval, const int64_t* qf,
                  const int64_t* parent, int64_t nsuper, const int64_t* sstart, const int64_t* upd_ptr,
                  const int64_t* upd_idx);
/* Same, from a libmfgpu symbolic object. */
int mfgpu_analyze_symbolic(mfgpu_ctx* h, int64_t n, const int64_t* colptr, const int64_t* rowval,
                           const mfgpu_symbolic* sym);

/* Numeric factorization of Diagonal(Rs) * A with A's values nzval (host
 * memory, pattern as analyzed); Rs may be NULL (no scaling, as
 * multifrontal_lu).  Replaces the hot loop of src/multifrontal.jl:198-357.
 * Returns 0, the singular column (check != 0), or an error. */
int mfgpu_factor(mfgpu_ctx* h, const double* nzval, const double* rs, int32_t check);
/* Same with device pointers (inputs already resident in HBM). */
int mfgpu_factor_device(mfgpu_ctx* h, const double* d_nzval, const double* d_rs, int32_t check);
/* splu's row scaling and factorization in one call: Rs = row_scaling(A,
 * scale) (MFGPU_SCALE_*) is computed on the device, bitwise equal to
 * mfgpu_row_scaling, then Diagonal(Rs) * A is factored (src/interface.jl:
 * 101-105).  mfgpu_get_row_scaling copies that Rs (n entries) to the host. */
int mfgpu_factor_scaled(mfgpu_ctx* h, const double* nzval, int32_t scale, int32_t check);
int mfgpu_get_row_scaling(mfgpu_ctx* h, double* rs);

/* out3 = {n, nnz(L), nnz(U)} of the last factorization. */
int mfgpu_factor_sizes(mfgpu_ctx* h, int64_t* out3);
/* Copy the factors to host CSC buffers (GPLUFactorization fields,
 * src/gplu.jl:45-51): L unit lower with its diagonal first, U upper with its
 * diagonal last, p, q, pinv; any pointer may be NULL. */
int mfgpu_get_factors(mfgpu_ctx* h, int64_t* lcolptr, int64_t* lrowval, double* lnzval, int64_t* ucolptr,
                      int64_t* urowval, double* unzval, int64_t* p, int64_t* q, int64_t* pinv);

/* solve(F, b; refine) for nrhs right-hand sides B (n x nrhs, column-major,
 * leading dimension ldb) into X (ldx), host memory.  The factors are those of
 * the last mfgpu_factor; Rs is the scaling given there; the refinement
 * residual r = b - A x uses the unscaled A values given there
 * (src/interface.jl:123-138, 170-177; src/solve.jl:10-39). */
int mfgpu_solve(mfgpu_ctx* h, int64_t nrhs, const double* b, int64_t ldb, double* x, int64_t ldx, int32_t refine);
/* mfgpu_factor then mfgpu_solve in one call -- solve(splu(A), b; refine) --
 * with the right-hand sides' host-to-device copy on a stream of its own,
 * overlapped with the factorization (fully when b is page-locked).  Returns
 * the factor status (a positive singular column when check is set: no solve
 * is done) or the solve's status; x is that of mfgpu_solve, bit for bit. */
int mfgpu_factor_solve(mfgpu_ctx* h, const double* nzval, const double* rs, int32_t check, int64_t nrhs,
                       const double* b, int64_t ldb, double* x, int64_t ldx, int32_t refine);
/* Same with device pointers. */
int mfgpu_solve_device(mfgpu_ctx* h, int64_t nrhs, const double* d_b, int64_t ldb, double* d_x, int64_t ldx,
                       int32_t refine);

/* Float32 matrices (the reference's generic Tv = Float32:
 * multifrontal_lu / splu of a SparseMatrixCSC{Float32}, test/
 * multifrontal_test.jl and bench/mf_verify.jl:33-37).  mfgpu_factor_f32
 * factors Diagonal(rs) * A from Float32 values and Float32 rs (NULL: no
 * scaling) with Float32 fronts -- assembly, pivoting and updates in FP32, the
 * large updates as BF16x3 tensor-core products unless
 * MFGPU_FLAG_NO_TENSOR_CORES -- and no FP64 refactor; the products
 * rs[i] * a_ij round exactly as Float32 multiplications.
 * mfgpu_get_factors_f32 returns the Float32 factor values;
 * mfgpu_solve_f32 is solve(F, b; refine) for Float32 b (n x nrhs,
 * column-major, leading dimension n) with the refinement residual in FP64,
 * rounded to Float32 x. */
int mfgpu_factor_f32(mfgpu_ctx* h, const float* nzval, const float* rs, int32_t check);
int mfgpu_get_factors_f32(mfgpu_ctx* h, int64_t* lcolptr, int64_t* lrowval, float* lnzval, int64_t* ucolptr,
                          int64_t* urowval, float* unzval, int64_t* p, int64_t* q, int64_t* pinv);
int mfgpu_solve_f32(mfgpu_ctx* h, int64_t nrhs, const float* b, float* x, int32_t refine);

/* ComplexF64 matrices (the reference's generic Tv = ComplexF64:
 * multifrontal_lu / splu of a SparseMatrixCSC{ComplexF64},
 * test/multifrontal_test.jl:63-75, bench/mf_verify.jl:27-31).  Values,
 * factors, b and x are interleaved (re, im) doubles -- Julia's ComplexF64
 * layout -- and Rs is real (mfgpu_row_scaling_c64).  The fronts are complex
 * FP64 on the GPU: every panel is factored with partial pivoting on the
 * first largest |re| + |im| of its pivot rows (LAPACK zgetrf's rule, as
 * Julia's lu!), the updates are complex products on the CUDA cores, and the
 * solves and refinement residuals are complex.  mfgpu_solve_c64 is
 * solve(F, b; refine) for nrhs right-hand sides (n x nrhs, column-major,
 * leading dimension n).  The real-valued entry points refuse complex
 * factors (MFGPU_ERR_STATE) and the complex ones real factors. */
int mfgpu_factor_c64(mfgpu_ctx* h, const double* nzval_ri, const double* rs, int32_t check);
int mfgpu_get_factors_c64(mfgpu_ctx* h, int64_t* lcolptr, int64_t* lrowval, double* lnzval_ri, int64_t* ucolptr,
                          int64_t* urowval, double* unzval_ri, int64_t* p, int64_t* q, int64_t* pinv);
int mfgpu_solve_c64(mfgpu_ctx* h, int64_t nrhs, const double* b_ri, double* x_ri, int32_t refine);

/* Normwise backward error max_k ||b_k - A x_k||_inf / (||A||_inf ||x_k||_inf + ||b_k||_inf)
 * of device arrays, computed in FP64 on the GPU with the analyzed pattern.
 * A NaN or Inf in x, b or A's values (or an overflow of the denominator)
 * gives NaN, so a broken solution never passes an accuracy check. */
int mfgpu_backward_error_device(mfgpu_ctx* h, int64_t nrhs, const double* d_b, int64_t ldb, const double* d_x,
                                int64_t ldx, double* out);

/* The same backward error, computed without allocating device memory, for
 * callers that cannot allocate when they check accuracy (services that
 * reserve all device memory at start-up, loops that must not take
 * cudaMalloc's device-wide synchronisation).  No counterpart in the
 * reference (PureUMFPACK.jl has no device code).  The residual is never
 * stored: per right-hand side the maxima go to one fixed device array inside
 * libmfgpu (98 KB, held on every GPU that loads the library until the
 * process exits), shared by all calls and all handles of a device.
 *   - nrhs must be 1..4096; larger counts return MFGPU_ERR_ARGUMENT.
 *   - The first call on a device looks up that array's device address; make
 *     that first call before any stream capture.  The address is kept for the
 *     life of the process, so a cudaDeviceReset after that first call is not
 *     supported (the array's memory is gone and later calls would use a
 *     stale address).
 *   - A 0 x 0 system gives 0; non-finite inputs give NaN, as
 *     mfgpu_backward_error_device.
 *   - The array keeps the last call's contents; each call clears it first.
 *     Calls whose GPU work overlaps (other streams, other handles on the same
 *     device, other host threads) race on it: serialise them.
 * Requires a factorization (the values of A given to mfgpu_factor*). */
int mfgpu_backward_error_noalloc(mfgpu_ctx* h, int64_t nrhs, const double* d_b, int64_t ldb, const double* d_x,
                                 int64_t ldx, double* out);

/* ------------------------------------------------------------------------
 * Batched systems: many independent square systems of uneven size through
 * one handle, one factor launch sequence and one solve launch sequence.  No
 * single counterpart in the reference: each system's result is that of
 * splu(A_i; method=:multifrontal, scale) (src/interface.jl:93-120) or, with
 * MFGPU_ORDER_COLAMD, of multifrontal_lu(Rs_i .* A_i; q=colamd_order(A_i))
 * (src/multifrontal.jl:152), and solve(F_i, b_i; refine)
 * (src/interface.jl:170-177) for every system.
 * ---------------------------------------------------------------------- */
enum { MFGPU_ORDER_AMD = 0, MFGPU_ORDER_COLAMD = 1 };

/* Analyze nsys systems; system i is n[i] x n[i] with pattern colptr[i] /
 * rowval[i].  Each system is ordered by itself, and the batch is analyzed as
 * one block-diagonal matrix whose elimination forest holds every system's
 * own tree: the fronts of all systems at one tree level share a launch.
 * Replaces any previous analysis of the handle. */
int mfgpu_batch_analyze(mfgpu_ctx* h, int64_t nsys, const int64_t* n, const int64_t* const* colptr,
                        const int64_t* const* rowval, int32_t ordering);
/* nsys, and the column (nsys+1) and value (nsys+1) offsets of every system
 * in the concatenated arrays that mfgpu_factor_device / mfgpu_solve_device
 * take for a batch (values of system i at nz_off[i].., its rows at
 * col_off[i].. of every right-hand-side column).  Any pointer may be NULL. */
int mfgpu_batch_layout(mfgpu_ctx* h, int64_t* nsys, int64_t* col_off, int64_t* nz_off);
/* Factor every system with its values nzval[i] and its own row scaling of
 * kind `scale`.  status[i] (nsys entries, may be NULL) receives 0 or the
 * system's first singular factor column (1-based, as SingularException).
 * Returns the number of singular systems when check != 0, else 0; or an error. */
int mfgpu_batch_factor(mfgpu_ctx* h, const double* const* nzval, int32_t scale, int32_t check, int64_t* status);
/* Solve every system for nrhs right-hand sides b[i] (n[i] x nrhs,
 * column-major) into x[i], with `refine` refinement steps. */
int mfgpu_batch_solve(mfgpu_ctx* h, int64_t nrhs, const double* const* b, double* const* x, int32_t refine);
/* out3 = {n[i], nnz(L_i), nnz(U_i)} of system i (0-based index). */
int mfgpu_batch_factor_sizes(mfgpu_ctx* h, int64_t sys, int64_t* out3);
/* System i's own factors, as mfgpu_get_factors gives them for one system. */
int mfgpu_batch_get_factors(mfgpu_ctx* h, int64_t sys, int64_t* lcolptr, int64_t* lrowval, double* lnzval,
                            int64_t* ucolptr, int64_t* urowval, double* unzval, int64_t* p, int64_t* q,
                            int64_t* pinv);

/* ------------------------------------------------------------------------
 * Gilbert-Peierls LU on the GPU: gplu(A; q, tol, check, sort_factors)
 * (src/gplu.jl:173-303), the factorization splu(A; method=:gplu, ordering,
 * tol, scale, check) runs by default (src/interface.jl:93-120), and the
 * solves over its factors: F \ b (src/solve.jl:66-77) or, with row scaling
 * and refinement, solve(F::PureLU, b; refine) (src/interface.jl:123-177).
 * Factors, pivots and solutions are bit for bit the reference's.  One warp
 * factors one system; a handle holds one or many independent systems.
 * ---------------------------------------------------------------------- */
typedef struct mfgpu_gplu mfgpu_gplu;
int mfgpu_gplu_create(int32_t device, mfgpu_gplu** out);
void mfgpu_gplu_destroy(mfgpu_gplu* g);
const char* mfgpu_gplu_last_error(const mfgpu_gplu* g);
/* Entries of L (and of U) each system gets on its first attempt; 0 (the
 * default) sizes them from the symbolic fill of (A + A^T)[q, q].  A system
 * that outgrows its room is factored again with three times as much. */
int mfgpu_gplu_set_initial_capacity(mfgpu_gplu* g, int64_t entries);
/* Factor nsys systems: system i is n[i] x n[i] (colptr[i], rowval[i],
 * nzval[i]; rows ascending in each column) in the column order q[i]
 * (1-based; q or q[i] NULL: natural), with its rows scaled by rs[i] (rs or
 * rs[i] NULL: unscaled), i.e. gplu(rs[i] .* A_i; q = q[i], tol, check,
 * sort_factors).  status[i] (may be NULL) receives 0 or, under check, the
 * first column without a nonzero pivot (SingularException(k)).  Returns the
 * number of singular systems when check != 0, else 0; MFGPU_ERR_ARGUMENT when
 * a system's pivot rows are not a permutation (check = 0 on a singular
 * matrix: the reference's invperm throws). */
int mfgpu_gplu_factor(mfgpu_gplu* g, int64_t nsys, const int64_t* n, const int64_t* const* colptr,
                      const int64_t* const* rowval, const double* const* nzval, const int64_t* const* q,
                      const double* const* rs, double tol, int32_t check, int32_t sort_factors, int64_t* status);
/* out3 = {n, nnz(L), nnz(U)} of system sys (0-based). */
int mfgpu_gplu_sizes(mfgpu_gplu* g, int64_t sys, int64_t* out3);
/* System sys's GPLUFactorization fields (gplu.jl:45-51), 1-based; any
 * pointer may be NULL. */
int mfgpu_gplu_get_factors(mfgpu_gplu* g, int64_t sys, int64_t* lcolptr, int64_t* lrowval, double* lnzval,
                           int64_t* ucolptr, int64_t* urowval, double* unzval, int64_t* p, int64_t* q,
                           int64_t* pinv);
/* x[i] = solve for b[i] (n[i] x nrhs, column-major) of every system, with
 * refine refinement steps against the unscaled A_i when the system was
 * factored with a row scaling (PureLU), or the raw F \ b otherwise. */
int mfgpu_gplu_solve(mfgpu_gplu* g, int64_t nrhs, const double* const* b, double* const* x, int32_t refine);
/* The same for the reference's other element types: Float32 values, Rs, b
 * and x (tol rounded to Float32, all arithmetic in Float32), and ComplexF64
 * values, b and x as interleaved (re, im) doubles with a real Float64 Rs
 * (Julia's complex product, division and abs).  A handle's factor-fetch and
 * solve calls must match the type it last factored (MFGPU_ERR_STATE). */
int mfgpu_gplu_factor_f32(mfgpu_gplu* g, int64_t nsys, const int64_t* n, const int64_t* const* colptr,
                          const int64_t* const* rowval, const float* const* nzval, const int64_t* const* q,
                          const float* const* rs, double tol, int32_t check, int32_t sort_factors, int64_t* status);
int mfgpu_gplu_get_factors_f32(mfgpu_gplu* g, int64_t sys, int64_t* lcolptr, int64_t* lrowval, float* lnzval,
                               int64_t* ucolptr, int64_t* urowval, float* unzval, int64_t* p, int64_t* q,
                               int64_t* pinv);
int mfgpu_gplu_solve_f32(mfgpu_gplu* g, int64_t nrhs, const float* const* b, float* const* x, int32_t refine);
int mfgpu_gplu_factor_c64(mfgpu_gplu* g, int64_t nsys, const int64_t* n, const int64_t* const* colptr,
                          const int64_t* const* rowval, const double* const* nzval_ri, const int64_t* const* q,
                          const double* const* rs, double tol, int32_t check, int32_t sort_factors,
                          int64_t* status);
int mfgpu_gplu_get_factors_c64(mfgpu_gplu* g, int64_t sys, int64_t* lcolptr, int64_t* lrowval, double* lnzval_ri,
                               int64_t* ucolptr, int64_t* urowval, double* unzval_ri, int64_t* p, int64_t* q,
                               int64_t* pinv);
int mfgpu_gplu_solve_c64(mfgpu_gplu* g, int64_t nrhs, const double* const* b_ri, double* const* x_ri,
                         int32_t refine);
/* {factor kernel ms (all attempts), finish kernel ms, last solve kernel ms,
 * factor launches, systems factored again} of the last calls. */
int mfgpu_gplu_timings(mfgpu_gplu* g, double* out5);

/* ------------------------------------------------------------------------
 * Autotuner interface (no counterpart in the reference).  The batched GEMM
 * launches of the mixed form -- factor updates, pivot-block inversion, and
 * the solve products for nrhs right-hand sides, in issue order -- can each run
 * as tcgen05 3xTF32 (128 x 128 tiles) or CUDA-core FP32 (64 x 64 tiles).
 * ---------------------------------------------------------------------- */
enum { MFGPU_TUNE_FEATURES = 11 };
/* Number of tunable launches, and with `feats` (cap floats) their features,
 * MFGPU_TUNE_FEATURES per launch: kind one-hot (factor, inversion, solve),
 * log10(1 + x) of flops, bytes, tasks, 64-tiles, 128-tiles, mean m, n, k. */
int mfgpu_tune_features(mfgpu_ctx* h, int64_t nrhs, int64_t* count, float* feats, int64_t cap);
/* Variant per tunable launch: 0 built-in rule, 1 tcgen05, 2 CUDA cores
 * (count 0 restores the rule everywhere).  Profiled launch records carry the
 * tunable index as their seventh field. */
int mfgpu_tune_set_choice(mfgpu_ctx* h, const int8_t* choice, int64_t count);

/* ------------------------------------------------------------------------
 * The autotuner's cost model: a small MLP (nin -> hidden -> hidden -> 1, tanh,
 * mean-squared error, Adam) trained and evaluated on the GPU by libmfgpu's
 * own kernels.  All arrays are host float32, samples row-major.
 * ---------------------------------------------------------------------- */
typedef struct mfgpu_mlp mfgpu_mlp;
int mfgpu_mlp_create(int32_t device, int32_t nin, int32_t hidden, uint64_t seed, mfgpu_mlp** out);
void mfgpu_mlp_destroy(mfgpu_mlp* m);
const char* mfgpu_mlp_last_error(const mfgpu_mlp* m);
int32_t mfgpu_mlp_nparams(const mfgpu_mlp* m);
/* Parameters: W1 (hidden x nin, row-major), b1, W2 (hidden x hidden), b2, w3 (hidden), b3. */
int mfgpu_mlp_get_params(mfgpu_mlp* m, float* out);
int mfgpu_mlp_set_params(mfgpu_mlp* m, const float* in);
int mfgpu_mlp_predict(mfgpu_mlp* m, const float* X, int64_t n, float* out);
/* Loss (1/n) sum (f(x_i) - y_i)^2 and its gradient with respect to the parameters. */
int mfgpu_mlp_loss_grad(mfgpu_mlp* m, const float* X, const float* Y, int64_t n, float* loss, float* grad);
/* iters full-batch Adam steps at learning rate lr; final_loss may be NULL. */
int mfgpu_mlp_train(mfgpu_mlp* m, const float* X, const float* Y, int64_t n, int32_t iters, float lr,
                    float* final_loss);

/* JSON object with the last call's phase times, sizes and counters, and the
 * per-kernel-class profile gathered since the last mfgpu_set_profiling. */
int mfgpu_stats_json(mfgpu_ctx* h, char* buf, int64_t cap);
/* Reset the launch counter and the kernel profile; on != 0 brackets every
 * kernel launch with CUDA events on the launching stream (device times per
 * kernel class, with their algorithmic flops and bytes). */
int mfgpu_set_profiling(mfgpu_ctx* h, int32_t on);
/* JSON array of the profiled launches since mfgpu_set_profiling:
 * [kernel class, tree level, tasks or tiles, device ms, flops, bytes] each.
 * Returns MFGPU_OK, or the buffer size needed when cap is too small. */
int mfgpu_launch_records(mfgpu_ctx* h, char* buf, int64_t cap);

#ifdef __cplusplus
}
#endif

#endif /* MFGPU_H */
