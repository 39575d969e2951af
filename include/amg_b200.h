/*
 * amg_b200.h -- C ABI of the B200 (sm_100a) multigrid solve phase.
 *
 * The reference (AMJax) exposes its solve phase as Python methods on
 * ``MultilevelSolver``; this ABI is what a binding of those methods calls.  Each entry
 * point names the reference interface it replaces (paths relative to the AMJax root).
 *
 * Conventions
 *  - Every pointer in a descriptor or argument is a DEVICE pointer unless stated.
 *  - The library never frees caller buffers.  Hierarchy arrays must stay alive and
 *    unchanged for the life of the hierarchy handle.
 *  - Vectors with k right-hand sides are stored row-major [n, k] (k contiguous).
 *  - All work is issued on the caller's stream (``stream`` is a cudaStream_t; NULL means
 *    the legacy default stream).
 *  - Functions return an ``amg_status``; no C++ exception crosses the ABI.
 *    ``amg_last_error()`` gives a human-readable message for the calling thread.
 *  - Matrix structure is checked on the device before use: by amg_hierarchy_create for
 *    the hierarchy, on every call for an A0 override, and the first time a stand-alone
 *    kernel (amg_jacobi, amg_spmv, amg_inverse_diagonal, amg_sampled_outer) sees a matrix
 *    (same pointers and sizes: a structure changed in place later is not re-checked).  The
 *    check waits for its verdict on the call's stream and is skipped while that stream is
 *    being captured into a CUDA graph.  A bad structure gives AMG_ERR_BAD_MATRIX.
 *  - Non-convergence is not an error (the reference returns x silently,
 *    amjax/multilevel.py:414-425); per-column iteration counts and final relative
 *    residuals are reported through ``iters_out`` / ``relres_out`` (host arrays of
 *    length k, may be NULL).
 */
#ifndef AMG_B200_H
#define AMG_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  AMG_OK = 0,
  AMG_ERR_INVALID_ARG = 1,   /* bad size, null pointer, unknown enum value */
  AMG_ERR_UNSUPPORTED = 2,   /* valid request this build does not implement */
  AMG_ERR_CUDA = 3,          /* a CUDA runtime call failed (message has the detail) */
  AMG_ERR_TIMEOUT = 4,       /* a bounded device wait gave up */
  AMG_ERR_BAD_MATRIX = 5     /* CSR validation failed (unsorted/out-of-range/short) */
} amg_status;

typedef enum { AMG_CYCLE_V = 0, AMG_CYCLE_W = 1, AMG_CYCLE_F = 2 } amg_cycle;

/* Precision of a solve.
 *  F64:   every vector, value and accumulation in FP64.
 *  F32:   FP32 hierarchy end to end (the reference's dtype=float32 mode); sums that
 *         decide convergence are accumulated in FP64.
 *  MIXED: the cycle runs on FP32 values and vectors with FP32 accumulation.  Standalone
 *         solve: the residual and the solution increment are FP32, updated after every
 *         cycle (r -= A e); the FP64 solution and the FP64 true residual b - A x are
 *         brought up to date under the same rule as PCG's, and a column stops only on
 *         the FP64 norm (the reference's rule).  PCG: CG with reliable updates:
 *         the CG vectors are FP32 (dot products and step lengths FP64); the FP64 solution
 *         and the FP64 true residual b - A x are brought up to date whenever the FP32
 *         residual has dropped by a fixed factor (AMG_RU_DELTA, default 3e-3) and before
 *         any column stops, so the stop rule is checked on the FP64 residual.  (With an
 *         A0 that has no FP32 values, and at k = 1, where its two extra launches per step
 *         outweigh the FP64 vector traffic it saves, PCG runs the MIXED_F64CG form.)
 *  MIXED_F64CG: the FP32 cycle inside FP64 outer loops: standalone, FP64 iterative
 *         refinement (residual b - A x, update and norm in FP64 every cycle); PCG, an FP64
 *         CG preconditioned by the FP32 cycle. */
typedef enum {
  AMG_PREC_F64 = 0,
  AMG_PREC_F32 = 1,
  AMG_PREC_MIXED = 2,
  AMG_PREC_MIXED_F64CG = 3
} amg_precision;

typedef enum { AMG_SMOOTH_NONE = 0, AMG_SMOOTH_JACOBI = 1 } amg_smoother_kind;

typedef enum {
  AMG_COARSE_PINV = 0,    /* x = A_inv b         (multilevel.py:509-516) */
  AMG_COARSE_LU = 1,      /* x = lu_solve(b)     (multilevel.py:519-526) */
  AMG_COARSE_QR = 2,      /* x = R^-1 Q^T b      (multilevel.py:529-536) */
  AMG_COARSE_JACOBI = 3   /* Jacobi sweeps from 0 (multilevel.py:501-507) */
} amg_coarse_kind;

/* One CSR matrix.  rowptr has n_rows+1 entries (int32), col nnz entries (int32,
 * sorted within a row is not required).  val64 / val32 hold the same values in FP64 /
 * FP32; a precision mode needs the one(s) it reads (F64: val64; F32: val32; MIXED: both
 * on level 0's A, val32 elsewhere). */
typedef struct {
  int32_t n_rows, n_cols;
  int64_t nnz;
  const int32_t* rowptr;
  const int32_t* col;
  const double* val64;
  const float* val32;
} amg_csr;

typedef struct {
  int32_t kind;       /* amg_smoother_kind */
  int32_t iterations; /* sweeps */
  double omega;       /* damping, already divided by rho when withrho was asked */
} amg_smoother;

/* One level.  P and R are ignored on the coarsest level. */
typedef struct {
  amg_csr A, P, R;
  const double* dinv64;
  const float* dinv32;
  amg_smoother pre, post;
} amg_level_desc;

/* Coarsest-level solver.  Dense matrices are row-major n x n in both precisions.
 *  PINV: m0 = A_inv.   LU: m0 = packed LU factors (unit-lower L below the diagonal),
 *  perm = row permutation (int32, perm[i] = row of b to place at i).
 *  QR: m0 = Q, m1 = R (upper).   JACOBI: uses the coarsest A/dinv, iterations, omega. */
typedef struct {
  int32_t kind;
  int32_t n;
  const double* m0_64; const float* m0_32;
  const double* m1_64; const float* m1_32;
  const int32_t* perm;
  int32_t iterations;
  double omega;
} amg_coarse_desc;

typedef struct amg_hierarchy amg_hierarchy;

/* Create a hierarchy handle over caller-owned device arrays (the arrays uploaded once
 * by MultilevelSolver.from_pyamg, amjax/multilevel.py:125-186 / _convert_hierarchy
 * :557-590).  Validates sizes, and the structure of every A, P and R on the device (row
 * pointers start at 0, never decrease and end at nnz; columns in [0, n_cols); columns
 * need not be sorted within a row): AMG_ERR_BAD_MATRIX otherwise.  Waits for the device
 * first.  The arrays are not copied. */
amg_status amg_hierarchy_create(const amg_level_desc* levels, int32_t n_levels,
                                const amg_coarse_desc* coarse, amg_hierarchy** out);
amg_status amg_hierarchy_destroy(amg_hierarchy* h);

/* Standalone solve: repeated cycles until ||b - A x|| < tol ||b|| per column or
 * maxiter cycles (MultilevelSolver.solve / _solve_loop, amjax/multilevel.py:341-425).
 * b, x: [n0, k] in FP64 for F64 and MIXED, FP32 for F32.  x is output only (x0 = 0;
 * the caller shifts b for a nonzero x0 as multilevel.py:384-394 does).
 * A0 (nullable) replaces the level-0 operator for smoothing and residuals
 * (the ``A=`` argument, multilevel.py:318,387-391); it must have A's shape.
 * Columns freeze independently once converged, as jax.vmap over the while-loop does. */
amg_status amg_solve(amg_hierarchy* h, int32_t precision, const void* b, void* x, int32_t k,
                     double tol, int32_t maxiter, int32_t cycle, int32_t cycles_per_level,
                     const amg_csr* A0, int32_t* iters_out, double* relres_out, void* stream);

/* One cycle from the zero vector: x = M b (MultilevelSolver.aspreconditioner,
 * amjax/multilevel.py:265-288).  b, x in the cycle's type: FP64 for F64, FP32 for F32
 * and MIXED. */
amg_status amg_precondition(amg_hierarchy* h, int32_t precision, const void* b, void* x,
                            int32_t k, int32_t cycle, int32_t cycles_per_level, void* stream);

/* Preconditioned CG with M = one cycle (jax.scipy.sparse.linalg.cg(A, b, M=ml.
 * aspreconditioner()) as the reference's benchmark calls it, benchmarks/benchmark.ipynb
 * cell 7; stopping rule <r,r> <= max(tol^2 <b,b>, atol^2)).  b, x FP64 ([n0,k]) for F64,
 * MIXED and MIXED_F64CG, FP32 for F32.  A0 as in amg_solve (used for the CG operator;
 * the preconditioner keeps the hierarchy's level 0). */
amg_status amg_pcg(amg_hierarchy* h, int32_t precision, const void* b, void* x, int32_t k,
                   double tol, double atol, int32_t maxiter, int32_t cycle,
                   int32_t cycles_per_level, const amg_csr* A0, int32_t* iters_out,
                   double* relres_out, void* stream);

/* amg_pcg with the right-hand sides and the solution in HOST memory (pinned, so that the
 * copies run asynchronously): what a caller whose data lives on the host -- a CPU-side
 * JAX array, a numpy user of MultilevelSolver.pcg -- would otherwise do as copy in, solve,
 * copy out one after another.  b_host, x_host: [n0, k] row-major FP64 (F64, MIXED,
 * MIXED_F64CG; F32 is AMG_ERR_UNSUPPORTED).  The k columns are solved in `blocks`
 * contiguous column blocks (columns are independent, each with its own stop rule), and
 * the copy of the next block in and of the previous block out overlap the current block's
 * solve (two copy streams, strided 2D copies).  Returns when x_host holds the solution.
 * The staging buffers (2 x 2 blocks of n0 x ceil(k / blocks) doubles) are kept with the
 * hierarchy; calls on one hierarchy are serialised. */
amg_status amg_pcg_host(amg_hierarchy* h, int32_t precision, const double* b_host, double* x_host, int32_t k,
                        int32_t blocks, double tol, double atol, int32_t maxiter, int32_t cycle,
                        int32_t cycles_per_level, int32_t* iters_out, double* relres_out, void* stream);

/* Adjoint of a solve in one call: the backward pass of the custom VJP of
 * MultilevelSolver.solve (_solve_bwd, amjax/multilevel.py:428-444).  Solves
 * A^T lam = gx (method 0: standalone cycles as amg_solve; 1: PCG as amg_pcg) on the
 * hierarchy `ht`, which must be built for A^T (the same handle when A and its hierarchy
 * are symmetric, R = P^T; explicit transposed levels otherwise, e.g. for AIR), with At
 * (nullable) overriding its level-0 operator as amg_solve's A0 does.  lam = dL/db [n, k].
 * When grad is not NULL, also writes dL/dA on A's pattern (`pattern`, n x n; values not
 * read): grad[e] = -sum_c lam[row(e), c] * x[col(e), c], with x [n, k] the forward
 * solution (FP64) -- the reference's dense -outer(lam, x) (:438-442) sampled where A has
 * entries, as amg_sampled_outer does.  gx, lam FP64 [n, k]; F32 is AMG_ERR_UNSUPPORTED.
 * The adjoint solve stores nothing from the forward iterations. */
amg_status amg_adjoint(amg_hierarchy* ht, int32_t precision, int32_t method, const void* gx, const double* x,
                       int32_t k, double tol, double atol, int32_t maxiter, int32_t cycle, int32_t cycles_per_level,
                       const amg_csr* At, const amg_csr* pattern, void* lam, double* grad, int32_t* iters_out,
                       double* relres_out, void* stream);

/* Several independent PCG solves in one graph launch: system i uses hierarchy hs[i], its own
 * k[i] right-hand sides b[i] -> x[i] (layouts as in amg_pcg), and the shared tol / atol /
 * maxiter / cycle.  The reference solves one system per call (jax.vmap batches right-hand
 * sides of one hierarchy only, README.md:60-66); this runs many hierarchies of different
 * sizes concurrently, each with its own convergence loop.  iters_out / relres_out (nullable)
 * get sum(k) entries, system after system.  Each hierarchy may appear once per call. */
amg_status amg_pcg_batch(amg_hierarchy* const* hs, int32_t nsys, int32_t precision,
                         const void* const* b, void* const* x, const int32_t* k, double tol,
                         double atol, int32_t maxiter, int32_t cycle, int32_t cycles_per_level,
                         int32_t* iters_out, double* relres_out, void* stream);

/* Damped Jacobi sweeps on one CSR matrix (amjax/relaxation/relaxation.py:64-98).
 * dtype 0 = FP64 (x, b, dinv, out double), 1 = FP32.  out may not alias x, b or dinv
 * (AMG_ERR_INVALID_ARG). */
amg_status amg_jacobi(const amg_csr* A, int32_t dtype, const void* x, const void* b,
                      const void* dinv, void* out, int32_t k, int32_t iterations,
                      double omega, void* stream);

/* amg_jacobi for callers that cannot allocate device memory when they call: a JAX/XLA
 * custom call (XLA has already reserved most of the GPU and owns scratch allocation), an
 * application on a fixed memory budget, a real-time caller that cannot afford an
 * allocator call.  No counterpart in the reference (AMJax only runs inside JAX).
 * Same arguments and results as amg_jacobi, but the iterate between sweeps lives in a
 * 16 MiB device array compiled into this library (held on every GPU that loads the
 * library until exit) instead of cudaMallocAsync; no cudaMalloc/cudaFree is called.
 * Limit: with iterations >= 2, n_rows * k * element size must be <= 16 MiB, else
 * AMG_ERR_INVALID_ARG.  The first call on a device looks up the array's device address
 * (once per device, on the current device): make that first call before any stream
 * capture.  All calls share the one array: calls whose work overlaps on the GPU (other
 * streams, other threads) race on it. */
amg_status amg_jacobi_noalloc(const amg_csr* A, int32_t dtype, const void* x, const void* b,
                              const void* dinv, void* out, int32_t k, int32_t iterations,
                              double omega, void* stream);

/* y = A x for [n_cols, k] x (the BCOO ``A @ x`` of the reference, multilevel.py:321,335). */
amg_status amg_spmv(const amg_csr* A, int32_t dtype, const void* x, void* y, int32_t k,
                    void* stream);

/* dinv = 1/diag(A), 0 where the diagonal is 0 (relaxation.py:36-61).  Duplicated
 * diagonal entries are summed. */
amg_status amg_inverse_diagonal(const amg_csr* A, int32_t dtype, void* dinv, void* stream);

/* Gradient of a loss through x = A^-1 b with respect to A's stored values: the
 * reference returns the dense -outer(lambda, x) (multilevel.py:438-442); this samples it
 * on the pattern: grad[e] = -sum_c lam[row(e), c] * x[col(e), c].  FP64. */
amg_status amg_sampled_outer(const amg_csr* A, const double* lam, const double* x, int32_t k,
                             double* grad, void* stream);

/* Diagnostic, no counterpart in the reference: times, on `stream`, each fine-level fused
 * kernel of one mixed-precision (reliable-update) PCG step for k right-hand sides -- the
 * <p, A p> pass with the direction update, the CG update, the post-smoothing sweep with
 * the fused <r, z>, the residual of the pre-smoothed iterate, restriction, prolongation
 * with correction, the FP64 true residual and the increment fold -- with the layouts the
 * solve uses (tuned first if not yet).  `reps` launches per kernel run back to back between
 * two CUDA events, alternating between two disjoint buffer sets so that each streams its
 * operands from DRAM.  Writes up to max_ops rows: a NUL-terminated name
 * (name_len bytes per row), the mean microseconds per launch and the kernel's algorithmic
 * bytes (every operand read or written once); *n_ops = rows written.  Uses the hierarchy's
 * mixed-precision scratch for k, so it must not overlap a solve on the same hierarchy. */
amg_status amg_time_pcg_ops(amg_hierarchy* h, int32_t k, int32_t reps, void* stream, int32_t max_ops,
                            char* names, int32_t name_len, double* us, double* bytes, int32_t* n_ops);

/* Number of kernels this library launched in the calling process (monotone counter;
 * one CUDA-graph launch counts every kernel node it contains). */
int64_t amg_kernel_launch_count(void);

/* Last error message of the calling thread ("" when none). */
const char* amg_last_error(void);

/* Library version string. */
const char* amg_version(void);

#ifdef __cplusplus
}
#endif
#endif /* AMG_B200_H */
