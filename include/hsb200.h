/*
 * hsb200.h — C ABI of libhsb200.so, the B200 (sm_100a) implementation of
 * HybridSmoothers.jl's preconditioner/smoother apply path.
 *
 * Plain C types only.  Every function returns an hs_status; the message for
 * the last non-zero status of the calling thread is hs_last_error().
 * Handles are not thread-safe: a caller serialises the calls on one handle.
 * `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *
 * Each entry point names the reference interface it replaces, as
 * `file:line` inside HybridSmoothers.jl v0.1.4.
 */
#ifndef HSB200_H
#define HSB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------- */
/* Status codes.  The reference raises Julia exceptions instead:          */
/*   error("... must be greater than 0")  src/l1_gauss_seidel.jl:201,217-218,327 -> HS_ERR_ARG */
/*   SingularException(col)               src/l1_gauss_seidel.jl:430            -> HS_ERR_SINGULAR */
/* ---------------------------------------------------------------------- */
typedef enum {
    HS_OK = 0,
    HS_ERR_ARG = 1,           /* invalid argument */
    HS_ERR_OOM = 2,           /* device allocation failed */
    HS_ERR_CUDA = 3,          /* CUDA runtime/driver error */
    HS_ERR_SINGULAR = 4,      /* missing or zero diagonal (non-symmetric CSC path) */
    HS_ERR_NONFINITE = 5,     /* NaN/Inf met where a finite value is required */
    HS_ERR_NOT_CONVERGED = 6, /* Krylov solver hit its iteration cap */
    HS_ERR_TIMEOUT = 7,       /* a bounded device-side wait gave up */
    HS_ERR_UNSUPPORTED = 8,   /* valid but not provided (e.g. a CPU backend) */
    HS_ERR_BUDGET = 9         /* request does not fit the configured HBM budget */
} hs_status;

enum { HS_F64 = 0, HS_F32 = 1 };
enum { HS_CSC = 0, HS_CSR = 1 };
/* ForwardSweep, BackwardSweep, SymmetricSweep: src/l1_gauss_seidel.jl:18,25,83 */
enum { HS_SWEEP_FORWARD = 0, HS_SWEEP_BACKWARD = 1, HS_SWEEP_SYMMETRIC = 2 };
/* PackedBufferCache, MatrixViewCache: src/l1_gauss_seidel.jl:93,100 */
enum { HS_CACHE_PACKED = 0, HS_CACHE_VIEW = 1 };
/* Chebyshev spectral estimate: the reference's 50-step power iteration
 * (src/chebyshev.jl:40-54) or Lanczos bounds (this library's addition). */
enum { HS_EIG_POWER = 0, HS_EIG_LANCZOS = 1 };

/* A square sparse matrix in HOST memory, 0-based int32 indices, sorted
 * indices within each column (CSC) or row (CSR) — SparseMatrixCSC /
 * SparseMatrixCSR at the reference boundary (src/HybridSmoothers.jl:31-36). */
typedef struct {
    int32_t n;
    int64_t nnz;
    int32_t format;       /* HS_CSC or HS_CSR */
    int32_t dtype;        /* HS_F64 or HS_F32 (value type) */
    const int32_t* ptr;   /* n+1: colptr (CSC) or rowptr (CSR) */
    const int32_t* idx;   /* nnz: rowval (CSC) or colval (CSR) */
    const void* val;      /* nnz values */
} hs_sparse;

typedef struct hs_l1gs_s hs_l1gs;
typedef struct hs_cheb_s hs_cheb;
typedef struct hs_matrix_s hs_matrix;

/* BlockPartitioning (src/l1_gauss_seidel.jl:118-124) plus storage facts. */
typedef struct {
    int32_t n, partsize, nparts, nchunks, chunksize;
    int32_t sweep, cache, is_sym, format;
    int32_t matrix_dtype, smoother_dtype;
    int64_t packed_len;        /* S: length of SLbuffer/SUbuffer in the reference layout */
    int64_t device_bytes;      /* device memory held by the preconditioner */
    double eta;
    int32_t threads_per_part;  /* 1, or the lanes sharing a partition (see hs_l1gs_options) */
    int32_t order;             /* 1: every row summed in the reference's order; 2: reordered */
} hs_l1gs_info;

/* Build options beyond the reference's arguments. */
typedef struct {
    /* Threads that share one partition of a packed sweep.  0: chosen by the
     * library (8 from partsize 30 where padding the partition to a multiple
     * of 8 adds at most 15 % to its triangle, else 1 while the partitions keep
     * the GPU busy); 1: one thread per partition, which sums every row in the
     * reference's order (bit-identical results); 8 with a partsize from 8: the
     * blocked sweep (8 x 8 tiles, the partition padded to a multiple of 8);
     * 4, 16 or 32: lanes of a warp share a partition, column by column.  With
     * several lanes, forward sweeps stay bit-identical; backward and
     * symmetric sweeps agree with the reference's ascending order to
     * rounding.  Matrix-view caches always use 1. */
    int32_t threads_per_part;
    /* Summation order of each row's terms.  0: chosen by the library; 1: the
     * reference's ascending order everywhere (bit-identical to the reference;
     * requires threads_per_part 0 or 1, or 8 for a forward sweep); 2: the
     * library may reorder a row's sum (partial sums combined at the end of
     * the row) or multiply by 1/D_Dl1 instead of dividing, agreeing with the
     * reference to rounding: relative 1e-12 in FP64. */
    int32_t order;
} hs_l1gs_options;

/* ---------------------------------------------------------------------- */
/* L1 Gauss-Seidel                                                        */
/* ---------------------------------------------------------------------- */

/*
 * Replaces L1GSPrecBuilder(backend::KA.GPU; threads, blocks)
 * (src/l1_gauss_seidel.jl:251-262) called on (A, partsize; isSymA, η, sweep,
 * cache_strategy) (src/l1_gauss_seidel.jl:287-313) -> build_l1prec (:317-338).
 * A is host memory and is copied to the device.  threads/blocks are recorded as
 * the reference's BlockPartitioning; results do not depend on them.
 * smoother_dtype: HS_F64, or HS_F32 for an FP32 smoother built from an FP64
 * matrix (D_Dl1 computed in FP64, then rounded).
 */
int hs_l1gs_create(const hs_sparse* A, int32_t partsize, int32_t is_sym, double eta,
                   int32_t sweep, int32_t cache, int32_t smoother_dtype, int32_t threads,
                   int32_t blocks, void* stream, hs_l1gs** out);

/* hs_l1gs_create with build options (NULL = defaults): the same builder call
 * (src/l1_gauss_seidel.jl:287-313) plus the threads-per-partition choice. */
int hs_l1gs_create_opts(const hs_sparse* A, int32_t partsize, int32_t is_sym, double eta,
                        int32_t sweep, int32_t cache, int32_t smoother_dtype, int32_t threads,
                        int32_t blocks, const hs_l1gs_options* opts, void* stream, hs_l1gs** out);

/*
 * LinearSolve.ldiv!(y, P, x) on device vectors (src/l1_gauss_seidel.jl:367-384
 * without the adapt/copyto!): y = M^-1 x.  x and y are device pointers of
 * length n in io_dtype (HS_F64 or HS_F32); x == y (in place) is allowed, any
 * other overlap is not.  Asynchronous on `stream`.
 */
int hs_l1gs_apply(hs_l1gs* P, const void* x, void* y, int32_t io_dtype, void* stream);

/*
 * The generic LinearSolve.ldiv!(y, P, x) with HOST vectors
 * (src/l1_gauss_seidel.jl:367-384): y .= x, adapt to the device, sweep,
 * copyto! back.  Synchronous (returns when y_host holds the result).
 * Page-locked (mapped) x_host and y_host, each one allocation of at least n
 * elements, are read and written by the apply kernel itself over PCIe (zero
 * copy).  Other host memory goes through device copies owned by P: vectors of
 * 8 MB and more move in chunks of whole partition groups whose copy in, apply
 * and copy out overlap on streams owned by P (ordered after earlier work on
 * `stream`).  Buffers on the GPU's NUMA node move fastest.
 */
int hs_l1gs_apply_host(hs_l1gs* P, const void* x_host, void* y_host, int32_t io_dtype, void* stream);

int hs_l1gs_info_get(const hs_l1gs* P, hs_l1gs_info* info);

/* P.sweep.op.D_DL1 (src/l1_gauss_seidel.jl:509,516): n values in smoother dtype. */
int hs_l1gs_get_diag(const hs_l1gs* P, void* out_host);

/* P.sweep.op.L.SLbuffer (which=0) / .U.SUbuffer (which=1) in the reference's
 * packed layout (src/l1_gauss_seidel.jl:480-502), packed cache only.
 * capacity = number of elements available at out_host. */
int hs_l1gs_get_packed(const hs_l1gs* P, int32_t which, void* out_host, int64_t capacity);

/* DiagonalIndices (src/l1_gauss_seidel.jl:417-436), 0-based; non-symmetric CSC only. */
int hs_l1gs_get_diag_indices(const hs_l1gs* P, int32_t* out_host);

int hs_l1gs_destroy(hs_l1gs* P);

/* ---------------------------------------------------------------------- */
/* Sparse matrix on the device: mul!(y, A, x[, α, β]) as SparseMatricesCSR  */
/* (called at src/chebyshev.jl:47,165,179,287,305 and by Krylov drivers).  */
/* ---------------------------------------------------------------------- */
int hs_matrix_create(const hs_sparse* A, int32_t dtype, void* stream, hs_matrix** out);
/* y = alpha*A*x + beta*y, device vectors in the matrix dtype.  (alpha,beta) =
 * (1,0) is the three-argument mul!; (-1,1) the five-argument form of
 * src/chebyshev.jl:179.  Other pairs compute y[i] = beta*y[i] + sum alpha*(a*x). */
int hs_matrix_spmv(hs_matrix* A, const void* x, void* y, double alpha, double beta, void* stream);
int hs_matrix_destroy(hs_matrix* A);

/* ---------------------------------------------------------------------- */
/* Chebyshev smoothers                                                    */
/* ---------------------------------------------------------------------- */
typedef struct {
    int32_t n, kind, degree, eig, smoother_dtype;
    double rho;            /* spectral estimate used by the recurrence */
    double rho_power;      /* 50-step power iteration (reference) */
    double lanczos_min, lanczos_max; /* Lanczos bounds on spec(M^-1 A), if computed */
    double astar;          /* a* (1st kind), else 0 */
} hs_cheb_info;

/*
 * Replaces ChebyshevFourth/ChebyshevFirst(; degree, backend) + _build_smoother
 * (src/chebyshev.jl:115-156, :218-276).  kind = 4 or 1.  A is a host CSC
 * matrix (FP64); l1 row sums and the spectral estimate are FP64 on the device;
 * smoother_dtype selects FP64 or FP32 smoothing arithmetic.
 */
int hs_cheb_create(const hs_sparse* A, int32_t kind, int32_t degree, int32_t eig,
                   int32_t smoother_dtype, void* stream, hs_cheb** out);
/* smooth!(x, s, b) (src/chebyshev.jl:158-183, :278-322), device vectors in smoother dtype. */
int hs_cheb_smooth(hs_cheb* S, void* x, const void* b, void* stream);
/* z = M^-1 r := smooth!(0, s, r); r and z in io_dtype (FP64 or the smoother dtype). */
int hs_cheb_apply(hs_cheb* S, const void* r, void* z, int32_t io_dtype, void* stream);
int hs_cheb_info_get(const hs_cheb* S, hs_cheb_info* info);
/* Override the spectral estimate (parity runs at a fixed rho). */
int hs_cheb_set_rho(hs_cheb* S, double rho);
int hs_cheb_destroy(hs_cheb* S);

/*
 * Chebyshev smoothing of x in place, for callers that cannot call cudaMalloc
 * where they smooth (a runtime that owns the whole device pool, code under an
 * allocator lock, a serving loop that forbids allocation on its hot path).
 * No counterpart in the reference.  The caller passes every operand as a
 * device buffer: the CSR
 * matrix (rp, ci, v; FP64, sorted columns), l1inv = 1 ./ (l1 row sums), kind
 * (4 or 1), degree, rho and, for the 1st kind, astar (see hs_cheb_info), and
 * x (updated in place) and b, all FP64.  The function allocates nothing: its
 * work vectors live in a static device array of 4 * 262144 doubles (8 MiB,
 * held on every GPU that loads the library), so n may not exceed 262144
 * (HS_ERR_ARG otherwise).  The first call on a device looks up that array's
 * device address and keeps it; make it before any stream capture.  The kept
 * address belongs to the device's context: after cudaDeviceReset on that
 * device, do not call this function again in the same process.  All calls
 * share the array, so calls whose GPU work overlaps race.
 */
int hs_cheb_smooth_noalloc(int32_t n, int64_t nnz, const int32_t* rp, const int32_t* ci, const double* v,
                           const double* l1inv, int32_t kind, int32_t degree, double rho, double astar,
                           double* x, const double* b, void* stream);

/* ---------------------------------------------------------------------- */
/* AMG smoother (ext/HybridSmoothersAMGExt.jl:8-33): the L1GS             */
/* preconditioner used as a Richardson smoother inside a multigrid cycle.  */
/* ---------------------------------------------------------------------- */
typedef struct hs_richardson_s hs_richardson;
/* HybridSmoother{A, s, residual, correction} (:8-13): A and P stay owned by
 * the caller and must outlive the smoother; the residual and correction
 * vectors (matrix dtype) are allocated here.  P must have been built from the
 * same matrix (any sweep/cache; an FP32 smoother with an FP64 matrix works on
 * FP64 vectors). */
int hs_richardson_create(const hs_matrix* A, hs_l1gs* P, hs_richardson** out);
/* AMG.smooth!(x, s, b) (:26-33): `sweeps` times (the reference: 2)
 *   residual = A x;  residual .-= b;  correction = P \ residual;  x .-= correction
 * with x and b device vectors in the matrix dtype; x is updated in place. */
int hs_richardson_smooth(hs_richardson* S, void* x, const void* b, int32_t sweeps, void* stream);
int hs_richardson_destroy(hs_richardson* S);

/* ---------------------------------------------------------------------- */
/* Krylov drivers (stand-ins for Krylov.jl's CG/GMRES reached through      */
/* LinearSolve: test/test_preconditioners.jl:65,93).  FP64, device vectors. */
/* ---------------------------------------------------------------------- */
enum { HS_PREC_NONE = 0, HS_PREC_L1GS = 1, HS_PREC_CHEB = 2 };
typedef struct {
    int32_t iterations;
    int32_t converged;
    double relres;      /* true ||b - A x|| / ||b|| at exit */
    double ms;          /* device time of the solve */
    double rnorm;       /* the residual norm the stopping test used, at exit */
} hs_solve_info;

/* This library's PCG: stops when the recursive residual satisfies
 * ||r|| <= rtol ||b||. */
int hs_pcg_solve(hs_matrix* A, int32_t prec_type, void* prec, const double* b, double* x,
                 double rtol, int32_t maxit, void* stream, hs_solve_info* info);
/* This library's restarted GMRES(m), right preconditioned (CGS2): stops when
 * ||b - A x|| <= rtol ||b||. */
int hs_gmres_solve(hs_matrix* A, int32_t prec_type, void* prec, int32_t restart, const double* b,
                   double* x, double rtol, int32_t maxit, void* stream, hs_solve_info* info);

/* Krylov.jl's cg as LinearSolve.solve(LinearProblem(A, b), KrylovJL_CG(); Pl = P)
 * runs it (test/test_preconditioners.jl:93, README.md:29): M = P applied with
 * ldiv!, x0 = 0, stop when sqrt(r.z) <= atol + rtol sqrt(r0.z0) with z = M^-1 r
 * (the preconditioned residual norm).  itmax 0 = 2n.  info->iterations is
 * Krylov.jl's niter, info->rnorm the final sqrt(r.z). */
int hs_cg_krylovjl(hs_matrix* A, int32_t prec_type, void* prec, const double* b, double* x,
                   double atol, double rtol, int32_t itmax, void* stream, hs_solve_info* info);
/* Krylov.jl's gmres as KrylovJL_GMRES(gmres_restart = memory) with Pl = P
 * runs it (test/test_preconditioners.jl:65): left preconditioner, modified
 * Gram-Schmidt, symmetric Givens reflections, restart after `memory` inner
 * iterations; stop when the estimate of ||M^-1 (b - A x)|| is at most
 * atol + rtol ||M^-1 b||.  itmax 0 = 2n. */
int hs_gmres_krylovjl(hs_matrix* A, int32_t prec_type, void* prec, int32_t memory, const double* b,
                      double* x, double atol, double rtol, int32_t itmax, void* stream,
                      hs_solve_info* info);

/* ---------------------------------------------------------------------- */
/* Batched, served PCG (no counterpart in the reference: the serving and   */
/* batching patterns around ldiv!).  Each admitted system keeps its FP64    */
/* matrix, an FP32 L1GS SymmetricSweep packed preconditioner and its PCG    */
/* state in HBM; hs_batch_step advances all of them with one set of        */
/* launches.  Requests are refused with HS_ERR_BUDGET until a slot and      */
/* enough of the HBM budget are free.                                      */
/* ---------------------------------------------------------------------- */
typedef struct hs_batch_s hs_batch;
/* How a launch runs the iterations (bitwise identical iterates):           */
/*   HS_BATCH_SEGMENTED   (default) one CUDA graph of 7 + (partsize classes) */
/*                        launches per iteration, replayed; each phase runs  */
/*                        at its own occupancy                               */
/*   HS_BATCH_PERSISTENT  one persistent kernel (captured in a graph) runs   */
/*                        every iteration of the launch for all systems;     */
/*                        CTAs take work items from a device queue and a     */
/*                        system's phases wait on its own stage word         */
/*                        (bounded waits: HS_ERR_TIMEOUT)                    */
enum { HS_BATCH_SEGMENTED = 0, HS_BATCH_PERSISTENT = 1 };
typedef struct {
    int32_t max_slots;     /* systems resident at once */
    int64_t hbm_budget;    /* bytes the batch may hold on the device */
    int32_t partsize;      /* default partsize (8, 16 or 32) */
    double rtol;           /* ||r|| <= rtol ||b|| */
    int32_t maxit;         /* per-system iteration cap */
    int32_t schedule;      /* HS_BATCH_SEGMENTED or HS_BATCH_PERSISTENT */
} hs_batch_config;
typedef struct {
    int64_t tag;
    int32_t iterations, converged;
    double relres;         /* recursive residual ||r_k|| / ||b|| at exit */
} hs_batch_result;
typedef struct {
    int32_t active, finished;
    int64_t hbm_used, hbm_budget, iterations_run;
} hs_batch_info;

/* The engine reserves its HBM budget (at most 90 % of the free device memory)
 * in the device's stream-ordered pool at creation; slots are carved from it. */
int hs_batch_create(const hs_batch_config* cfg, void* stream, hs_batch** out);
/* Admit one system (host matrix, host b); x_host receives the solution when
 * it converges.  partsize 0 = the batch default.  A must be symmetric (the
 * engine runs CG): a CSC is read as its own transpose.  May be called while a
 * launch is in flight; the system joins at the next launch. */
int hs_batch_submit(hs_batch* B, const hs_sparse* A, const double* b_host, double* x_host, int64_t tag,
                    int32_t partsize, int32_t* slot);
/* Run `iters` batched PCG iterations over every active system; *finished =
 * systems that converged (or hit maxit) during this call. */
int hs_batch_step(hs_batch* B, int32_t iters, int32_t* finished);
/* hs_batch_step in two halves, so the host can admit the next requests while
 * the GPU iterates: launch enqueues the iterations and returns; wait blocks
 * until they are done and collects finished systems (as step does). */
int hs_batch_launch(hs_batch* B, int32_t iters);
int hs_batch_wait(hs_batch* B, int32_t* finished);
/* Collect finished systems and release their device memory. */
int hs_batch_poll(hs_batch* B, hs_batch_result* results, int32_t max_results, int32_t* count);
int hs_batch_info_get(const hs_batch* B, hs_batch_info* info);
int hs_batch_destroy(hs_batch* B);

/* ---------------------------------------------------------------------- */
/* Diagnostics                                                            */
/* ---------------------------------------------------------------------- */
const char* hs_last_error(void);
/* Column (1-based, like SingularException) of the last HS_ERR_SINGULAR. */
int32_t hs_last_singular_col(void);
/* Reads and clears the device-side error word that bounded waits set
 * (0 = none).  Synchronises `stream`. */
int hs_device_error(void* stream, int32_t* code);
/* Number of kernels this library has launched in this process. */
int64_t hs_kernel_launches(void);
const char* hs_version(void);

#ifdef __cplusplus
}
#endif
#endif /* HSB200_H */
