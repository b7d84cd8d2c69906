/*
 * bbjd_gpu.h -- device-operator extension of the bbjd.h C-ABI.
 *
 * The reference applies A, B and the preconditioner through host callbacks
 * (reference include/bbjd.h:101-109, bbjd.py:181-219, _bbjd_c.c:43-123).
 * This header adds device-resident operators for block-bordered pencils
 * (BBT: block-tridiagonal A with t dense border columns and t dense tau
 * rows, block-diagonal B with zero tau rows) and a device preconditioner,
 * so that a whole JDQZ solve runs on one GPU with only k x k data crossing
 * to the host per iteration.  Nothing here has a counterpart in the
 * reference except where a line cites one.
 *
 * Layout of every host or device array passed here: column-major.
 *   blocks  Ad, Al, Au, Bd : nblk consecutive b x b column-major blocks;
 *                            block j of Al couples block row j to block
 *                            column j-1 (Al[0] unused), of Au to j+1
 *                            (Au[nblk-1] unused).
 *   E                       : nb x t column-major (ld = nb), A[0:nb, nb:n]
 *   F                       : t x n column-major (ld = t),   A[nb:n, 0:n]
 * with nb = nblk * b and n = nb + t.  Device vectors are contiguous,
 * 16-byte aligned complex128 (or complex64 where stated).
 */
#ifndef BBJD_GPU_H
#define BBJD_GPU_H

#include "bbjd.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bbjd_bbt_matrix bbjd_bbt_matrix;   /* opaque: A and B on one device */
typedef struct bbjd_precond    bbjd_precond;      /* opaque: device M^-1          */

enum { BBJD_FP64 = 0, BBJD_MIXED = 1 };
/* Projected eigenproblem of each outer iteration:
 *   BBJD_PROJ_QZ    : ZGGES + ZTGSEN on (W^H A V, W^H B V), as the reference
 *                     (reference jd_core.c:319-462);
 *   BBJD_PROJ_SCHUR : the same deflating subspaces from the Schur form of the
 *                     k x k matrix H = (nu0 MA + mu0 MB)^-1 MB (its eigenvalues
 *                     are 1/(nu0 lambda + mu0)), reordered only when a thick
 *                     restart needs the leading block; about 4x cheaper than
 *                     ZGGES at k = 200.  Needs nu0 != 0 (targets 'nearest'
 *                     and 'SM'); other targets and a singular
 *                     nu0 MA + mu0 MB fall back to QZ for that iteration;
 *   BBJD_PROJ_AUTO  : SCHUR where it applies, else QZ. */
enum { BBJD_PROJ_AUTO = 0, BBJD_PROJ_QZ = 1, BBJD_PROJ_SCHUR = 2 };
/* Which Ritz values count as already converged (locked):
 *   BBJD_LOCK_ROBUST    : |lambda - lambda_j| < max(100 tol, lock_rel max(1, |lambda_j|))
 *                         for a locked lambda_j, and a pair that converges again
 *                         (its vector lies in span(Q_right) to 1e-8 and its value
 *                         within 1e-4 relative of lambda_j) is not returned twice:
 *                         lambda_j's window widens to 10x the observed drift.
 *   BBJD_LOCK_REFERENCE : the reference's absolute |lambda - lambda_j| < 100 tol
 *                         (reference jd_core.c:369, 439), which returns an
 *                         ill-conditioned eigenvalue many times over. */
enum { BBJD_LOCK_ROBUST = 0, BBJD_LOCK_REFERENCE = 1 };

/* Layout of result->eigenvectors from a device solve. */
enum { BBJD_EVEC_COLUMN_MAJOR = 0, BBJD_EVEC_ROW_MAJOR = 1 };

/* How the harmonic Schur-form projected solve picks the target between
 * restarts (bbjd_device_ext.ritz_estimate).  FP64: the k projected
 * eigenvalues in FP64, the target's eigenvector by inverse iteration.
 * FP32: the k eigenvalues in complex64 (about half the host time), used only
 * to rank the candidates; the chosen one is refined in FP64 by Rayleigh-
 * quotient iteration on the FP64 projected matrix until its residual is
 * 16 k eps ||H||_1, re-checked against the locked values, and the FP64 path
 * runs whenever a refinement does not converge.  Returned eigenvalues,
 * residuals and the convergence test are FP64 either way.  AUTO = FP32. */
enum { BBJD_RITZ_AUTO = 0, BBJD_RITZ_FP64 = 1, BBJD_RITZ_FP32 = 2 };

/* Host/device overlap of the FP32-estimate target rule (bbjd_device_ext.
 * host_overlap).  Between restarts the target is, by rule, the eigenpair that
 * Rayleigh-quotient iteration reaches from the previous target when the k
 * complex64 estimates rank it first, else the estimates' winner refined in
 * FP64.  AUTO: a lone solve computes that guess first, starts the device
 * iteration on it, and checks it against the estimates computed meanwhile
 * on a second host thread; a rejected guess repeats the iteration's device
 * work with the right target.  OFF: the same rule, serially.  Both give the
 * same results bit for bit.  The solves of bbjd_solve_batch run serially. */
enum { BBJD_OVERLAP_AUTO = 0, BBJD_OVERLAP_OFF = 1 };

enum { BBJD_PC_NONE = 0, BBJD_PC_BBT_LU = 1, BBJD_PC_BLOCK_JACOBI = 2 };

/* Copy a BBT pencil to the current device.  from_host = 1: pointers are host
 * memory; 0: device memory (copied).  b must be 8, 16 or 32. */
bbjd_status bbjd_bbt_create(bbjd_int b, bbjd_int nblk, bbjd_int t,
                            const bbjd_zomplex *Ad, const bbjd_zomplex *Al,
                            const bbjd_zomplex *Au, const bbjd_zomplex *E,
                            const bbjd_zomplex *F, const bbjd_zomplex *Bd,
                            int from_host, bbjd_bbt_matrix **out);
void        bbjd_bbt_free(bbjd_bbt_matrix *m);
bbjd_int    bbjd_bbt_n(const bbjd_bbt_matrix *m);
/* Algorithmic bytes one fused A,B product reads and writes (HBM roofline). */
double      bbjd_bbt_matvec_bytes(const bbjd_bbt_matrix *m);

/* yA = A x and yB = B x on device vectors, one fused pass (replaces the
 * matvec_A / matvec_B callbacks, reference jd_core.c:884-885). */
bbjd_status bbjd_bbt_matvec(const bbjd_bbt_matrix *m, const bbjd_zomplex *x,
                            bbjd_zomplex *yA, bbjd_zomplex *yB, void *stream);

/* Device preconditioner for A - sigma B.
 *   kind BBJD_PC_BBT_LU       : exact block-bordered LU (block cyclic
 *                               reduction of the block-tridiagonal interior,
 *                               t x t Schur complement for the border);
 *   kind BBJD_PC_BLOCK_JACOBI : inverses of the diagonal blocks and of the
 *                               t x t tau corner.
 * precision BBJD_MIXED stores the factors in complex64. */
bbjd_status bbjd_precond_create(const bbjd_bbt_matrix *m, bbjd_zomplex sigma,
                                int kind, int precision, bbjd_precond **out);
void        bbjd_precond_free(bbjd_precond *pc);
double      bbjd_precond_solve_bytes(const bbjd_precond *pc, int nrhs);
double      bbjd_precond_factor_seconds(const bbjd_precond *pc);
/* x[:, j] = M^-1 r[:, j] for nrhs <= 2 device vectors stored with stride n. */
bbjd_status bbjd_precond_solve(const bbjd_precond *pc, int nrhs,
                               const bbjd_zomplex *r, bbjd_zomplex *x, void *stream);

/* Options and instrumentation of a device solve. */
typedef struct {
    int     precision;          /* BBJD_FP64 (default) or BBJD_MIXED            */
    int     record_timing;      /* 1: fill the timing fields (adds syncs)       */
    int     projected;          /* BBJD_PROJ_AUTO (default), _QZ or _SCHUR      */
    int     lock_rule;          /* BBJD_LOCK_ROBUST (default) or _REFERENCE     */
    double  lock_rel;           /* relative lock window; 0 = 1e-6               */
    void   *stream;             /* cudaStream_t, NULL = a private stream        */
    int     evec_layout;        /* BBJD_EVEC_COLUMN_MAJOR (default): n x nev
                                   column-major, as bbjd_solve.
                                   BBJD_EVEC_ROW_MAJOR: result->eigenvectors
                                   holds the (n, nconv) row-major array a
                                   Python caller returns, transposed on the
                                   device at the end of the solve (saves the
                                   host an O(n nconv) strided copy)          */
    int     ritz_estimate;      /* BBJD_RITZ_AUTO (default), _FP64 or _FP32     */
    int     host_overlap;       /* BBJD_OVERLAP_AUTO (default) or _OFF          */
    int64_t *conv_iters;        /* optional (NULL): nev entries, filled with the
                                   outer iteration at which each returned pair
                                   converged (0-based, as the reference's
                                   verbose log numbers them)                 */
    /* out */
    double  seconds_total;      /* wall time of the solve                       */
    double  seconds_qz;         /* host projected QZ + reorder                  */
    double  seconds_device;     /* device time (CUDA events, summed)            */
    double  seconds_restart;    /* device time spent in thick restarts          */
    double  bytes_device;       /* algorithmic HBM bytes of the device work     */
    int64_t kernel_launches;    /* kernels this library launched                */
    int64_t dgks_passes;        /* second CGS passes taken                      */
    int64_t restarts;
    int64_t duplicates;         /* re-converged locked pairs not returned again */
    int64_t ritz_refinements;   /* FP64 LU factorisations of the FP32 target
                                   refinement (BBJD_RITZ_FP32)                */
    int64_t ritz_fallbacks;     /* FP32 estimates replaced by the FP64 path    */
    double  seconds_qz_exposed; /* of seconds_qz, the part the thread driving
                                   the device spent (not hidden behind it)     */
    int64_t guess_hits;         /* iterations whose guessed target held         */
    int64_t guess_misses;       /* guesses rejected (device work repeated when
                                   host_overlap is AUTO)                      */
    double  kernel_ms[8];       /* per kernel class: spmv, orth, pencil, ritz,
                                   precond, restart, small, gmres (if timed)    */
    double  kernel_bytes[8];
    int64_t kernel_calls[8];
} bbjd_device_ext;

void bbjd_device_ext_init(bbjd_device_ext *ext);

/* JDQZ with device operators: params->matvec_A/B/precond/op_data are
 * ignored; A and B are `m`, the preconditioner is `pc` (NULL = identity).
 * ws comes from bbjd_workspace_alloc with the same params.  Same algorithm,
 * constants and result contract as bbjd_solve. */
bbjd_status bbjd_solve_device(const bbjd_params *params, bbjd_device_ext *ext,
                              const bbjd_bbt_matrix *m, const bbjd_precond *pc,
                              bbjd_workspace *ws, bbjd_result *result);

/* Independent device solves of a sigma-sweep on one GPU (the reference's
 * deployment runs one sigma per MPI rank, reference README.md:59-83): solve i
 * uses params[i], mats[i], pcs[i] (may be NULL), wss[i], results[i] and, when
 * exts != NULL, exts[i].  Up to `threads` solves run at once, each on its own
 * host thread and CUDA stream, so the host-side projected QZ of one solve
 * overlaps the device work of the others; solves start largest first (by
 * n x maxiter x maxsub).  Every params[i].v0 must be set
 * (the seeded start vector uses the C library's global rand()), and no two
 * solves may share a preconditioner or a workspace (their scratch is
 * written during the solve); solves may share a matrix (a sweep over sigma
 * of one pencil: each solve reads it and has its own product scratch).  Returns the first failing status, else BBJD_SUCCESS (or
 * BBJD_MAX_ITER if any solve stopped at maxiter). */
bbjd_status bbjd_solve_batch(int count, const bbjd_params *params, bbjd_device_ext *exts,
                             const bbjd_bbt_matrix *const *mats, const bbjd_precond *const *pcs,
                             bbjd_workspace *const *wss, bbjd_result *results, int threads);

/* ---- device kernels exposed for parity tests (device pointers) ---------- */

/* CGS + DGKS of v (length n) against the k columns of Q (ld = ldq); returns
 * ||v|| afterwards through *norm_out (host).  reference jd_core.c:207-241 */
bbjd_status bbjd_dev_orthogonalize(bbjd_int n, bbjd_int k, const bbjd_zomplex *Q,
                                   bbjd_int ldq, bbjd_zomplex *v, double *norm_out,
                                   int *second_pass_out, void *stream);

/* The same orthogonalisation as bbjd_dev_orthogonalize, allocating nothing
 * (no counterpart in the reference).  For callers that cannot call
 * cudaMalloc there: a framework that owns all device memory and forbids
 * allocation after start-up, or a pipeline that must not stall the device
 * (cudaMalloc and cudaFree synchronise it).  Its reduction scratch is one
 * static device array of about 2.7 MB in the library, held until exit by
 * every GPU on which the library's module has been loaded.  Limits: n <= BBJD_STATIC_ORTH_MAX_N,
 * k <= BBJD_STATIC_ORTH_MAX_K; larger sizes return BBJD_ERR_INVALID with a
 * message on stderr.  The first call on each device looks the array up
 * (cudaGetSymbolAddress); under CUDA's lazy module loading (the default)
 * that first call also loads the module holding the array, which allocates
 * it and may synchronise the device, so make one warm-up call per device
 * (k = 0 will do) at start-up, before any stream capture.  Calls share the
 * array: two calls that overlap on the GPU (other streams or host threads
 * on the same device) race, so serialise them.  Q and v are device pointers; *norm_out and
 * *second_pass_out are host. */
#define BBJD_STATIC_ORTH_MAX_N 8388608
#define BBJD_STATIC_ORTH_MAX_K 256
bbjd_status bbjd_dev_orthogonalize_static(bbjd_int n, bbjd_int k, const bbjd_zomplex *Q,
                                          bbjd_int ldq, bbjd_zomplex *v, double *norm_out,
                                          int *second_pass_out, void *stream);

/* out = X[:, 0:k] * Z[0:k, 0:keep]  (X, out ld = ldx; Z host k x keep col-major,
 * ldz).  Thick-restart compression, reference jd_core.c:989-999. */
bbjd_status bbjd_dev_restart_gemm(bbjd_int n, bbjd_int k, bbjd_int keep,
                                  const bbjd_zomplex *X, bbjd_int ldx,
                                  const bbjd_zomplex *Z_host, bbjd_int ldz,
                                  bbjd_zomplex *out, void *stream);

/* Failure-detection check of the restart GEMM's bounded waits (no
 * counterpart in the reference): the same TMA-staged kernel, with every
 * stage's mbarrier expecting 16 bytes more than its loads bring, so no
 * stage completes; each wait gives up after ~1 ms and the call returns
 * BBJD_ERR_DEVICE_TIMEOUT with out unchanged and the context usable.
 * keep <= 80. */
bbjd_status bbjd_dev_restart_gemm_stalled(bbjd_int n, bbjd_int k, bbjd_int keep,
                                          const bbjd_zomplex *X, bbjd_int ldx,
                                          const bbjd_zomplex *Z_host, bbjd_int ldz,
                                          bbjd_zomplex *out, void *stream);

/* C (host, keep x keep, ldc) = X^H Y for device X, Y (n x keep, ld = ldx).
 * reference jd_core.c:1020-1025 */
bbjd_status bbjd_dev_gram(bbjd_int n, bbjd_int keep, const bbjd_zomplex *X,
                          const bbjd_zomplex *Y, bbjd_int ldx,
                          bbjd_zomplex *C_host, bbjd_int ldc, void *stream);

/* Library version / build string. */
const char *bbjd_gpu_version(void);

#ifdef __cplusplus
}
#endif

#endif /* BBJD_GPU_H */
