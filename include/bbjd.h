/*
 * bbjd.h -- C-ABI of the B200 JDQZ engine, drop-in for the reference's
 * public header (reference include/bbjd.h:61-282).
 *
 * The types, enums, structs and function signatures below keep the
 * reference's ABI byte for byte, so that a program compiled against the
 * reference header links against libbbjd_gpu.so unchanged:
 *
 *   bbjd_zomplex / bbjd_int        reference include/bbjd.h:64-65
 *   bbjd_status                    reference include/bbjd.h:70-78
 *   bbjd_target                    reference include/bbjd.h:83-91
 *   bbjd_matvec_fn/_precond_fn     reference include/bbjd.h:101-109
 *   bbjd_params                    reference include/bbjd.h:114-150
 *   bbjd_result                    reference include/bbjd.h:155-162
 *   bbjd_workspace                 reference include/bbjd.h:170-224
 *
 * What changes behind the ABI: bbjd_workspace_alloc places the n-row
 * arrays (V, W, AV, BV, swap_nm, Q_right, Q_left, gmres_V, tmp1..tmp4)
 * in device memory (HBM) with leading dimension n; the maxsub-square
 * arrays (MA, MB, SA, SB, ZA, ZB), the GMRES Hessenberg data and h_work
 * stay in host memory.  The reference documents the workspace as opaque
 * (reference include/bbjd.h:164-169), so no caller reads those pointers.
 * The callbacks keep host pointers: bbjd_solve copies each operand to a
 * pinned host buffer, calls the callback and copies the result back.
 * The device-operator path (no callbacks) is declared in bbjd_gpu.h.
 *
 * All dense matrices are column-major.  Complex arithmetic throughout.
 */
#ifndef BBJD_H
#define BBJD_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
#include <complex>
typedef std::complex<double> bbjd_zomplex;   /* layout-compatible with C's double complex */
extern "C" {
#else
#include <complex.h>
typedef double complex bbjd_zomplex;
#endif

typedef int64_t bbjd_int;

/* Return codes: reference include/bbjd.h:70-78, plus device-side codes. */
typedef enum {
    BBJD_SUCCESS           =  0,
    BBJD_MAX_ITER          =  1,  /* fewer than nev pairs converged          */
    BBJD_ERR_ALLOC         = -1,
    BBJD_ERR_INVALID       = -2,
    BBJD_ERR_CALLBACK      = -3,
    BBJD_ERR_LAPACK        = -4,
    BBJD_ERR_BREAKDOWN     = -5,
    BBJD_ERR_CUDA          = -6,  /* a CUDA call or kernel launch failed     */
    BBJD_ERR_DEVICE_TIMEOUT = -7, /* a bounded device-side wait ran out      */
} bbjd_status;

/* Eigenvalue selection: reference include/bbjd.h:83-91. */
typedef enum {
    BBJD_TARGET_NEAREST,
    BBJD_TARGET_LARGEST_MAG,
    BBJD_TARGET_SMALLEST_MAG,
    BBJD_TARGET_LARGEST_REAL,
    BBJD_TARGET_SMALLEST_REAL,
    BBJD_TARGET_LARGEST_IMAG,
    BBJD_TARGET_SMALLEST_IMAG,
} bbjd_target;

/* y = Op x on host vectors of length n; 0 on success.
 * Reference include/bbjd.h:101-109. */
typedef int (*bbjd_matvec_fn)(bbjd_int n, const bbjd_zomplex *x,
                              bbjd_zomplex *y, void *data);
typedef int (*bbjd_precond_fn)(bbjd_int n, const bbjd_zomplex *x,
                               bbjd_zomplex *y, void *data);

/* Solver parameters: field order and types of reference include/bbjd.h:114-150. */
typedef struct {
    bbjd_int        n;
    bbjd_int        nev;
    bbjd_zomplex    sigma;
    bbjd_target     target;
    bbjd_int        maxsub;          /* 0 => max(3 nev + 10, 40), capped at n */
    bbjd_int        minsub;          /* 0 => max(2 nev + 5, 20)               */
    double          tol;
    bbjd_int        maxiter;
    bbjd_int        inner_maxiter;   /* 0 => Sleijpen-van der Vorst step      */
    double          inner_tol;
    const bbjd_zomplex *v0;          /* host, length n; NULL => seeded random */
    bbjd_matvec_fn  matvec_A;
    bbjd_matvec_fn  matvec_B;
    bbjd_precond_fn precond;         /* NULL => identity                      */
    void           *op_data;
    int             verbose;         /* 0 silent, 1 locks, 2 per iteration    */
} bbjd_params;

/* Result (host memory, freed by bbjd_result_free): reference include/bbjd.h:155-162. */
typedef struct {
    bbjd_int        nconv;
    bbjd_zomplex   *eigenvalues;     /* nev entries, nconv filled, convergence order */
    bbjd_zomplex   *eigenvectors;    /* n x nev column-major, nconv columns filled   */
    double         *residuals;       /* ||theta_b A u - theta_a B u|| / (|a|+|b|)    */
    bbjd_int        iters;
    bbjd_status     status;
} bbjd_result;

/* Workspace: field order of reference include/bbjd.h:170-224.
 * [D] = device memory (HBM), [H] = host memory. */
typedef struct {
    bbjd_int    n, maxsub, nev;
    bbjd_zomplex *V;                 /* [D] n x maxsub search space               */
    bbjd_zomplex *W;                 /* [D] n x maxsub test space                 */
    bbjd_zomplex *AV;                /* [D] n x maxsub                            */
    bbjd_zomplex *BV;                /* [D] n x maxsub                            */
    bbjd_zomplex *MA;                /* [H] maxsub x maxsub  W^H A V              */
    bbjd_zomplex *MB;                /* [H] maxsub x maxsub  W^H B V              */
    bbjd_zomplex *SA, *SB;           /* [H] generalized Schur form                */
    bbjd_zomplex *ZA, *ZB;           /* [H] left / right Schur vectors            */
    bbjd_int     nlock;
    bbjd_int     kdim;
    bbjd_zomplex *gmres_V;           /* [D] n x (inner_maxiter + 1)               */
    bbjd_zomplex *gmres_H;           /* [H] (inner_maxiter + 1) x inner_maxiter   */
    bbjd_zomplex *gmres_cs;          /* [H]                                       */
    bbjd_zomplex *gmres_sn;          /* [H]                                       */
    bbjd_zomplex *gmres_g;           /* [H]                                       */
    bbjd_int      inner_maxiter;
    bbjd_zomplex *tmp1, *tmp2, *tmp3, *tmp4;   /* [D] length n each                */
    bbjd_zomplex *swap_nm;           /* [D] n x maxsub restart output             */
    bbjd_zomplex *Q_right;           /* [D] n x (nev + 1) deflation basis         */
    bbjd_zomplex *Q_left;            /* [D] n x (nev + 1) test images             */
    bbjd_zomplex *h_work;            /* [H] 2 maxsub + nev + 4                    */
} bbjd_workspace;

/* Defaults of reference jd_core.c:73-84. */
void bbjd_params_init(bbjd_params *p);

/* Reference jd_core.c:87-161 / 163-176.  Device arrays come from cudaMalloc on
 * the current device; NULL when any allocation fails. */
bbjd_workspace *bbjd_workspace_alloc(const bbjd_params *p);
void            bbjd_workspace_free(bbjd_workspace *ws);

/* Reference jd_core.c:743-1120: JDQZ with host callbacks for A, B and M^-1.
 * The subspace work (orthogonalisation, projected pencil, restart, Ritz
 * vectors) runs on the device; the projected QZ runs on the host. */
bbjd_status bbjd_solve(const bbjd_params *params, bbjd_workspace *ws,
                       bbjd_result *result);

/* Reference jd_core.c:178-183. */
void bbjd_result_free(bbjd_result *result);

/* Reference jd_core.c:244-266: CGS with a DGKS re-pass of v against the k
 * columns of Q (n x k, column-major).  Q and v are HOST pointers here, as
 * in the reference; v is updated in place; returns ||v|| afterwards. */
double bbjd_mgs_orthogonalize(bbjd_int n, bbjd_int k,
                              const bbjd_zomplex *Q, bbjd_zomplex *v);

/* Reference jd_core.c:568-727: left-preconditioned GMRES on the projected
 * correction equation.  As in the reference implementation (not its header
 * comment), q and p are the n x (ws->nlock + 1) projector bases Q_right and
 * Q_left.  All vector arguments are HOST pointers; the callbacks are the
 * host callbacks of bbjd_params.  Returns 0 on success. */
int bbjd_correction_gmres(
    bbjd_int n,
    const bbjd_zomplex *q,
    const bbjd_zomplex *p,
    bbjd_zomplex        theta_a,
    bbjd_zomplex        theta_b,
    const bbjd_zomplex *r,
    bbjd_zomplex       *z,
    bbjd_matvec_fn      matvec_A,
    bbjd_matvec_fn      matvec_B,
    bbjd_precond_fn     precond,
    void               *op_data,
    bbjd_int            maxiter,
    double              tol,
    bbjd_workspace     *ws);

#ifdef __cplusplus
}
#endif

#endif /* BBJD_H */
