/*
 * bbt_oracle.c -- CPU checker (test infrastructure, not product).
 *
 * Exact LU of A - sigma B for a block-bordered pencil, in plain C, used
 * (a) to check the device preconditioner and (b) as the preconditioner of
 * the reference's CPU run in bench.py's CPU-baseline leg.  The reference
 * takes M^-1 from its caller (reference bbjd.py:208-219; in production an
 * external sparse LU, README.md:38-44); its test suite uses SuperLU
 * (tests/test_bbjd.py:62-73), which does not fit n = 10^6 in memory.
 *
 * Method: block Thomas elimination of the block-tridiagonal interior K
 * (D'_0 = D_0, D'_j = D_j - Lo_j D'_{j-1}^-1 Up_{j-1}), each D'_j factored by
 * LU with partial pivoting inside the block, and the t x t Schur complement
 * S = G - F1 K^-1 E of the border.  Inputs are row-major blocks [j][i][c],
 * E row-major nb x t, F row-major t x n (the host layout of
 * bbjd_b200.pencils.BBTPencil).
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef double complex zc;

typedef struct {
    int64_t b, nblk, t, nb, n;
    zc *LU;        /* nblk blocks: LU factors of D'_j (row-major) */
    int *piv;      /* nblk * b */
    zc *Lo, *Up;   /* copies of the couplings (row-major) */
    zc *Y;         /* nb x t row-major: K^-1 E */
    zc *S;         /* t x t LU of the Schur complement (row-major) */
    int *spiv;
    zc *F;         /* t x n row-major (copy) */
} bbt_lu;

/* LU with partial pivoting of an m x m row-major matrix; 0 or -1 (singular). */
static int lu_factor(int64_t m, zc *a, int *piv) {
    for (int64_t p = 0; p < m; ++p) {
        int64_t q = p;
        double best = cabs(a[p * m + p]);
        for (int64_t i = p + 1; i < m; ++i) {
            double v = cabs(a[i * m + p]);
            if (v > best) { best = v; q = i; }
        }
        piv[p] = (int)q;
        if (best == 0.0) return -1;
        if (q != p)
            for (int64_t c = 0; c < m; ++c) { zc tmp = a[p * m + c]; a[p * m + c] = a[q * m + c]; a[q * m + c] = tmp; }
        const zc inv = 1.0 / a[p * m + p];
        for (int64_t i = p + 1; i < m; ++i) {
            const zc f = a[i * m + p] * inv;
            a[i * m + p] = f;
            for (int64_t c = p + 1; c < m; ++c) a[i * m + c] -= f * a[p * m + c];
        }
    }
    return 0;
}

/* Solve (LU) x = v in place for one vector. */
static void lu_solve(int64_t m, const zc *a, const int *piv, zc *v) {
    for (int64_t p = 0; p < m; ++p) {
        const int q = piv[p];
        if (q != p) { zc tmp = v[p]; v[p] = v[q]; v[q] = tmp; }
    }
    for (int64_t i = 1; i < m; ++i) {
        zc s = v[i];
        for (int64_t c = 0; c < i; ++c) s -= a[i * m + c] * v[c];
        v[i] = s;
    }
    for (int64_t i = m - 1; i >= 0; --i) {
        zc s = v[i];
        for (int64_t c = i + 1; c < m; ++c) s -= a[i * m + c] * v[c];
        v[i] = s / a[i * m + i];
    }
}

/* y = M x (row-major m x m), y -= M x when sub. */
static void matvec(int64_t m, const zc *M, const zc *x, zc *y, int sub) {
    for (int64_t i = 0; i < m; ++i) {
        zc s = 0.0;
        for (int64_t c = 0; c < m; ++c) s += M[i * m + c] * x[c];
        y[i] = sub ? y[i] - s : s;
    }
}

/* Interior solve K x = r (vectors of length nb), x may alias r. */
static void interior_solve(const bbt_lu *h, const zc *r, zc *x, zc *work) {
    const int64_t b = h->b, N = h->nblk, bb = b * b;
    /* forward: z_j = D'_j^-1 (r_j - Lo_j z_{j-1}) */
    for (int64_t j = 0; j < N; ++j) {
        zc *zj = work + j * b;
        memcpy(zj, r + j * b, sizeof(zc) * b);
        if (j > 0) matvec(b, h->Lo + j * bb, work + (j - 1) * b, zj, 1);
        lu_solve(b, h->LU + j * bb, h->piv + j * b, zj);
    }
    /* backward: x_j = z_j - D'_j^-1 Up_j x_{j+1} */
    zc *tmp = (zc *)malloc(sizeof(zc) * b);
    memcpy(x + (N - 1) * b, work + (N - 1) * b, sizeof(zc) * b);
    for (int64_t j = N - 2; j >= 0; --j) {
        matvec(b, h->Up + j * bb, x + (j + 1) * b, tmp, 0);
        lu_solve(b, h->LU + j * bb, h->piv + j * b, tmp);
        for (int64_t i = 0; i < b; ++i) x[j * b + i] = work[j * b + i] - tmp[i];
    }
    free(tmp);
}

void bbt_lu_free(bbt_lu *h) {
    if (!h) return;
    free(h->LU); free(h->piv); free(h->Lo); free(h->Up); free(h->Y); free(h->S);
    free(h->spiv); free(h->F);
    free(h);
}

bbt_lu *bbt_lu_factor(int64_t b, int64_t nblk, int64_t t, const zc *Ad, const zc *Al,
                      const zc *Au, const zc *Bd, const zc *E, const zc *F, double sr, double si) {
    const zc sigma = sr + si * I;
    const int64_t bb = b * b, nb = b * nblk, n = nb + t;
    bbt_lu *h = (bbt_lu *)calloc(1, sizeof(bbt_lu));
    h->b = b; h->nblk = nblk; h->t = t; h->nb = nb; h->n = n;
    h->LU = (zc *)malloc(sizeof(zc) * bb * nblk);
    h->piv = (int *)malloc(sizeof(int) * b * nblk);
    h->Lo = (zc *)malloc(sizeof(zc) * bb * nblk);
    h->Up = (zc *)malloc(sizeof(zc) * bb * nblk);
    memcpy(h->Lo, Al, sizeof(zc) * bb * nblk);
    memcpy(h->Up, Au, sizeof(zc) * bb * nblk);
    zc *X = (zc *)malloc(sizeof(zc) * bb);
    for (int64_t j = 0; j < nblk; ++j) {
        zc *D = h->LU + j * bb;
        for (int64_t e = 0; e < bb; ++e) D[e] = Ad[j * bb + e] - sigma * Bd[j * bb + e];
        if (j > 0) {
            /* D -= Lo_j D'_{j-1}^-1 Up_{j-1}: columns of X = D'^-1 Up_{j-1} */
            for (int64_t c = 0; c < b; ++c) {
                zc col[128];
                for (int64_t i = 0; i < b; ++i) col[i] = Au[(j - 1) * bb + i * b + c];
                lu_solve(b, h->LU + (j - 1) * bb, h->piv + (j - 1) * b, col);
                for (int64_t i = 0; i < b; ++i) X[i * b + c] = col[i];
            }
            const zc *L = Al + j * bb;
            for (int64_t i = 0; i < b; ++i)
                for (int64_t c = 0; c < b; ++c) {
                    zc s = 0.0;
                    for (int64_t q = 0; q < b; ++q) s += L[i * b + q] * X[q * b + c];
                    D[i * b + c] -= s;
                }
        }
        if (lu_factor(b, D, h->piv + j * b)) { free(X); bbt_lu_free(h); return NULL; }
    }
    free(X);
    if (t > 0) {
        h->F = (zc *)malloc(sizeof(zc) * t * n);
        memcpy(h->F, F, sizeof(zc) * t * n);
        h->Y = (zc *)malloc(sizeof(zc) * nb * t);
        /* Y[:, c] = K^-1 E[:, c], columns in parallel */
        #pragma omp parallel
        {
            zc *col = (zc *)malloc(sizeof(zc) * nb);
            zc *work = (zc *)malloc(sizeof(zc) * nb);
            #pragma omp for schedule(dynamic, 1)
            for (int64_t c = 0; c < t; ++c) {
                for (int64_t i = 0; i < nb; ++i) col[i] = E[i * t + c];
                interior_solve(h, col, col, work);
                for (int64_t i = 0; i < nb; ++i) h->Y[i * t + c] = col[i];
            }
            free(col);
            free(work);
        }
        h->S = (zc *)malloc(sizeof(zc) * t * t);
        h->spiv = (int *)malloc(sizeof(int) * t);
        #pragma omp parallel for schedule(static)
        for (int64_t a = 0; a < t; ++a)
            for (int64_t c = 0; c < t; ++c) {
                zc s = 0.0;
                for (int64_t i = 0; i < nb; ++i) s += F[a * n + i] * h->Y[i * t + c];
                h->S[a * t + c] = F[a * n + nb + c] - s;
            }
        if (lu_factor(t, h->S, h->spiv)) { bbt_lu_free(h); return NULL; }
    }
    return h;
}

/* x = M^-1 r for M = [[K, E], [F1, G]] (vectors of length n). */
int bbt_lu_solve(const bbt_lu *h, const zc *r, zc *x) {
    const int64_t nb = h->nb, t = h->t, n = h->n;
    zc *work = (zc *)malloc(sizeof(zc) * nb);
    if (!work) return -1;
    interior_solve(h, r, x, work);
    if (t > 0) {
        zc x2[256];
        for (int64_t a = 0; a < t; ++a) {
            zc s = r[nb + a];
            for (int64_t i = 0; i < nb; ++i) s -= h->F[a * n + i] * x[i];
            x2[a] = s;
        }
        lu_solve(t, h->S, h->spiv, x2);
        for (int64_t a = 0; a < t; ++a) x[nb + a] = x2[a];
        for (int64_t i = 0; i < nb; ++i) {
            zc s = 0.0;
            for (int64_t a = 0; a < t; ++a) s += h->Y[i * t + a] * x2[a];
            x[i] -= s;
        }
    }
    free(work);
    return 0;
}
