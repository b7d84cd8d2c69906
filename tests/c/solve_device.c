/* A C caller of libbbjd_gpu.so, the way a C program written against the
 * reference's header uses the library (no Python, no PyTorch in the
 * process): a block-bordered pencil is built on the host, solved once with
 * the device operators (bbjd_solve_device) and once with the reference's
 * host-callback interface (bbjd_solve: host products and a dense host LU as
 * the preconditioner), and every returned pair is checked
 * against the pencil with a host product.  Exit status 0 = all checks pass.
 *
 * Pencil: b = 8, nblk = 24, t = 2 (n = 194); diagonal blocks
 * noise + (j/4 + i j/2) I, off-diagonal blocks noise, border and tau entries
 * noise / sqrt(n), B = blockdiag(I + 0.1 noise) with zero tau rows; noise
 * from a fixed 64-bit LCG.  All blocks column-major. */
#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "bbjd.h"
#include "bbjd_gpu.h"

enum { B = 8, NBLK = 24, T = 2, NB = B * NBLK, N = NB + T, K = 3 };
static double complex Ad[NBLK * B * B], Al[NBLK * B * B], Au[NBLK * B * B], Bd[NBLK * B * B];
static double complex E[NB * T], F[T * N];   /* E col-major nb x t; F stored F^T: [col][tau] */

static unsigned long long lcg = 88172645463325252ULL;
static double urand(void) {
    lcg = lcg * 6364136223846793005ULL + 1442695040888963407ULL;
    return (double)(lcg >> 11) / 9007199254740992.0 - 0.5;
}
static double complex crand(void) { return urand() + I * urand(); }

static void build(void) {
    for (int j = 0; j < NBLK; ++j)
        for (int c = 0; c < B; ++c)
            for (int i = 0; i < B; ++i) {
                const int e = j * B * B + c * B + i;
                Ad[e] = crand() / sqrt((double)B) + (i == c ? (0.25 * j + 0.5 * I * j) : 0.0);
                Al[e] = j > 0 ? crand() / sqrt((double)B) : 0.0;
                Au[e] = j + 1 < NBLK ? crand() / sqrt((double)B) : 0.0;
                Bd[e] = (i == c ? 1.0 : 0.0) + 0.1 * crand() / sqrt((double)B);
            }
    for (int e = 0; e < NB * T; ++e) E[e] = crand() / sqrt((double)N);
    for (int e = 0; e < T * N; ++e) F[e] = crand() / sqrt((double)N);
}

/* yA = A x, yB = B x on the host */
static void host_product(const double complex *x, double complex *yA, double complex *yB) {
    for (int r = 0; r < N; ++r) yA[r] = yB[r] = 0.0;
    for (int j = 0; j < NBLK; ++j)
        for (int c = 0; c < B; ++c)
            for (int i = 0; i < B; ++i) {
                const int e = j * B * B + c * B + i, row = j * B + i;
                yA[row] += Ad[e] * x[j * B + c];
                if (j > 0) yA[row] += Al[e] * x[(j - 1) * B + c];
                if (j + 1 < NBLK) yA[row] += Au[e] * x[(j + 1) * B + c];
                yB[row] += Bd[e] * x[j * B + c];
            }
    for (int tau = 0; tau < T; ++tau) {
        for (int row = 0; row < NB; ++row) yA[row] += E[tau * NB + row] * x[NB + tau];
        double complex s = 0.0;
        for (int col = 0; col < N; ++col) s += F[col * T + tau] * x[col];
        yA[NB + tau] = s;
    }
}

static int mvA(bbjd_int n, const bbjd_zomplex *x, bbjd_zomplex *y, void *d) {
    (void)n; (void)d;
    static double complex tmp[N];
    host_product(x, y, tmp);
    return 0;
}
static int mvB(bbjd_int n, const bbjd_zomplex *x, bbjd_zomplex *y, void *d) {
    (void)n; (void)d;
    static double complex tmp[N];
    host_product(x, tmp, y);
    return 0;
}

/* dense LU (partial pivoting) of M = A - sigma B for the callback
 * preconditioner, as a host sparse LU would be in the reference's usage */
static double complex LU[N * N];
static int piv[N];
static void factor(double complex sigma) {
    static double complex x[N], yA[N], yB[N];
    for (int c = 0; c < N; ++c) {                  /* column c of M */
        for (int i = 0; i < N; ++i) x[i] = (i == c);
        host_product(x, yA, yB);
        for (int i = 0; i < N; ++i) LU[i + c * N] = yA[i] - sigma * yB[i];
    }
    for (int k = 0; k < N; ++k) {
        int p = k;
        for (int i = k + 1; i < N; ++i)
            if (cabs(LU[i + k * N]) > cabs(LU[p + k * N])) p = i;
        piv[k] = p;
        if (p != k)
            for (int c = 0; c < N; ++c) {
                const double complex tmp = LU[k + c * N];
                LU[k + c * N] = LU[p + c * N];
                LU[p + c * N] = tmp;
            }
        for (int i = k + 1; i < N; ++i) {
            LU[i + k * N] /= LU[k + k * N];
            for (int c = k + 1; c < N; ++c) LU[i + c * N] -= LU[i + k * N] * LU[k + c * N];
        }
    }
}
static int lu_solve(bbjd_int n, const bbjd_zomplex *r, bbjd_zomplex *x, void *d) {
    (void)n; (void)d;
    for (int i = 0; i < N; ++i) x[i] = r[i];
    for (int k = 0; k < N; ++k) {
        if (piv[k] != k) {
            const double complex tmp = x[k];
            x[k] = x[piv[k]];
            x[piv[k]] = tmp;
        }
        for (int i = k + 1; i < N; ++i) x[i] -= LU[i + k * N] * x[k];
    }
    for (int i = N - 1; i >= 0; --i) {
        for (int c = i + 1; c < N; ++c) x[i] -= LU[i + c * N] * x[c];
        x[i] /= LU[i + i * N];
    }
    return 0;
}

/* largest ||A x - lam B x|| / ||x|| over the returned pairs */
static double worst_residual(const bbjd_result *r) {
    static double complex yA[N], yB[N];
    double worst = 0.0;
    for (bbjd_int p = 0; p < r->nconv; ++p) {
        const double complex *x = r->eigenvectors + (size_t)p * N;
        host_product(x, yA, yB);
        double num = 0.0, den = 0.0;
        for (int i = 0; i < N; ++i) {
            const double complex d = yA[i] - r->eigenvalues[p] * yB[i];
            num += creal(d * conj(d));
            den += creal(x[i] * conj(x[i]));
        }
        const double res = sqrt(num / den);
        if (res > worst) worst = res;
    }
    return worst;
}

int main(void) {
    build();
    static double complex v0[N];
    for (int i = 0; i < N; ++i) v0[i] = 1.0 + 0.01 * i;
    const double complex sigma = 3.0 + 5.0 * I;

    bbjd_bbt_matrix *m = NULL;
    bbjd_precond *pc = NULL;
    if (bbjd_bbt_create(B, NBLK, T, Ad, Al, Au, E, F, Bd, 1, &m) != BBJD_SUCCESS) return 10;
    if (bbjd_bbt_n(m) != N) return 11;
    if (bbjd_precond_create(m, sigma, BBJD_PC_BBT_LU, BBJD_FP64, &pc) != BBJD_SUCCESS) return 12;

    bbjd_params p;
    bbjd_params_init(&p);
    p.n = N;
    p.nev = K;
    p.sigma = sigma;
    p.tol = 1e-10;
    p.maxiter = 600;
    p.maxsub = 40;
    p.minsub = 16;
    p.v0 = v0;

    /* device operators */
    bbjd_workspace *ws = bbjd_workspace_alloc(&p);
    if (!ws) return 13;
    bbjd_device_ext ext;
    bbjd_device_ext_init(&ext);
    bbjd_result rd;
    memset(&rd, 0, sizeof rd);
    const bbjd_status sd = bbjd_solve_device(&p, &ext, m, pc, ws, &rd);
    bbjd_workspace_free(ws);
    const double wd = worst_residual(&rd);
    printf("device: status %d, %lld pairs, %lld iterations, worst residual %.2e, %lld kernels\n",
           (int)sd, (long long)rd.nconv, (long long)rd.iters, wd, (long long)ext.kernel_launches);
    if (sd != BBJD_SUCCESS || rd.nconv != K || !(wd < 1e-8) || ext.kernel_launches <= 0) return 20;

    /* the reference's callback interface: host products and a host LU */
    factor(sigma);
    p.matvec_A = mvA;
    p.matvec_B = mvB;
    p.precond = lu_solve;
    ws = bbjd_workspace_alloc(&p);
    if (!ws) return 14;
    bbjd_result rc;
    memset(&rc, 0, sizeof rc);
    const bbjd_status sc = bbjd_solve(&p, ws, &rc);
    bbjd_workspace_free(ws);
    const double wc = worst_residual(&rc);
    printf("callbacks: status %d, %lld pairs, %lld iterations, worst residual %.2e\n", (int)sc,
           (long long)rc.nconv, (long long)rc.iters, wc);
    if (sc != BBJD_SUCCESS || rc.nconv != K || !(wc < 1e-8)) return 30;

    /* both found the K eigenvalues nearest sigma: the same set */
    for (int a = 0; a < K; ++a) {
        double best = 1e300;
        for (int b = 0; b < K; ++b) {
            const double d = cabs(rd.eigenvalues[a] - rc.eigenvalues[b]);
            if (d < best) best = d;
        }
        if (best > 1e-6) {
            printf("eigenvalue %d differs by %.2e\n", a, best);
            return 40;
        }
    }
    bbjd_result_free(&rd);
    bbjd_result_free(&rc);
    bbjd_precond_free(pc);
    bbjd_bbt_free(m);
    printf("ok\n");
    return 0;
}
