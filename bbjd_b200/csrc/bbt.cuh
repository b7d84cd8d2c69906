// Device-resident block-bordered (BBT) pencil and its preconditioners.
#pragma once

#include <mutex>
#include <vector>

#include "dense.cuh"

struct bbjd_precond;

namespace bbjd {
// Reduction scratch of one fused product (tau-row partials and the residual
// norm).  The matrix owns one; each device solve owns another, so solves on
// different streams never share it.
struct BBTScratch {
    int G = 0;                       // CTAs of the product kernel
    cplx *tau_part = nullptr;        // [G][t]
    double *rn_part = nullptr;       // [G]
    double *rnorm = nullptr;         // ||r|| of the last residual product
    double *rtau_nsq = nullptr;      // [t] |r|^2 of the tau rows
    unsigned *counter = nullptr;     // completion counter of the norm reduction
};
}  // namespace bbjd

struct bbjd_bbt_matrix {
    int b = 0, t = 0;
    int64_t nblk = 0, nb = 0, n = 0;
    bbjd::cplx *Ad = nullptr, *Al = nullptr, *Au = nullptr, *Bd = nullptr;  // [nblk][b*b] col-major
    bbjd::cplx *E = nullptr;   // nb x t col-major
    bbjd::cplx *FT = nullptr;  // n x t row-major == F (t x n) col-major
    bbjd::cplx *mem = nullptr;
    bbjd::BBTScratch sc;             // scratch of bbjd_bbt_matvec
};

namespace bbjd {

// yA = A x, yB = B x; if r != nullptr also r = tb*yA - ta*yB and
// *rnorm = ||r|| (device; sc->rnorm when null).  One pass over the pencil's
// storage, with the caller's scratch (the matrix's own when sc is null; two
// products in flight at once need two scratches).
bbjd_status bbt_apply(const bbjd_bbt_matrix *m, const BBTScratch *sc, const cplx *x, cplx *yA,
                      cplx *yB, cplx ta, cplx tb, cplx *r, double *rnorm, cudaStream_t st);
bbjd_status bbt_scratch_alloc(const bbjd_bbt_matrix *m, BBTScratch *sc);
void bbt_scratch_free(BBTScratch *sc);
bbjd_status precond_solve(const bbjd_precond *pc, int nrhs, const cplx *r, cplx *x, int64_t stride,
                          cudaStream_t st);
double precond_bytes(const bbjd_precond *pc, int nrhs);

double bbt_bytes(const bbjd_bbt_matrix *m, bool with_residual);

}  // namespace bbjd

struct bbjd_precond {
    int kind = 0, precision = 0;
    int b = 0, t = 0;
    int64_t nblk = 0, nb = 0, n = 0;
    // block cyclic reduction of the block-tridiagonal interior
    struct Level {
        int64_t N = 0, n_odd = 0, n_even = 0;
        bbjd::cplx *Dinv = nullptr, *DinvLo = nullptr, *DinvUp = nullptr;  // n_odd blocks
        bbjd::cplx *Alpha = nullptr, *Beta = nullptr;                      // n_even blocks
        int64_t vec_off = 0;  // offset of this level's compact vectors in lvl_rhs / lvl_x
    };
    std::vector<Level> levels;
    bbjd::cplx *Dinv_top = nullptr;
    bbjd::cplx *pool = nullptr;     // all factor blocks (FP64; released in mixed precision)
    const bbjd::cplx *pool_base = nullptr;  // the FP64 pool's address: offsets into pool32
    int64_t pool_elems = 0;
    float2 *pool32 = nullptr;       // complex64 copy of the factor blocks (mixed precision)
    float2 *Y32 = nullptr, *FT32 = nullptr;
    // border (t > 0): Y = K^-1 E (nb x t col-major), Sinv = (G - F1 Y)^-1 (t x t)
    bbjd::cplx *Y = nullptr;
    bbjd::cplx *Sinv = nullptr;
    const bbjd::cplx *FT = nullptr; // borrowed from the matrix
    // block Jacobi: Dinv for every block, Ginv for the tau corner
    bbjd::cplx *Ginv = nullptr;
    // solve scratch
    bbjd::cplx *lvl_rhs = nullptr, *lvl_x = nullptr;   // 2 RHS x (sum of level sizes)
    int64_t lvl_total = 0;
    int64_t top_off = 0;
    int G = 0;
    bbjd::cplx *tau_part = nullptr;  // [G][2][t]
    bbjd::cplx *x2 = nullptr;        // [2][t]
    bbjd::cplx *gbuf = nullptr;      // [2][t] r2 - F1 y
    // The reduced system of level `cut` (the first level with <= 64 blocks,
    // mcut = N b unknowns) solved by its dense inverse instead of the levels
    // below it and the top block: one matrix-vector product in place of a
    // dozen dependent small-level kernels.
    int64_t cut = -1, mcut = 0;
    bbjd::cplx *Minv = nullptr;      // mcut x mcut column-major
    bbjd::cplx *mpart = nullptr;     // [MV_CHUNKS][2][mcut] partial products
    int *err = nullptr;              // device: singular pivot seen
    double factor_seconds = 0.0;
    double min_pivot = 0.0;
    // The BCR solve captured as CUDA graphs, one per (r, x, stride, nrhs,
    // stream) seen twice: a solve calls the preconditioner with the same
    // buffers every outer iteration, and one graph launch replaces its
    // ~24 kernel launches.
    struct Graph {
        const void *r = nullptr;
        void *x = nullptr;
        int64_t stride = 0;
        int nrhs = 0;
        cudaStream_t st = nullptr;
        cudaGraphExec_t exec = nullptr;
        int launches = 0;               // kernels in the graph
    };
    std::vector<Graph> graphs;
    std::mutex graph_mu;
};
