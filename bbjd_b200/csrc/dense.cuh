// Host-side interface of the tall-skinny dense kernels (dense.cu).
#pragma once

#include "common.cuh"

namespace bbjd {

const char *last_error();

// Device flag set (never cleared within a solve) by a kernel whose bounded
// mbarrier wait ran out.
constexpr int SCRATCH_FLAG_TMO = 15;

// Per-solve scratch for two-stage reductions.  One Scratch per stream:
// the last-CTA norm counter is not shared between concurrent launches.
struct Scratch {
    int64_t n = 0;
    int G = 0;          // CTAs of the dot kernels
    int64_t rpc = 0;    // rows per dot CTA
    int G2 = 0;         // CTAs of the streaming update kernels
    int64_t maxX = 0;
    cplx *partial = nullptr;
    double *nrm_part = nullptr;
    unsigned *counter = nullptr;
    cplx *red = nullptr;     // reduced dot outputs
    double *scal = nullptr;  // device scalar slots
    int *flags = nullptr;    // device flags (16); flags[SCRATCH_FLAG_TMO]: a bounded wait ran out
    bbjd_status init(int64_t n, int max_cols, int nvec);
    void release();
};

// out[x] = sum over rows of conj(Q_m[:, j]) v_p, x = (m*NV + p)*ncols + j;
// out[NM*NV*ncols + p] = ||v_p||^2.  Skipped when flag && *flag == 0.
bbjd_status tsdot(Scratch &S, int NM, int NV, int ncols, int64_t ld, const cplx *Q0,
                  const cplx *Q1, const cplx *v0, const cplx *v1, cplx *out, const int *flag,
                  cudaStream_t st);

// v_out = a v_in + b w_in - Q (c1 h1 + c2 h2); *norm_out = ||v_out||;
// *flag_out = ||v_out|| < 0.7071 ||v_before|| with ||v_before|| = sqrt(ref_nsq.x)
// or *ref_nrm.  Skipped when flag_in && !*flag_in.  Q may be null when ncols == 0.
bbjd_status update(Scratch &S, int ncols, int64_t ld, const cplx *Q, const cplx *h1,
                   const cplx *h2, cplx c1, cplx c2, cplx a, const cplx *v_in, cplx b,
                   const cplx *w_in, cplx *v_out, double *norm_out, const cplx *ref_nsq,
                   const double *ref_nrm, int *flag_out, const int *flag_in, cudaStream_t st);

// The rest of a CGS2 / DGKS step once the first pass's dots h1 (and h2) are
// known: v_out = a v_in + b w_in - Q (c1 h1 + c2 h2), ||v_out|| into
// *norm_out and the DGKS flag into *flag (as update()); then, where the
// flag is raised, h_re = Q^H v_out and v_out -= Q h_re, ||v_out||.  For
// ncols within update_dot_fits() the re-pass dots come from the update's
// own read of Q (one pass over Q fewer).  h_re holds ncols + 1 values.
bool update_dot_fits(int ncols);
bbjd_status cgs_tail(Scratch &S, int ncols, int64_t ld, const cplx *Q, const cplx *h1,
                     const cplx *h2, cplx c1, cplx c2, cplx a, const cplx *v_in, cplx b,
                     const cplx *w_in, cplx *v_out, double *norm_out, const cplx *ref_nsq,
                     const double *ref_nrm, int *flag, cplx *h_re, cudaStream_t st);
bbjd_status scale_by_norm(Scratch &S, const cplx *v, const double *norm, double thresh,
                          cplx *out, cudaStream_t st);
bbjd_status axpby(Scratch &S, const cplx *a_dev, cplx a, const cplx *x, const cplx *b_dev, cplx b,
                  const cplx *y, cplx *out, cudaStream_t st);
// out[0:count] = a x + b y (y may be null), host scalars.
bbjd_status axpby_n(int64_t count, cplx a, const cplx *x, cplx b, const cplx *y, cplx *out,
                    cudaStream_t st);
bbjd_status svdv(Scratch &S, const cplx *dots, const cplx *z, const cplx *s, cplx *out,
                 cudaStream_t st);
// out (n x keep) = X (n x k) Z (k x keep); out may alias X.  With err (a
// device int) the operands are staged by TMA and a bounded wait that runs
// out sets *err to 1 (nothing is written then).
bbjd_status restart_gemm(int64_t n, int k, int keep, const cplx *X, int64_t ldx, const cplx *Z_dev,
                         int ldz, cplx *out, cudaStream_t st, int *err = nullptr);
// The TMA-staged form with a transaction count that never completes (the
// failure-detection test): its bounded waits run out and set *err.
bbjd_status restart_gemm_stalled(int64_t n, int k, int keep, const cplx *X, int64_t ldx,
                                 const cplx *Z_dev, int ldz, cplx *out, cudaStream_t st, int *err);
// Raise the dynamic shared-memory limit of the one-matrix, one-vector dot
// kernel to `bytes` (no-op up to 48 KB).
bbjd_status tsdot_allow_smem(size_t bytes);
// out[x] = sum_g partial[g*X + x], fixed order.
bbjd_status reduce_partials(const cplx *partial, int G, int X, cplx *out, cudaStream_t st);
// out (keep x keep col-major, device) = X^H Y; partial holds Gg*keep*keep.
bbjd_status gram(Scratch &S, int keep, const cplx *X, const cplx *Y, int64_t ldx, cplx *partial,
                 int Gg, cplx *out, cudaStream_t st);

// out (rows x ncols, row-major) = rows [r0, r0+rows) of the column-major Q.
bbjd_status to_row_major(int64_t r0, int64_t rows, int ncols, int64_t ld, const cplx *Q, cplx *out,
                         cudaStream_t st);

// Mixed precision: out = complex64(in) and back; a CGS pass over a complex64
// basis Q with an FP64 vector v, FP64 accumulation (dots into out[0:ncols],
// ||v||^2 into out[ncols]; v -= Q h, ||v|| into *norm_out and, with
// ref_nsq / flag_out, the DGKS flag as update()).  Skipped when flag /
// flag_in is set and *flag == 0.
bbjd_status to_c64(int64_t count, const cplx *in, float2 *out, cudaStream_t st);
bbjd_status to_c128(int64_t count, const float2 *in, cplx *out, cudaStream_t st);
bbjd_status tsdot32(Scratch &S, int ncols, int64_t ld, const float2 *Q, const cplx *v, cplx *out,
                    cudaStream_t st, const int *flag = nullptr);
bbjd_status update32(Scratch &S, int ncols, int64_t ld, const float2 *Q, const cplx *h, cplx *v,
                     double *norm_out, cudaStream_t st, const cplx *ref_nsq = nullptr,
                     int *flag_out = nullptr, const int *flag_in = nullptr);

}  // namespace bbjd
