// Tall-skinny dense kernels of the JDQZ iteration (FP64 complex, sm_100a).
//
// Replaces the OpenBLAS calls the reference makes on n-row data:
//   zgemv 'C' / 'N' + dznrm2 of CGS2/DGKS  (reference jd_core.c:207-241)
//   zgemv 'N' Ritz vector u = V x          (reference jd_core.c:870-877)
//   zgemv 'C' + zdotc pencil column/row    (reference jd_core.c:1085-1104)
//   zdotc + zaxpy SvdV step                (reference jd_core.c:966-971)
//   zgemm restart V*ZB, AV*ZB, BV*ZB       (reference jd_core.c:989-999)
//   zgemm W^H AV, W^H BV                   (reference jd_core.c:1020-1025)
//
// All are HBM-bound except the restart/Gram GEMMs (FP64 FMA-bound).  Every
// reduction is two-stage with a fixed summation order, so results do not
// depend on scheduling.
#include "dense.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdio>
#include <map>
#include <mutex>

namespace bbjd {

// Basis loads: FP64, or the complex64 shadow of the mixed-precision form
// widened to FP64.
__device__ __forceinline__ cplx ldq(const double2 *p) { return __ldcs(p); }
__device__ __forceinline__ cplx ldq(const float2 *p) {
    const float2 f = __ldcs(p);
    return mk((double)f.x, (double)f.y);
}

// ---------------------------------------------------------------------------
// Stage 1 of Q^H v: partial[g][x] for x = (m*NV + p)*ncols + j, plus the
// squared norms of the vectors at x = NM*NV*ncols + p.
// One CTA owns a contiguous row range; its slice of each vector is staged in
// shared memory once; warp w streams columns j = w, w + nwarps, ... of Q.
template <int NM, int NV, typename QT = cplx>
__global__ void __launch_bounds__(256) k_tsdot(int64_t n, int ncols, int64_t ld,
                                               const QT *__restrict__ Q0,
                                               const QT *__restrict__ Q1,
                                               const cplx *__restrict__ v0,
                                               const cplx *__restrict__ v1, int64_t rpc,
                                               cplx *__restrict__ partial, const int *flag) {
    if (flag && *flag == 0) return;
    extern __shared__ cplx sv[];
    const int64_t r0 = (int64_t)blockIdx.x * rpc;
    const int64_t r1 = min(n, r0 + rpc);
    const int nr = (int)max((int64_t)0, r1 - r0);
    const int X = NM * NV * ncols + NV;
    cplx *out = partial + (int64_t)blockIdx.x * X;

    double nsq[NV];
#pragma unroll
    for (int p = 0; p < NV; ++p) nsq[p] = 0.0;
    for (int i = threadIdx.x; i < nr; i += blockDim.x) {
        cplx a = v0[r0 + i];
        sv[i] = a;
        nsq[0] += cabs2(a);
        if (NV > 1) {
            cplx b = v1[r0 + i];
            sv[rpc + i] = b;
            nsq[NV - 1] += cabs2(b);
        }
    }
    __shared__ double snorm[NV][8];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
#pragma unroll
    for (int p = 0; p < NV; ++p) {
        double s = warp_sum(nsq[p]);
        if (lane == 0) snorm[p][warp] = s;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double s = 0.0;
        for (int w = 0; w < nwarps; ++w) s += snorm[threadIdx.x][w];
        out[NM * NV * ncols + threadIdx.x] = mk(s, 0.0);
    }

    for (int cj = warp; cj < NM * ncols; cj += nwarps) {
        const int m = cj / ncols, j = cj - m * ncols;
        const QT *q = ((NM > 1 && m == 1) ? Q1 : Q0) + (int64_t)j * ld + r0;
        cplx acc[NV];
#pragma unroll
        for (int p = 0; p < NV; ++p) acc[p] = mk(0.0, 0.0);
        int i = lane;
        for (; i + 96 < nr; i += 128) {
            cplx q0 = ldq(q + i), q1 = ldq(q + i + 32);
            cplx q2 = ldq(q + i + 64), q3 = ldq(q + i + 96);
#pragma unroll
            for (int p = 0; p < NV; ++p) {
                const cplx *s = sv + p * rpc;
                cfmac(acc[p], q0, s[i]);
                cfmac(acc[p], q1, s[i + 32]);
                cfmac(acc[p], q2, s[i + 64]);
                cfmac(acc[p], q3, s[i + 96]);
            }
        }
        for (; i < nr; i += 32) {
            cplx qv = ldq(q + i);
#pragma unroll
            for (int p = 0; p < NV; ++p) cfmac(acc[p], qv, sv[p * rpc + i]);
        }
#pragma unroll
        for (int p = 0; p < NV; ++p) {
            cplx s = warp_sum(acc[p]);
            if (lane == 0) out[(m * NV + p) * ncols + j] = s;
        }
    }
}

// Stage 2: out[x] = sum_g partial[g][x] in a fixed order.
__global__ void __launch_bounds__(256) k_reduce(const cplx *__restrict__ partial, int G, int X,
                                                cplx *__restrict__ out, const int *flag) {
    if (flag && *flag == 0) return;
    __shared__ cplx s[8][33];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int x = blockIdx.x * 32 + tx;
    cplx acc = mk(0.0, 0.0);
    if (x < X) {
        // four independent chains keep four loads in flight per thread
        cplx a1 = mk(0.0, 0.0), a2 = mk(0.0, 0.0), a3 = mk(0.0, 0.0);
        int g = ty;
        for (; g + 24 < G; g += 32) {
            acc = cadd(acc, partial[(int64_t)g * X + x]);
            a1 = cadd(a1, partial[(int64_t)(g + 8) * X + x]);
            a2 = cadd(a2, partial[(int64_t)(g + 16) * X + x]);
            a3 = cadd(a3, partial[(int64_t)(g + 24) * X + x]);
        }
        for (; g < G; g += 8) acc = cadd(acc, partial[(int64_t)g * X + x]);
        acc = cadd(cadd(acc, a1), cadd(a2, a3));
    }
    s[ty][tx] = acc;
    __syncthreads();
    if (ty == 0 && x < X) {
        cplx r = s[0][tx];
        for (int k = 1; k < 8; ++k) r = cadd(r, s[k][tx]);
        out[x] = r;
    }
}

// ---------------------------------------------------------------------------
// v_out = a v_in + b w_in - Q (c1 h1 + c2 h2), and ||v_out||.
// The last CTA to finish sums the per-CTA squared norms in a fixed order,
// stores the norm, and (optionally) raises the DGKS flag
//   flag_out = ||v_out|| < 0.7071 ||v_before||       (reference jd_core.c:232)
// where ||v_before||^2 is read from ref_nsq (the x = NM*NV*ncols slot the
// first-pass dot kernel wrote).
template <typename QT>
__global__ void __launch_bounds__(256) k_update(
    int64_t n, int ncols, int64_t ld, const QT *__restrict__ Q, const cplx *__restrict__ h1,
    const cplx *__restrict__ h2, cplx c1, cplx c2, cplx a, const cplx *v_in, cplx b,
    const cplx *__restrict__ w_in, cplx *v_out, double *__restrict__ nrm_part,
    unsigned *counter, double *norm_out, const cplx *ref_nsq, const double *ref_nrm, int *flag_out,
    const int *flag_in) {
    if (flag_in && *flag_in == 0) return;
    extern __shared__ cplx hs[];
    for (int j = threadIdx.x; j < ncols; j += blockDim.x) {
        cplx h = cmul(c1, h1[j]);
        if (h2) cfma(h, c2, h2[j]);
        hs[j] = h;
    }
    __syncthreads();
    double nsq = 0.0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        cplx acc = mk(0.0, 0.0);
        if (v_in) acc = cmul(a, v_in[i]);
        if (w_in) cfma(acc, b, w_in[i]);
        const QT *q = Q + i;
        int j = 0;
        for (; j + 8 <= ncols; j += 8) {
            cplx qv[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) qv[u] = ldq(q + (int64_t)(j + u) * ld);
#pragma unroll
            for (int u = 0; u < 8; ++u) cfms(acc, qv[u], hs[j + u]);
        }
        for (; j < ncols; ++j) cfms(acc, ldq(q + (int64_t)j * ld), hs[j]);
        v_out[i] = acc;
        nsq += cabs2(acc);
    }
    __shared__ double red[8];
    __shared__ bool last;
    double s = warp_sum(nsq);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        nrm_part[blockIdx.x] = t;
        __threadfence();
        last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    double t = 0.0;
    for (int g = threadIdx.x; g < (int)gridDim.x; g += blockDim.x) t += __ldcg(nrm_part + g);
    t = warp_sum(t);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
        const double nrm = sqrt(tot);
        *norm_out = nrm;
        if (flag_out) {
            const double before = ref_nsq ? sqrt(ref_nsq->x) : (ref_nrm ? *ref_nrm : 0.0);
            *flag_out = (nrm < 0.7071 * before) ? 1 : 0;
        }
        *counter = 0u;
    }
}

// ---------------------------------------------------------------------------
// A CGS update fused with the dots of the DGKS re-pass that may follow it:
// v_out, ||v_out|| and the DGKS flag exactly as k_update, and, from the same
// read of Q, per-CTA partials of Q^H v_out (partial[g][j], j < ncols;
// partial[g][ncols] = the CTA's ||v_out||^2) for k_reduce.  Without it the
// re-pass reads Q twice more (dots, then the update); with it once.
//
// One persistent CTA of 16 warps per SM walks tiles of 32 rows.  A tile's
// 32 x ncols slice of Q, and its 32 rows of v_in and w_in, are copied to
// shared memory by cp.async into a ring of NST buffers (NST - 1 tiles in
// flight while one is used; three where they fit, ncols <= 143, else two).
// A tile's column j sits at j * 33 (one 16-byte pad per column), so a warp
// reading one row across 32 columns and a warp reading one column across
// 32 rows both touch every bank group equally.  Two phases per tile, two
// barriers:
//   1. warp w forms rows w and w + 16: each lane sums Q[row, j] h[j] over
//      its columns j = lane + 32 c (h held in registers), a butterfly warp
//      sum gives the row's (Q h)[row], and v_out[row] = a v_in + b w_in -
//      (Q h)[row] goes to global memory and to the tile's v_out in shared
//      memory;
//   2. warp w owns columns w, w + 16, ... and lane l row l: every lane
//      accumulates conj(Q) v_out for its columns in registers across tiles;
//      the warp sums happen once, at the end.
// Summation orders are fixed (no atomics on values).
constexpr int UD_TR = 32;          // rows per tile
constexpr int UD_LD = UD_TR + 1;   // shared-memory stride of a tile column
constexpr int UD_WARPS = 16;
constexpr int UD_CPW = 14;         // phase-2 columns per warp (largest instance): ncols <= 224
constexpr int UD_HPL = 7;          // phase-1 columns per lane (largest instance)
constexpr int UD_MIN_COLS = 64;    // below, the separate dot pass is as cheap
constexpr size_t UD_SMEM_LIMIT = 231424;

// one ring buffer: the Q tile, then 32 rows of v_in and of w_in
__host__ __device__ inline size_t update_dot_stage(int ncols) { return (size_t)ncols * UD_LD + 2 * UD_TR; }
static size_t update_dot_smem(int ncols, int stages = 2) {
    return sizeof(cplx) * ((size_t)stages * update_dot_stage(ncols) + UD_TR + UD_WARPS);
}
// Three tile buffers (two tiles in flight while one is used) where they fit
// in shared memory (ncols <= 143), else two.
static int update_dot_stages(int ncols) {
    return update_dot_smem(ncols, 3) <= UD_SMEM_LIMIT ? 3 : 2;
}

bool update_dot_fits(int ncols) {
    return ncols >= UD_MIN_COLS && ncols <= UD_WARPS * UD_CPW && ncols <= 32 * UD_HPL &&
           update_dot_smem(ncols) <= UD_SMEM_LIMIT;
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int src_bytes) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(a), "l"(gmem), "r"(src_bytes)
                 : "memory");
}

template <int NST, int CPW>
__global__ void __launch_bounds__(UD_WARPS * 32, 1) k_update_dot(
    int64_t n, int ncols, int64_t ld, const cplx *__restrict__ Q, const cplx *__restrict__ h1,
    const cplx *__restrict__ h2, cplx c1, cplx c2, cplx a, const cplx *v_in, cplx b,
    const cplx *w_in, cplx *v_out, cplx *__restrict__ partial, double *__restrict__ nrm_part,
    unsigned *counter, double *norm_out, const cplx *ref_nsq, const double *ref_nrm,
    int *flag_out) {
    extern __shared__ cplx ud_smem[];
    const int per = (int)update_dot_stage(ncols);
    const int qper = ncols * UD_LD;
    cplx *ring = ud_smem;                       // NST x [Q tile | v_in rows | w_in rows]
    cplx *vs = ring + NST * per;                // the tile's v_out
    double *wn = reinterpret_cast<double *>(vs + UD_TR);   // per-warp ||v_out||^2
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // phase-1 coefficients of this lane's columns
    constexpr int HPL = CPW / 2;   // phase-1 columns per lane
    cplx hr[HPL];
#pragma unroll
    for (int c = 0; c < HPL; ++c) {
        const int j = lane + 32 * c;
        cplx h = mk(0.0, 0.0);
        if (j < ncols) {
            h = cmul(c1, h1[j]);
            if (h2) cfma(h, c2, h2[j]);
        }
        hr[c] = h;
    }
    const int64_t ntiles = (n + UD_TR - 1) / UD_TR;
    // Thread tid copies element (tid & 31) of columns (tid >> 5) + 16 i,
    // i = 0, 1, ...: its source and destination advance by fixed strides.
    const int cr = tid & (UD_TR - 1), cj0 = tid >> 5;
    const cplx *qsrc = Q + (int64_t)cj0 * ld + cr;
    const int64_t qstep = (int64_t)UD_WARPS * ld;
    const int dst0 = cj0 * UD_LD + cr;
    // rows past n are zero-filled (source size 0), so they add nothing
    auto issue = [&](int64_t tile, cplx *dst) {
        const int64_t row0 = tile * UD_TR;
        const bool in = row0 + cr < n;
        const cplx *src = qsrc + (in ? row0 : -cr);
        const int bytes = in ? 16 : 0;
        int d = dst0;
        for (int j = cj0; j < ncols; j += UD_WARPS) {
            cp_async16(dst + d, src, bytes);
            src += qstep;
            d += UD_WARPS * UD_LD;
        }
        if (tid < 2 * UD_TR) {
            const cplx *src = tid < UD_TR ? v_in : w_in;
            const int r = tid & (UD_TR - 1);
            const int64_t row = row0 + r;
            if (src) {
                const bool in = row < n;
                cp_async16(dst + qper + tid, src + (in ? row : 0), in ? 16 : 0);
            }
        }
    };
    cplx acc[CPW];
#pragma unroll
    for (int c = 0; c < CPW; ++c) acc[c] = mk(0.0, 0.0);
    double nsq = 0.0;
    int buf = 0;
    int64_t tile = blockIdx.x;
    // prologue: the first NST - 1 tiles, one commit group each (possibly
    // empty, so the group count stays in step with the tiles)
#pragma unroll
    for (int p = 0; p < NST - 1; ++p) {
        const int64_t t = tile + (int64_t)p * gridDim.x;
        if (t < ntiles) issue(t, ring + p * per);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    for (; tile < ntiles; tile += gridDim.x) {
        // all but the newest NST - 2 groups complete: this tile has landed
        if constexpr (NST == 3)
            asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        else
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        __syncthreads();    // tile landed everywhere; the buffer and vs of the last tile are free
        const int64_t next = tile + (int64_t)(NST - 1) * gridDim.x;
        const int nbuf = buf + NST - 1 >= NST ? buf - 1 : buf + NST - 1;
        if (next < ntiles) issue(next, ring + nbuf * per);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        const cplx *Qt = ring + buf * per;
        const int64_t row0 = tile * UD_TR;
        // phase 1: rows warp and warp + 16
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int r = warp + UD_WARPS * q;
            cplx p = mk(0.0, 0.0);
#pragma unroll
            for (int c = 0; c < HPL; ++c) {
                const int j = lane + 32 * c;
                if (j < ncols) cfma(p, Qt[j * UD_LD + r], hr[c]);
            }
            p = warp_sum(p);
            if (lane == 0) {
                const int64_t row = row0 + r;
                cplx vo = mk(0.0, 0.0);
                if (row < n) {
                    cplx base = mk(0.0, 0.0);
                    if (v_in) base = cmul(a, Qt[qper + r]);
                    if (w_in) cfma(base, b, Qt[qper + UD_TR + r]);
                    vo = csub(base, p);
                    v_out[row] = vo;
                    nsq += cabs2(vo);
                }
                vs[r] = vo;
            }
        }
        __syncthreads();
        // phase 2: conj(Q) v_out for this warp's columns, lane = row
        const cplx vo = vs[lane];
#pragma unroll
        for (int c = 0; c < CPW; ++c) {
            const int j = warp + UD_WARPS * c;
            if (j < ncols) cfmac(acc[c], Qt[j * UD_LD + lane], vo);
        }
        buf = buf + 1 == NST ? 0 : buf + 1;
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    cplx *out = partial + (int64_t)blockIdx.x * (ncols + 1);
#pragma unroll
    for (int c = 0; c < CPW; ++c) {
        const int j = warp + UD_WARPS * c;
        const cplx sum = warp_sum(acc[c]);
        if (lane == 0 && j < ncols) out[j] = sum;
    }
    if (lane == 0) wn[warp] = nsq;
    __syncthreads();
    __shared__ bool last;
    if (warp == 0) {
        if (lane == 0) {
            double t = 0.0;
            for (int w = 0; w < UD_WARPS; ++w) t += wn[w];
            out[ncols] = mk(t, 0.0);
            nrm_part[blockIdx.x] = t;
            __threadfence();
            last = (atomicAdd(counter, 1u) == gridDim.x - 1);
        }
    }
    __syncthreads();
    if (!last || warp != 0) return;
    double t = 0.0;
    for (int g = lane; g < (int)gridDim.x; g += 32) t += __ldcg(nrm_part + g);
    t = warp_sum(t);
    if (lane == 0) {
        const double nrm = sqrt(t);
        *norm_out = nrm;
        if (flag_out) {
            const double before = ref_nsq ? sqrt(ref_nsq->x) : (ref_nrm ? *ref_nrm : 0.0);
            *flag_out = (nrm < 0.7071 * before) ? 1 : 0;
        }
        *counter = 0u;
    }
}

// out = v / norm (norm read on the device); if norm <= thresh, out = v.
__global__ void k_scale(int64_t n, const cplx *v, const double *norm, double thresh, cplx *out) {
    const double nr = *norm;
    const double s = nr > thresh ? 1.0 / nr : 1.0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = cscale(v[i], s);
}

// out = a x + b y with device-resident complex coefficients.
__global__ void k_axpby(int64_t n, const cplx *a_dev, cplx a_host, const cplx *x,
                        const cplx *b_dev, cplx b_host, const cplx *y, cplx *out) {
    const cplx a = a_dev ? *a_dev : a_host;
    const cplx b = b_dev ? *b_dev : b_host;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        cplx r = cmul(a, x[i]);
        if (y) cfma(r, b, y[i]);
        out[i] = r;
    }
}

// SvdV step (reference jd_core.c:966-971): dots = [u^H z, u^H s] from the
// reduce kernel; out = z - s (u^H z)/(u^H s) when |u^H s| > 1e-300, else z.
__global__ void k_svdv(int64_t n, const cplx *__restrict__ dots, const cplx *__restrict__ z,
                       const cplx *__restrict__ s, cplx *__restrict__ out) {
    const cplx uz = dots[0], us = dots[1];
    const double den = cabs2(us);
    cplx coeff = mk(0.0, 0.0);
    if (sqrt(den) > 1e-300) {
        // -(uz / us)
        coeff = mk(-(uz.x * us.x + uz.y * us.y) / den, -(uz.y * us.x - uz.x * us.y) / den);
    }
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        cplx r = z[i];
        cfma(r, coeff, s[i]);
        out[i] = r;
    }
}

// ---------------------------------------------------------------------------
// Restart compression out[:, 0:keep] = X[:, 0:k] Z[0:k, 0:keep] (FP64).
// A CTA owns 64 rows; the k x keep coefficient block Z is read from L2
// through 32-row K-slices staged in shared memory.  Each thread holds a
// 4 x RC register tile.  The CTA writes its rows only after it has read all
// of X's columns for them, so out may alias X (in-place restart, no swap
// buffer and no copy-back as in reference jd_core.c:991-999).
constexpr int RG_ROWS = 64, RG_KS = 16;
template <int RC>
__global__ void __launch_bounds__(256) k_restart_gemm(int64_t n, int k, int keep,
                                                      const cplx *X, int64_t ldx,
                                                      const cplx *__restrict__ Z, int ldz,
                                                      cplx *out) {
    // thread layout: 16 row-groups x 16 column-groups; rows r = rg + 16*u (u<4),
    // columns c = cg + 16*v (v < RC) -> covers 64 rows x 16*RC columns.
    __shared__ cplx sX[RG_KS][RG_ROWS];
    __shared__ cplx sZ[RG_KS][16 * RC];
    const int tid = threadIdx.x, rg = tid & 15, cg = tid >> 4;
    const int64_t row0 = (int64_t)blockIdx.x * RG_ROWS;
    const int colbase = blockIdx.y * 16 * RC;
    cplx acc[4][RC];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < RC; ++v) acc[u][v] = mk(0.0, 0.0);

    for (int j0 = 0; j0 < k; j0 += RG_KS) {
        for (int e = tid; e < RG_KS * RG_ROWS; e += 256) {
            const int jj = e / RG_ROWS, rr = e - jj * RG_ROWS;
            const int64_t row = row0 + rr;
            sX[jj][rr] = (j0 + jj < k && row < n) ? X[(int64_t)(j0 + jj) * ldx + row] : mk(0.0, 0.0);
        }
        for (int e = tid; e < RG_KS * 16 * RC; e += 256) {
            const int jj = e % RG_KS, cc = e / RG_KS;
            const int col = colbase + cc;
            sZ[jj][cc] = (j0 + jj < k && col < keep) ? Z[(int64_t)col * ldz + j0 + jj] : mk(0.0, 0.0);
        }
        __syncthreads();
#pragma unroll 4
        for (int jj = 0; jj < RG_KS; ++jj) {
            cplx xv[4], zv[RC];
#pragma unroll
            for (int u = 0; u < 4; ++u) xv[u] = sX[jj][rg + 16 * u];
#pragma unroll
            for (int v = 0; v < RC; ++v) zv[v] = sZ[jj][cg + 16 * v];
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < RC; ++v) cfma(acc[u][v], xv[u], zv[v]);
        }
        __syncthreads();
    }
    // every CTA of this row block must finish reading X before any writes
    // when out aliases X: the grid's y dimension splits columns, so the
    // in-place form is only used with gridDim.y == 1 (checked on the host).
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int64_t row = row0 + rg + 16 * u;
        if (row >= n) continue;
#pragma unroll
        for (int v = 0; v < RC; ++v) {
            const int col = colbase + cg + 16 * v;
            if (col < keep) out[(int64_t)col * ldx + row] = acc[u][v];
        }
    }
}

// The same GEMM with its operands staged by the tensor-memory accelerator:
// per 16-column K-slice, one 2D TMA load brings the CTA's 64 x 16 tile of X
// (a box of 128 doubles x 16 columns over X viewed as a 2n x k FP64 array)
// and one the 16 x 16 RC slice of Z, into a four-stage ring completed
// through mbarrier transaction counts; thread 0 issues, three slices stay in
// flight while one is multiplied.  Out-of-range rows and columns arrive as
// zeros.  The FP64 FMA loop and the register tile are k_restart_gemm's.
// Every mbarrier wait is bounded: a wait that runs out sets *err and the
// CTA returns without writing (the caller reports a device timeout).
__device__ __forceinline__ unsigned smem_u32(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
// true once the barrier's phase `parity` has completed; false when that
// has not happened within `max_cycles` SM clock cycles
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity, long long max_cycles) {
    const unsigned a = smem_u32(bar);
    const long long t0 = clock64();
    for (;;) {
        unsigned ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
        if (clock64() - t0 > max_cycles) return false;
    }
}
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y,
                                            unsigned long long *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

constexpr int RT_STAGES = 4;
// a stage that has not landed after ~1 s (2e9 cycles at <= 2 GHz) never will
constexpr long long RT_WAIT_CYCLES = 2000000000LL;
template <int RC>
constexpr size_t restart_tma_smem() {
    // + 128: the ring starts at the first 128-byte boundary of the block
    return sizeof(cplx) * (size_t)RT_STAGES * (RG_KS * RG_ROWS + 16 * RC * RG_KS) + 128;
}

template <int RC>
__global__ void __launch_bounds__(256, 1) k_restart_gemm_tma(const __grid_constant__ CUtensorMap tx,
                                                             const __grid_constant__ CUtensorMap tz,
                                                             int64_t n, int k, int keep, int64_t ldx,
                                                             cplx *out, int *err, long long wait_cycles,
                                                             unsigned tx_extra) {
    constexpr int XT = RG_KS * RG_ROWS;     // X tile: [16 columns][64 rows]
    constexpr int ZT = 16 * RC * RG_KS;     // Z slice: [16 RC columns][16 rows]
    constexpr unsigned BYTES = (unsigned)(sizeof(cplx) * (XT + ZT));
    extern __shared__ __align__(128) unsigned char rt_smem[];
    // TMA destinations 128-byte aligned whatever the block's static layout
    unsigned char *base = rt_smem + ((128u - (smem_u32(rt_smem) & 127u)) & 127u);
    cplx *sx = reinterpret_cast<cplx *>(base);
    cplx *sz = sx + RT_STAGES * XT;
    __shared__ __align__(8) unsigned long long full[RT_STAGES];
    __shared__ int abort_flag;
    const int tid = threadIdx.x, rg = tid & 15, cg = tid >> 4;
    const int64_t row0 = (int64_t)blockIdx.x * RG_ROWS;
    const int nk = (k + RG_KS - 1) / RG_KS;
    if (tid == 0) {
        for (int st = 0; st < RT_STAGES; ++st) mbar_init(&full[st], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        abort_flag = 0;
    }
    __syncthreads();
    auto load = [&](int kt) {
        const int st = kt % RT_STAGES;
        mbar_expect_tx(&full[st], BYTES + tx_extra);
        tma_load_2d(sx + st * XT, &tx, (int)(2 * row0), kt * RG_KS, &full[st]);
        tma_load_2d(sz + st * ZT, &tz, kt * 2 * RG_KS, 0, &full[st]);
    };
    if (tid == 0)
        for (int kt = 0; kt < RT_STAGES - 1 && kt < nk; ++kt) load(kt);
    cplx acc[4][RC];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < RC; ++v) acc[u][v] = mk(0.0, 0.0);
    for (int kt = 0; kt < nk; ++kt) {
        const int st = kt % RT_STAGES;
        // the stage of slice kt - 1 was released by the barrier that ended it
        if (tid == 0 && kt + RT_STAGES - 1 < nk) load(kt + RT_STAGES - 1);
        if (!mbar_wait(&full[st], (unsigned)((kt / RT_STAGES) & 1), wait_cycles)) abort_flag = 1;
        const cplx *X = sx + st * XT, *Z = sz + st * ZT;
#pragma unroll 4
        for (int jj = 0; jj < RG_KS; ++jj) {
            cplx xv[4], zv[RC];
#pragma unroll
            for (int u = 0; u < 4; ++u) xv[u] = X[jj * RG_ROWS + rg + 16 * u];
#pragma unroll
            for (int v = 0; v < RC; ++v) zv[v] = Z[(cg + 16 * v) * RG_KS + jj];
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < RC; ++v) cfma(acc[u][v], xv[u], zv[v]);
        }
        __syncthreads();
        if (abort_flag) {
            if (tid == 0) {
                atomicExch(err, 1);
                // wait (bounded) for the slices still in flight before leaving
                const int issued = min(nk, kt + RT_STAGES);
                for (int q = kt; q < issued; ++q)
                    mbar_wait(&full[q % RT_STAGES], (unsigned)((q / RT_STAGES) & 1), wait_cycles);
            }
            return;
        }
    }
    // every CTA reads only its own 64 rows of X, so out may alias X
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int64_t row = row0 + rg + 16 * u;
        if (row >= n) continue;
#pragma unroll
        for (int v = 0; v < RC; ++v) {
            const int col = cg + 16 * v;
            if (col < keep) out[(int64_t)col * ldx + row] = acc[u][v];
        }
    }
}

// Gram stage 1: partial[g] (keep x keep, column-major) = X_g^H Y_g over the
// CTA's row range.  Each thread holds a 5 x 5 tile (keep <= 80 per launch
// tile; larger keep tiles over blockIdx.y / z).  The 8-row slices of X and
// Y are staged by cp.async into two buffers, so the next slice loads while
// this one is multiplied; rows past the range and columns past keep are
// zero-filled.
constexpr int GR_T = 80, GR_SUB = 8;
__global__ void __launch_bounds__(256) k_gram(int64_t n, int keep, const cplx *__restrict__ X,
                                              const cplx *__restrict__ Y, int64_t ldx,
                                              int64_t rpc, cplx *__restrict__ partial) {
    __shared__ __align__(16) cplx sX[2][GR_SUB][GR_T];
    __shared__ __align__(16) cplx sY[2][GR_SUB][GR_T];
    const int tid = threadIdx.x, ta = tid & 15, tb = tid >> 4;
    const int a0 = blockIdx.y * GR_T, b0 = blockIdx.z * GR_T;
    const int64_t r0 = (int64_t)blockIdx.x * rpc, r1 = min(n, r0 + rpc);
    cplx acc[5][5];
#pragma unroll
    for (int u = 0; u < 5; ++u)
#pragma unroll
        for (int v = 0; v < 5; ++v) acc[u][v] = mk(0.0, 0.0);
    // thread tid copies rows rr of columns c = e / GR_SUB, e = tid + 256 i:
    // consecutive threads take consecutive rows of one column
    auto stage = [&](int64_t rs, int buf) {
        for (int e = tid; e < GR_SUB * GR_T; e += 256) {
            const int c = e / GR_SUB, rr = e - c * GR_SUB;
            const int64_t row = rs + rr;
            const bool okx = row < r1 && a0 + c < keep;
            const bool oky = row < r1 && b0 + c < keep;
            cp_async16(&sX[buf][rr][c], X + (okx ? (int64_t)(a0 + c) * ldx + row : 0), okx ? 16 : 0);
            cp_async16(&sY[buf][rr][c], Y + (oky ? (int64_t)(b0 + c) * ldx + row : 0), oky ? 16 : 0);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    if (r0 < r1) stage(r0, 0);
    int buf = 0;
    for (int64_t rs = r0; rs < r1; rs += GR_SUB) {
        if (rs + GR_SUB < r1) {
            stage(rs + GR_SUB, buf ^ 1);       // the buffer the last slice used
            asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        }
        __syncthreads();
#pragma unroll 4
        for (int rr = 0; rr < GR_SUB; ++rr) {
            cplx xv[5], yv[5];
#pragma unroll
            for (int u = 0; u < 5; ++u) xv[u] = sX[buf][rr][ta + 16 * u];
#pragma unroll
            for (int v = 0; v < 5; ++v) yv[v] = sY[buf][rr][tb + 16 * v];
#pragma unroll
            for (int u = 0; u < 5; ++u)
#pragma unroll
                for (int v = 0; v < 5; ++v) cfmac(acc[u][v], xv[u], yv[v]);
        }
        __syncthreads();                      // this buffer is free for the slice after next
        buf ^= 1;
    }
    cplx *out = partial + (int64_t)blockIdx.x * keep * keep;
#pragma unroll
    for (int u = 0; u < 5; ++u) {
        const int a = a0 + ta + 16 * u;
        if (a >= keep) continue;
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            const int bb = b0 + tb + 16 * v;
            if (bb < keep) out[(int64_t)bb * keep + a] = acc[u][v];
        }
    }
}

// ===========================================================================
// Host wrappers
// ===========================================================================

std::atomic<long long> g_launches{0};

// SM count of the current device (cached per device).
int num_sms() {
    static std::mutex mu;
    static std::map<int, int> sms;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> g(mu);
    auto it = sms.find(dev);
    if (it != sms.end()) return it->second;
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return sms[dev] = v > 0 ? v : 148;
}

// A kernel's dynamic shared-memory limit is a per-device, per-process
// setting: raise it on the current device to at least `bytes`, never lower
// it (a concurrent solve on the same device may have raised it further for
// its own launches).
bbjd_status raise_smem_limit(const void *func, size_t bytes) {
    if (bytes <= 48 * 1024) return BBJD_SUCCESS;
    static std::mutex mu;
    static std::map<std::pair<int, const void *>, size_t> done;
    int dev = 0;
    BBJD_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> g(mu);
    size_t &cur = done[{dev, func}];
    if (cur >= bytes) return BBJD_SUCCESS;
    BBJD_CUDA_TRY(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    cur = bytes;
    return BBJD_SUCCESS;
}

static thread_local char g_errbuf[512];
void set_last_error(cudaError_t e, const char *what, const char *file, int line) {
    snprintf(g_errbuf, sizeof(g_errbuf), "%s: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
    fprintf(stderr, "bbjd_gpu: %s\n", g_errbuf);
}
const char *last_error() { return g_errbuf; }

bbjd_status Scratch::init(int64_t n_, int max_cols, int nvec) {
    n = n_;
    const int sms = num_sms();
    G = (int)std::max<int64_t>(1, std::min<int64_t>(4 * sms, (n + 255) / 256));
    rpc = ((n + G - 1) / G + 31) / 32 * 32;
    G = (int)((n + rpc - 1) / rpc);
    G2 = (int)std::max<int64_t>(1, std::min<int64_t>(8 * sms, (n + 255) / 256));
    maxX = 2 * 2 * (int64_t)max_cols + 4;
    BBJD_CUDA_TRY(cudaMalloc(&partial, sizeof(cplx) * (size_t)G * maxX));
    BBJD_CUDA_TRY(cudaMalloc(&nrm_part, sizeof(double) * (size_t)G2));
    BBJD_CUDA_TRY(cudaMalloc(&counter, sizeof(unsigned) * 4));
    BBJD_CUDA_TRY(cudaMemset(counter, 0, sizeof(unsigned) * 4));
    BBJD_CUDA_TRY(cudaMalloc(&red, sizeof(cplx) * (size_t)(nvec > 0 ? nvec : 1) * maxX));
    BBJD_CUDA_TRY(cudaMalloc(&scal, sizeof(double) * 64));
    BBJD_CUDA_TRY(cudaMalloc(&flags, sizeof(int) * 16));
    BBJD_CUDA_TRY(cudaMemset(flags, 0, sizeof(int) * 16));
    // the fused CGS update stages tiles of the basis in up to 226 KB
    bbjd_status s;
    for (const void *f : {(const void *)k_update_dot<3, 4>, (const void *)k_update_dot<3, 6>,
                          (const void *)k_update_dot<3, 8>, (const void *)k_update_dot<3, 10>,
                          (const void *)k_update_dot<2, 10>, (const void *)k_update_dot<2, 12>,
                          (const void *)k_update_dot<2, 14>})
        if ((s = raise_smem_limit(f, UD_SMEM_LIMIT))) return s;
    const size_t smem_need = sizeof(cplx) * 2 * (size_t)rpc;
    if ((s = raise_smem_limit((const void *)k_tsdot<1, 2>, smem_need))) return s;
    if ((s = raise_smem_limit((const void *)k_tsdot<2, 1>, smem_need))) return s;
    if ((s = raise_smem_limit((const void *)k_tsdot<1, 1>, smem_need))) return s;
    return BBJD_SUCCESS;
}

void Scratch::release() {
    cudaFree(partial); cudaFree(nrm_part); cudaFree(counter);
    cudaFree(red); cudaFree(scal); cudaFree(flags);
    partial = red = nullptr; nrm_part = scal = nullptr; counter = nullptr; flags = nullptr;
}

bbjd_status tsdot(Scratch &S, int NM, int NV, int ncols, int64_t ld, const cplx *Q0,
                  const cplx *Q1, const cplx *v0, const cplx *v1, cplx *out, const int *flag,
                  cudaStream_t st) {
    const int X = NM * NV * ncols + NV;
    if (X > S.maxX) return BBJD_ERR_INVALID;
    const size_t smem = sizeof(cplx) * NV * (size_t)S.rpc;
    if (NM == 1 && NV == 1)
        k_tsdot<1, 1><<<S.G, 256, smem, st>>>(S.n, ncols, ld, Q0, Q1, v0, v1, S.rpc, S.partial, flag);
    else if (NM == 1 && NV == 2)
        k_tsdot<1, 2><<<S.G, 256, smem, st>>>(S.n, ncols, ld, Q0, Q1, v0, v1, S.rpc, S.partial, flag);
    else if (NM == 2 && NV == 1)
        k_tsdot<2, 1><<<S.G, 256, smem, st>>>(S.n, ncols, ld, Q0, Q1, v0, v1, S.rpc, S.partial, flag);
    else
        return BBJD_ERR_INVALID;
    BBJD_LAUNCH_CHECK();
    k_reduce<<<(X + 31) / 32, 256, 0, st>>>(S.partial, S.G, X, out, flag);
    BBJD_LAUNCH_CHECK();
    return BBJD_SUCCESS;
}

bbjd_status tsdot_allow_smem(size_t bytes) { return raise_smem_limit((const void *)k_tsdot<1, 1>, bytes); }

bbjd_status reduce_partials(const cplx *partial, int G, int X, cplx *out, cudaStream_t st) {
    k_reduce<<<(X + 31) / 32, 256, 0, st>>>(partial, G, X, out, nullptr);
    BBJD_LAUNCH_CHECK();
    return BBJD_SUCCESS;
}

bbjd_status update(Scratch &S, int ncols, int64_t ld, const cplx *Q, const cplx *h1,
                   const cplx *h2, cplx c1, cplx c2, cplx a, const cplx *v_in, cplx b,
                   const cplx *w_in, cplx *v_out, double *norm_out, const cplx *ref_nsq,
                   const double *ref_nrm, int *flag_out, const int *flag_in, cudaStream_t st) {
    const size_t smem = sizeof(cplx) * (size_t)std::max(ncols, 1);
    k_update<<<S.G2, 256, smem, st>>>(S.n, ncols, ld, Q, h1, h2, c1, c2, a, v_in, b, w_in, v_out,
                                      S.nrm_part, S.counter, norm_out, ref_nsq, ref_nrm, flag_out,
                                      flag_in);
    BBJD_LAUNCH_CHECK();
    return BBJD_SUCCESS;
}

bbjd_status cgs_tail(Scratch &S, int ncols, int64_t ld, const cplx *Q, const cplx *h1,
                     const cplx *h2, cplx c1, cplx c2, cplx a, const cplx *v_in, cplx b,
                     const cplx *w_in, cplx *v_out, double *norm_out, const cplx *ref_nsq,
                     const double *ref_nrm, int *flag, cplx *h_re, cudaStream_t st) {
    bbjd_status s;
    if (ncols > 0 && update_dot_fits(ncols) && ncols + 1 <= S.maxX) {
        // the shared-memory limit was raised on this device by Scratch::init
        const int64_t ntiles = (S.n + UD_TR - 1) / UD_TR;
        const int G = (int)std::max<int64_t>(1, std::min<int64_t>({(int64_t)num_sms(), ntiles,
                                                                    (int64_t)S.G}));
        const int nst = update_dot_stages(ncols);
        // the narrowest instance that covers ncols: 16 CPW columns
        const int cpw = std::max(4, ((ncols + 15) / 16 + 1) / 2 * 2);
#define BBJD_UD(NST, CPW)                                                                         \
    k_update_dot<NST, CPW><<<G, UD_WARPS * 32, update_dot_smem(ncols, NST), st>>>(                \
        S.n, ncols, ld, Q, h1, h2, c1, c2, a, v_in, b, w_in, v_out, S.partial, S.nrm_part, S.counter, \
        norm_out, ref_nsq, ref_nrm, flag)
        if (nst == 3) {
            if (cpw <= 4) BBJD_UD(3, 4);
            else if (cpw <= 6) BBJD_UD(3, 6);
            else if (cpw <= 8) BBJD_UD(3, 8);
            else BBJD_UD(3, 10);
        } else {
            if (cpw <= 10) BBJD_UD(2, 10);
            else if (cpw <= 12) BBJD_UD(2, 12);
            else BBJD_UD(2, 14);
        }
#undef BBJD_UD
        BBJD_LAUNCH_CHECK();
        k_reduce<<<(ncols + 1 + 31) / 32, 256, 0, st>>>(S.partial, G, ncols + 1, h_re, flag);
        BBJD_LAUNCH_CHECK();
    } else {
        if ((s = update(S, ncols, ld, Q, h1, h2, c1, c2, a, v_in, b, w_in, v_out, norm_out, ref_nsq,
                        ref_nrm, flag, nullptr, st)))
            return s;
        if (ncols == 0) return BBJD_SUCCESS;
        if ((s = tsdot(S, 1, 1, ncols, ld, Q, nullptr, v_out, nullptr, h_re, flag, st))) return s;
    }
    return update(S, ncols, ld, Q, h_re, nullptr, mk(1, 0), mk(0, 0), mk(1, 0), v_out, mk(0, 0),
                  nullptr, v_out, norm_out, nullptr, nullptr, nullptr, flag, st);
}

bbjd_status scale_by_norm(Scratch &S, const cplx *v, const double *norm, double thresh,
                          cplx *out, cudaStream_t st) {
    k_scale<<<S.G2, 256, 0, st>>>(S.n, v, norm, thresh, out);
    BBJD_LAUNCH_CHECK();
    return BBJD_SUCCESS;
}

bbjd_status axpby(Scratch &S, const cplx *a_dev, cplx a, const cplx *x, const cplx *b_dev, cplx b,
                  const cplx *y, cplx *out, cudaStream_t st) {
    k_axpby<<<S.G2, 256, 0, st>>>(S.n, a_dev, a, x, b_dev, b, y, out);
    BBJD_LAUNCH_CHECK();
    return BBJD_SUCCESS;
}

bbjd_status axpby_n(int64_t count, cplx a, const cplx *x, cplx b, const cplx *y, cplx *out,
                    cudaStream_t st) {
    const int64_t g = std::min<int64_t>(8 * num_sms(), std::max<int64_t>(1, (count + 255) / 256));
    k_axpby<<<(unsigned)g, 256, 0, st>>>(count, nullptr, a, x, nullptr, b, y, out);
    BBJD_LAUNCH_CHECK();
    return BBJD_SUCCESS;
}

bbjd_status svdv(Scratch &S, const cplx *dots, const cplx *z, const cplx *s, cplx *out,
                 cudaStream_t st) {
    k_svdv<<<S.G2, 256, 0, st>>>(S.n, dots, z, s, out);
    BBJD_LAUNCH_CHECK();
    return BBJD_SUCCESS;
}

// cuTensorMapEncodeTiled from the driver, through the runtime (no link
// against libcuda); null when the driver does not provide it.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// A 2D FP64 tensor map: d0 contiguous doubles per column, d1 columns
// stride_bytes apart, boxes of b0 x b1, zeros outside.
static bool fp64_map(CUtensorMap *m, const void *base, uint64_t d0, uint64_t d1, uint64_t stride_bytes,
                     uint32_t b0, uint32_t b1) {
    const auto fn = tensor_map_encoder();
    if (!fn || ((uintptr_t)base & 15) || (stride_bytes & 15)) return false;
    cuuint64_t dims[2] = {d0, d1};
    cuuint64_t strides[1] = {stride_bytes};
    cuuint32_t box[2] = {b0, b1};
    cuuint32_t es[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<void *>(base), dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int RC>
static bool restart_gemm_tma(int64_t n, int k, int keep, const cplx *X, int64_t ldx, const cplx *Z_dev,
                             int ldz, cplx *out, int *err, cudaStream_t st,
                             long long wait_cycles = RT_WAIT_CYCLES, unsigned tx_extra = 0) {
    CUtensorMap tx, tz;
    // X as a 2n x k FP64 array (real and imaginary parts interleaved); its
    // tile origin x = 2 row0 is a multiple of 128 doubles, so 16-byte aligned
    if (!fp64_map(&tx, X, 2 * (uint64_t)n, (uint64_t)k, 16 * (uint64_t)ldx, 2 * RG_ROWS, RG_KS)) return false;
    if (!fp64_map(&tz, Z_dev, 2 * (uint64_t)k, (uint64_t)keep, 16 * (uint64_t)ldz, 2 * RG_KS, 16 * RC))
        return false;
    if (raise_smem_limit((const void *)k_restart_gemm_tma<RC>, restart_tma_smem<RC>())) return false;
    const unsigned gx = (unsigned)((n + RG_ROWS - 1) / RG_ROWS);
    k_restart_gemm_tma<RC><<<gx, 256, restart_tma_smem<RC>(), st>>>(tx, tz, n, k, keep, ldx, out, err,
                                                                    wait_cycles, tx_extra);
    return true;
}

bbjd_status restart_gemm_stalled(int64_t n, int k, int keep, const cplx *X, int64_t ldx,
                                 const cplx *Z_dev, int ldz, cplx *out, cudaStream_t st, int *err) {
    // every stage expects 16 bytes more than its two loads bring, so no
    // stage ever completes; each wait gives up after ~1 ms
    if (keep > 16 * 5 || !restart_gemm_tma<5>(n, k, keep, X, ldx, Z_dev, ldz, out, err, st, 2000000LL, 16u))
        return BBJD_ERR_INVALID;
    BBJD_LAUNCH_CHECK();
    return BBJD_SUCCESS;
}

bbjd_status restart_gemm(int64_t n, int k, int keep, const cplx *X, int64_t ldx, const cplx *Z_dev,
                         int ldz, cplx *out, cudaStream_t st, int *err) {
    // TMA-staged form (one column tile, keep <= 128) when the caller takes a
    // timeout flag; the plain form otherwise
    if (err && k > 0 && keep > 0 && keep <= 16 * 8) {
        bool ok = keep <= 16 * 2   ? restart_gemm_tma<2>(n, k, keep, X, ldx, Z_dev, ldz, out, err, st)
                  : keep <= 16 * 5 ? restart_gemm_tma<5>(n, k, keep, X, ldx, Z_dev, ldz, out, err, st)
                                   : restart_gemm_tma<8>(n, k, keep, X, ldx, Z_dev, ldz, out, err, st);
        if (ok) {
            BBJD_LAUNCH_CHECK();
            return BBJD_SUCCESS;
        }
    }
    const unsigned gx = (unsigned)((n + RG_ROWS - 1) / RG_ROWS);
    // one column tile covers keep <= 16*RC; in-place needs a single tile
    if (keep <= 16 * 2) {
        k_restart_gemm<2><<<dim3(gx, 1), 256, 0, st>>>(n, k, keep, X, ldx, Z_dev, ldz, out);
    } else if (keep <= 16 * 5) {
        k_restart_gemm<5><<<dim3(gx, 1), 256, 0, st>>>(n, k, keep, X, ldx, Z_dev, ldz, out);
    } else if (keep <= 16 * 8) {
        k_restart_gemm<8><<<dim3(gx, 1), 256, 0, st>>>(n, k, keep, X, ldx, Z_dev, ldz, out);
    } else {
        if (out == X) return BBJD_ERR_INVALID;   // multi-tile form cannot run in place
        const unsigned gy = (unsigned)((keep + 16 * 8 - 1) / (16 * 8));
        k_restart_gemm<8><<<dim3(gx, gy), 256, 0, st>>>(n, k, keep, X, ldx, Z_dev, ldz, out);
    }
    BBJD_LAUNCH_CHECK();
    return BBJD_SUCCESS;
}

bbjd_status gram(Scratch &S, int keep, const cplx *X, const cplx *Y, int64_t ldx, cplx *partial,
                 int Gg, cplx *out, cudaStream_t st) {
    const int64_t rpc = ((S.n + Gg - 1) / Gg + 15) / 16 * 16;
    const unsigned gt = (unsigned)((keep + GR_T - 1) / GR_T);
    k_gram<<<dim3((unsigned)Gg, gt, gt), 256, 0, st>>>(S.n, keep, X, Y, ldx, rpc, partial);
    BBJD_LAUNCH_CHECK();
    const int XX = keep * keep;
    k_reduce<<<(XX + 31) / 32, 256, 0, st>>>(partial, Gg, XX, out, nullptr);
    BBJD_LAUNCH_CHECK();
    return BBJD_SUCCESS;
}

// ---------------------------------------------------------------------------
// out (rows x ncols row-major, row stride ncols) = rows [r0, r0+rows) of Q
// (column-major, ld).  32 x 32 tiles staged through shared memory, so both
// the column reads and the row writes are coalesced; the +1 pad keeps the
// transposed reads of the tile free of bank conflicts.
__global__ void k_to_row_major(int64_t r0, int64_t rows, int ncols, int64_t ld,
                               const cplx *__restrict__ Q, cplx *__restrict__ out) {
    __shared__ cplx tile[32][33];
    const int64_t i0 = (int64_t)blockIdx.x * 32;
    const int j0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;      // 32 x 8 threads
    for (int c = ty; c < 32; c += 8) {
        const int64_t i = i0 + tx;
        const int j = j0 + c;
        if (i < rows && j < ncols) tile[c][tx] = Q[(int64_t)j * ld + r0 + i];
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int64_t i = i0 + r;
        const int j = j0 + tx;
        if (i < rows && j < ncols) out[i * ncols + j] = tile[tx][r];
    }
}

bbjd_status to_row_major(int64_t r0, int64_t rows, int ncols, int64_t ld, const cplx *Q, cplx *out,
                         cudaStream_t st) {
    if (rows <= 0 || ncols <= 0) return BBJD_SUCCESS;
    const dim3 grid((unsigned)((rows + 31) / 32), (unsigned)((ncols + 31) / 32)), block(32, 8);
    k_to_row_major<<<grid, block, 0, st>>>(r0, rows, ncols, ld, Q, out);
    BBJD_LAUNCH_CHECK();
    return BBJD_SUCCESS;
}

// ---------------------------------------------------------------------------
// Mixed-precision helpers: complex64 copies and passes over a complex64 basis.
__global__ void k_cvt_c64(int64_t count, const double2 *__restrict__ in, float2 *__restrict__ out) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride)
        out[i] = make_float2((float)in[i].x, (float)in[i].y);
}

bbjd_status to_c64(int64_t count, const cplx *in, float2 *out, cudaStream_t st) {
    const int64_t g = std::min<int64_t>(8 * num_sms(), std::max<int64_t>(1, (count + 255) / 256));
    k_cvt_c64<<<(unsigned)g, 256, 0, st>>>(count, in, out);
    BBJD_LAUNCH_CHECK();
    return BBJD_SUCCESS;
}

bbjd_status tsdot32(Scratch &S, int ncols, int64_t ld, const float2 *Q, const cplx *v, cplx *out,
                    cudaStream_t st, const int *flag) {
    const int X = ncols + 1;
    if (X > S.maxX) return BBJD_ERR_INVALID;
    const size_t smem = sizeof(cplx) * (size_t)S.rpc;
    bbjd_status s = raise_smem_limit((const void *)k_tsdot<1, 1, float2>, smem);
    if (s) return s;
    k_tsdot<1, 1, float2><<<S.G, 256, smem, st>>>(S.n, ncols, ld, Q, Q, v, nullptr, S.rpc, S.partial, flag);
    BBJD_LAUNCH_CHECK();
    k_reduce<<<(X + 31) / 32, 256, 0, st>>>(S.partial, S.G, X, out, flag);
    BBJD_LAUNCH_CHECK();
    return BBJD_SUCCESS;
}

bbjd_status update32(Scratch &S, int ncols, int64_t ld, const float2 *Q, const cplx *h, cplx *v,
                     double *norm_out, cudaStream_t st, const cplx *ref_nsq, int *flag_out,
                     const int *flag_in) {
    const size_t smem = sizeof(cplx) * (size_t)std::max(ncols, 1);
    k_update<float2><<<S.G2, 256, smem, st>>>(S.n, ncols, ld, Q, h, nullptr, mk(1, 0), mk(0, 0), mk(1, 0),
                                              v, mk(0, 0), nullptr, v, S.nrm_part, S.counter, norm_out,
                                              ref_nsq, nullptr, flag_out, flag_in);
    BBJD_LAUNCH_CHECK();
    return BBJD_SUCCESS;
}

__global__ void k_cvt_c128(int64_t count, const float2 *__restrict__ in, double2 *__restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float2 a = in[i];
        out[i] = make_double2((double)a.x, (double)a.y);
    }
}

bbjd_status to_c128(int64_t count, const float2 *in, cplx *out, cudaStream_t st) {
    const int64_t g = std::min<int64_t>(8 * num_sms(), std::max<int64_t>(1, (count + 255) / 256));
    k_cvt_c128<<<(unsigned)g, 256, 0, st>>>(count, in, out);
    BBJD_LAUNCH_CHECK();
    return BBJD_SUCCESS;
}

}  // namespace bbjd
