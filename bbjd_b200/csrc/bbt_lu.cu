// Device preconditioners for A - sigma B of a block-bordered pencil.
//
// The reference leaves M^-1 to the caller (preconditioner.solve, reference
// bbjd.py:208-219, _bbjd_c.c:99-123; in production an external sparse LU,
// README.md:38-44).  This file builds it on the device:
//
//  * exact block-bordered LU.  With K the block-tridiagonal interior of
//    A - sigma B, E its border columns and [F1 G] its tau rows,
//        M = [[K, E], [F1, G]],   S = G - F1 K^-1 E  (t x t Schur complement)
//    and a solve is  y = K^-1 r1;  x2 = S^-1 (r2 - F1 y);  x1 = y - (K^-1 E) x2.
//    K^-1 is applied by block cyclic reduction (BCR): level l eliminates the
//    odd blocks of the level's block-tridiagonal system, leaving a system of
//    half the size on the even blocks, for log2(nblk) levels.  Each level is
//    one fully parallel pass, so a solve is ~2 log2(nblk) short kernels instead
//    of nblk sequential block steps.  Diagonal blocks are inverted by
//    Gauss-Jordan elimination with partial pivoting inside the block.
//  * block Jacobi: the inverses of the diagonal blocks of A - sigma B and of
//    the tau corner G (the approximate preconditioner of the inner-GMRES
//    configuration).
#include "bbt.cuh"

#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <vector>

extern "C" void scipy_zgesv_(const int *n, const int *nrhs, bbjd_zomplex *a, const int *lda,
                             int *ipiv, bbjd_zomplex *b, const int *ldb, int *info);

namespace bbjd {

// Factor loads: FP64 blocks, or complex64 blocks (the mixed-precision form)
// widened to FP64 for the arithmetic.
__device__ __forceinline__ cplx ldm(const double2 *p) { return __ldcs(p); }
__device__ __forceinline__ cplx ldm(const float2 *p) {
    const float2 f = __ldcs(p);
    return mk((double)f.x, (double)f.y);
}

__global__ void k_to_c64(int64_t count, const double2 *__restrict__ in, float2 *__restrict__ out) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride)
        out[i] = make_float2((float)in[i].x, (float)in[i].y);
}

// ---------------------------------------------------------------------------
// Shared-memory block helpers (row-major, padded row stride).
template <int BS>
struct Blk {
    static constexpr int LD = BS + 1;       // padded row stride of a b x b tile
    static constexpr int LDA = 2 * BS + 1;  // padded row stride of [M | I]
};

// Load a column-major global block into a row-major smem tile (stride ld).
template <int BS>
__device__ void load_blk(cplx *s, int ld, const cplx *__restrict__ g) {
    for (int e = threadIdx.x; e < BS * BS; e += blockDim.x) {
        const int i = e % BS, c = e / BS;
        s[i * ld + c] = g[e];
    }
}
template <int BS>
__device__ void store_blk(cplx *__restrict__ g, const cplx *s, int ld, double sign) {
    for (int e = threadIdx.x; e < BS * BS; e += blockDim.x) {
        const int i = e % BS, c = e / BS;
        g[e] = cscale(s[i * ld + c], sign);
    }
}
// C (stride ldc) = A (stride lda) * B (stride ldb), all BS x BS in smem.
template <int BS>
__device__ void mul_blk(cplx *C, int ldc, const cplx *A, int lda, const cplx *B, int ldb) {
    for (int e = threadIdx.x; e < BS * BS; e += blockDim.x) {
        const int i = e % BS, c = e / BS;
        cplx acc = mk(0.0, 0.0);
#pragma unroll 8
        for (int j = 0; j < BS; ++j) cfma(acc, A[i * lda + j], B[j * ldb + c]);
        C[i * ldc + c] = acc;
    }
}
// C -= A * B
template <int BS>
__device__ void mulsub_blk(cplx *C, int ldc, const cplx *A, int lda, const cplx *B, int ldb) {
    for (int e = threadIdx.x; e < BS * BS; e += blockDim.x) {
        const int i = e % BS, c = e / BS;
        cplx acc = C[i * ldc + c];
#pragma unroll 8
        for (int j = 0; j < BS; ++j) cfms(acc, A[i * lda + j], B[j * ldb + c]);
        C[i * ldc + c] = acc;
    }
}

// In-place Gauss-Jordan inversion of the left half of M = [A | I] (row-major,
// stride LDA), partial pivoting by rows inside the block.  On return the
// right half holds A^-1.  A zero pivot sets *err and leaves that step out.
template <int BS>
__device__ void gj_invert(cplx *M, int *err, double *minpiv) {
    constexpr int LDA = Blk<BS>::LDA;
    __shared__ int s_q;
    __shared__ cplx s_pinv;
    __shared__ cplx fcol[BS];
    for (int p = 0; p < BS; ++p) {
        if (threadIdx.x < 32) {
            const int i = threadIdx.x;
            double v = (i >= p && i < BS) ? cabs2(M[i * LDA + p]) : -1.0;
            int q = i;
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_xor_sync(0xffffffffu, v, o);
                const int oq = __shfl_xor_sync(0xffffffffu, q, o);
                if (ov > v || (ov == v && oq < q)) { v = ov; q = oq; }
            }
            if (i == 0) s_q = q;
        }
        __syncthreads();
        const int q = s_q;
        if (q != p)
            for (int c = p + threadIdx.x; c < 2 * BS; c += blockDim.x) {
                const cplx a = M[p * LDA + c];
                M[p * LDA + c] = M[q * LDA + c];
                M[q * LDA + c] = a;
            }
        __syncthreads();
        if (threadIdx.x == 0) {
            const cplx d = M[p * LDA + p];
            const double d2 = cabs2(d);
            if (d2 == 0.0) {
                atomicExch(err, 1);
                s_pinv = mk(0.0, 0.0);
            } else {
                s_pinv = mk(d.x / d2, -d.y / d2);
            }
            const double ad = sqrt(d2);
            if (minpiv && ad < *minpiv) *minpiv = ad;
        }
        for (int i = threadIdx.x; i < BS; i += blockDim.x) fcol[i] = M[i * LDA + p];
        __syncthreads();
        const cplx pinv = s_pinv;
        for (int c = p + threadIdx.x; c < 2 * BS; c += blockDim.x) M[p * LDA + c] = cmul(M[p * LDA + c], pinv);
        __syncthreads();
        const int w = 2 * BS - p;
        for (int e = threadIdx.x; e < BS * w; e += blockDim.x) {
            const int i = e / w, c = p + e % w;
            if (i == p) continue;
            cfms(M[i * LDA + c], fcol[i], M[p * LDA + c]);
        }
        __syncthreads();
    }
}

template <int BS>
__device__ void load_aug(cplx *M, const cplx *__restrict__ g) {
    constexpr int LDA = Blk<BS>::LDA;
    for (int e = threadIdx.x; e < BS * BS; e += blockDim.x) {
        const int i = e % BS, c = e / BS;
        M[i * LDA + c] = g[e];
        M[i * LDA + BS + c] = mk(i == c ? 1.0 : 0.0, 0.0);
    }
    __syncthreads();
}

// Dg = Ad - sigma Bd for every block.
__global__ void k_shift(int64_t count, const cplx *__restrict__ Ad, const cplx *__restrict__ Bd,
                        cplx sigma, cplx *__restrict__ Dg) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
        cplx v = Ad[i];
        cfms(v, sigma, Bd[i]);
        Dg[i] = v;
    }
}

// Plain inversion of `count` blocks (block Jacobi and the BCR top block).
template <int BS>
__global__ void __launch_bounds__(256) k_invert_blocks(int64_t count, const cplx *__restrict__ D,
                                                       cplx *__restrict__ Dinv, int *err,
                                                       double *minpiv) {
    extern __shared__ cplx smem[];
    cplx *M = smem;
    constexpr int BB = BS * BS, LDA = Blk<BS>::LDA;
    for (int64_t blk = blockIdx.x; blk < count; blk += gridDim.x) {
        load_aug<BS>(M, D + blk * BB);
        gj_invert<BS>(M, err, blockIdx.x == 0 ? minpiv : nullptr);
        store_blk<BS>(Dinv + blk * BB, M + BS, LDA, 1.0);
        __syncthreads();
    }
}

// BCR level, odd blocks m = 2i+1: Dinv, Dinv Lo_m, Dinv Up_m.
template <int BS>
__global__ void __launch_bounds__(256) k_bcr_odd(int64_t N, const cplx *__restrict__ Dg,
                                                 const cplx *__restrict__ Lo,
                                                 const cplx *__restrict__ Up, cplx *Dinv,
                                                 cplx *DinvLo, cplx *DinvUp, int *err) {
    extern __shared__ cplx smem[];
    constexpr int BB = BS * BS, LD = Blk<BS>::LD, LDA = Blk<BS>::LDA;
    cplx *M = smem;                    // BS x LDA
    cplx *T = smem + BS * LDA;         // BS x LD
    cplx *C = T + BS * LD;             // BS x LD
    const int64_t nodd = N / 2;
    for (int64_t i = blockIdx.x; i < nodd; i += gridDim.x) {
        const int64_t m = 2 * i + 1;
        load_aug<BS>(M, Dg + m * BB);
        gj_invert<BS>(M, err, nullptr);
        store_blk<BS>(Dinv + i * BB, M + BS, LDA, 1.0);
        load_blk<BS>(T, LD, Lo + m * BB);
        __syncthreads();
        mul_blk<BS>(C, LD, M + BS, LDA, T, LD);
        __syncthreads();
        store_blk<BS>(DinvLo + i * BB, C, LD, 1.0);
        load_blk<BS>(T, LD, Up + m * BB);
        __syncthreads();
        mul_blk<BS>(C, LD, M + BS, LDA, T, LD);
        __syncthreads();
        store_blk<BS>(DinvUp + i * BB, C, LD, 1.0);
        __syncthreads();
    }
}

// BCR level, even blocks m = 2i: multipliers and the next level's blocks
//   Alpha = Lo_m Dinv_{m-1},  Beta = Up_m Dinv_{m+1}
//   Dg'   = Dg_m - Lo_m DinvUp_{m-1} - Up_m DinvLo_{m+1}
//   Lo'   = -Lo_m DinvLo_{m-1},  Up' = -Up_m DinvUp_{m+1}
template <int BS>
__global__ void __launch_bounds__(256) k_bcr_even(
    int64_t N, const cplx *__restrict__ Dg, const cplx *__restrict__ Lo,
    const cplx *__restrict__ Up, const cplx *__restrict__ Dinv, const cplx *__restrict__ DinvLo,
    const cplx *__restrict__ DinvUp, cplx *Alpha, cplx *Beta, cplx *Dg2, cplx *Lo2, cplx *Up2) {
    extern __shared__ cplx smem[];
    constexpr int BB = BS * BS, LD = Blk<BS>::LD;
    cplx *Ls = smem, *Us = Ls + BS * LD, *Acc = Us + BS * LD, *Nb = Acc + BS * LD, *C = Nb + BS * LD;
    const int64_t neven = (N + 1) / 2;
    for (int64_t i = blockIdx.x; i < neven; i += gridDim.x) {
        const int64_t m = 2 * i;
        const bool has_prev = m >= 1, has_next = m + 1 < N;
        load_blk<BS>(Acc, LD, Dg + m * BB);
        load_blk<BS>(Ls, LD, Lo + m * BB);
        load_blk<BS>(Us, LD, Up + m * BB);
        __syncthreads();
        if (has_prev) {
            const int64_t io = (m - 1) / 2;  // odd index of m-1
            load_blk<BS>(Nb, LD, Dinv + io * BB);
            __syncthreads();
            mul_blk<BS>(C, LD, Ls, LD, Nb, LD);
            __syncthreads();
            store_blk<BS>(Alpha + i * BB, C, LD, 1.0);
            load_blk<BS>(Nb, LD, DinvUp + io * BB);
            __syncthreads();
            mulsub_blk<BS>(Acc, LD, Ls, LD, Nb, LD);
            __syncthreads();
            load_blk<BS>(Nb, LD, DinvLo + io * BB);
            __syncthreads();
            mul_blk<BS>(C, LD, Ls, LD, Nb, LD);
            __syncthreads();
            store_blk<BS>(Lo2 + i * BB, C, LD, -1.0);
        } else {
            for (int e = threadIdx.x; e < BB; e += blockDim.x) {
                Alpha[i * BB + e] = mk(0.0, 0.0);
                Lo2[i * BB + e] = mk(0.0, 0.0);
            }
        }
        __syncthreads();
        if (has_next) {
            const int64_t io = m / 2;  // odd index of m+1
            load_blk<BS>(Nb, LD, Dinv + io * BB);
            __syncthreads();
            mul_blk<BS>(C, LD, Us, LD, Nb, LD);
            __syncthreads();
            store_blk<BS>(Beta + i * BB, C, LD, 1.0);
            load_blk<BS>(Nb, LD, DinvLo + io * BB);
            __syncthreads();
            mulsub_blk<BS>(Acc, LD, Us, LD, Nb, LD);
            __syncthreads();
            load_blk<BS>(Nb, LD, DinvUp + io * BB);
            __syncthreads();
            mul_blk<BS>(C, LD, Us, LD, Nb, LD);
            __syncthreads();
            store_blk<BS>(Up2 + i * BB, C, LD, -1.0);
        } else {
            for (int e = threadIdx.x; e < BB; e += blockDim.x) {
                Beta[i * BB + e] = mk(0.0, 0.0);
                Up2[i * BB + e] = mk(0.0, 0.0);
            }
        }
        __syncthreads();
        store_blk<BS>(Dg2 + i * BB, Acc, LD, 1.0);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Solve kernels: a warp owns 32/BS blocks; lane = row; R right-hand sides
// stored with a stride.  y_row += M v with v spread over the block's lanes.
template <int BS, int R, typename T>
__device__ __forceinline__ void bmv_add(cplx (&acc)[R], const T *__restrict__ Mb, int row,
                                        const cplx (&v)[R], int base, double sign) {
#pragma unroll 16
    for (int c = 0; c < BS; ++c) {
        const cplx mv = ldm(Mb + c * BS + row);
#pragma unroll
        for (int q = 0; q < R; ++q) {
            const cplx vc = shfl(v[q], base + c);
            if (sign > 0) cfma(acc[q], mv, vc);
            else cfms(acc[q], mv, vc);
        }
    }
}

// rhs_next[m/2] = rhs[m] - Alpha rhs[m-1] - Beta rhs[m+1] for even m.
template <int BS, int R, typename T>
__global__ void __launch_bounds__(256, 2) k_bcr_fwd(int64_t N, const T *__restrict__ Alpha,
                                                 const T *__restrict__ Beta,
                                                 const cplx *__restrict__ rhs, int64_t rs,
                                                 cplx *__restrict__ nxt, int64_t ns) {
    constexpr int BPW = 32 / BS, BB = BS * BS;
    const int lane = threadIdx.x & 31, hw = lane / BS, row = lane - hw * BS, base = hw * BS;
    const int64_t neven = (N + 1) / 2;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t g = gw; g * BPW < neven; g += nw) {
        const int64_t i = g * BPW + hw;
        const bool valid = i < neven;
        const int64_t ic = valid ? i : neven - 1;
        const int64_t m = 2 * ic;
        cplx acc[R], vp[R], vn[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
            acc[q] = rhs[q * rs + m * BS + row];
            vp[q] = m >= 1 ? rhs[q * rs + (m - 1) * BS + row] : mk(0.0, 0.0);
            vn[q] = m + 1 < N ? rhs[q * rs + (m + 1) * BS + row] : mk(0.0, 0.0);
        }
        bmv_add<BS, R, T>(acc, Alpha + ic * BB, row, vp, base, -1.0);
        bmv_add<BS, R, T>(acc, Beta + ic * BB, row, vn, base, -1.0);
        if (valid)
#pragma unroll
            for (int q = 0; q < R; ++q) nxt[q * ns + i * BS + row] = acc[q];
    }
}

// x = Dinv rhs for a single block (top of the reduction).
template <int BS, int R, typename T>
__global__ void k_bcr_top(const T *__restrict__ Dinv, const cplx *__restrict__ rhs, int64_t rs,
                          cplx *__restrict__ x, int64_t xs) {
    const int lane = threadIdx.x & 31, row = lane % BS, base = 0;
    const bool active = lane < BS;
    cplx acc[R], v[R];
#pragma unroll
    for (int q = 0; q < R; ++q) {
        acc[q] = mk(0.0, 0.0);
        v[q] = active ? rhs[q * rs + row] : mk(0.0, 0.0);
    }
    bmv_add<BS, R, T>(acc, Dinv, row, v, base, 1.0);
    if (active)
#pragma unroll
        for (int q = 0; q < R; ++q) x[q * xs + row] = acc[q];
}

// Back substitution of one level: even m copy from the level above,
// odd m: x = Dinv rhs - DinvLo x[m-1] - DinvUp x[m+1].
template <int BS, int R, typename T>
__global__ void __launch_bounds__(256, 2) k_bcr_bwd(int64_t N, const T *__restrict__ Dinv,
                                                 const T *__restrict__ DinvLo,
                                                 const T *__restrict__ DinvUp,
                                                 const cplx *__restrict__ rhs, int64_t rs,
                                                 const cplx *__restrict__ xup, int64_t us,
                                                 cplx *__restrict__ x, int64_t xs) {
    constexpr int BPW = 32 / BS, BB = BS * BS;
    const int lane = threadIdx.x & 31, hw = lane / BS, row = lane - hw * BS, base = hw * BS;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t nodd = N / 2;
    // even blocks: plain copy
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < ((N + 1) / 2) * BS;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t ie = e / BS, rr = e - ie * BS;
#pragma unroll
        for (int q = 0; q < R; ++q) x[q * xs + (2 * ie) * BS + rr] = xup[q * us + ie * BS + rr];
    }
    for (int64_t g = gw; g * BPW < nodd; g += nw) {
        const int64_t i = g * BPW + hw;
        const bool valid = i < nodd;
        const int64_t ic = valid ? i : nodd - 1;
        const int64_t m = 2 * ic + 1;
        cplx acc[R], r[R], vp[R], vn[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
            acc[q] = mk(0.0, 0.0);
            r[q] = rhs[q * rs + m * BS + row];
            vp[q] = xup[q * us + ic * BS + row];                                  // x[m-1]
            vn[q] = m + 1 < N ? xup[q * us + (ic + 1) * BS + row] : mk(0.0, 0.0);  // x[m+1]
        }
        bmv_add<BS, R, T>(acc, Dinv + ic * BB, row, r, base, 1.0);
        bmv_add<BS, R, T>(acc, DinvLo + ic * BB, row, vp, base, -1.0);
        bmv_add<BS, R, T>(acc, DinvUp + ic * BB, row, vn, base, -1.0);
        if (valid)
#pragma unroll
            for (int q = 0; q < R; ++q) x[q * xs + m * BS + row] = acc[q];
    }
}

// Small levels: one CTA per block.  The BS columns of each b x b block are
// split over NS = 256/BS column slots (slot = 8 warps x 32/BS lane groups),
// so each thread's chain of dependent loads is BS^2/256 columns long instead
// of BS; the slots' partial sums meet in shared memory.  Used when a level
// has too few blocks to fill the GPU with one warp per block.
template <int BS, int R, typename T>
__device__ __forceinline__ void slot_mv(cplx (&acc)[R], const T *__restrict__ Mb, int row, int c0,
                                        int nc, const cplx (&v)[R], int base, double sign) {
    for (int c = c0; c < c0 + nc; ++c) {
        const cplx mv = ldm(Mb + c * BS + row);
#pragma unroll
        for (int q = 0; q < R; ++q) {
            const cplx vc = shfl(v[q], base + c);
            if (sign > 0) cfma(acc[q], mv, vc);
            else cfms(acc[q], mv, vc);
        }
    }
}

template <int BS, int R, typename T>
__global__ void __launch_bounds__(256) k_bcr_fwd_cta(int64_t N, const T *__restrict__ Alpha,
                                                     const T *__restrict__ Beta,
                                                     const cplx *__restrict__ rhs, int64_t rs,
                                                     cplx *__restrict__ nxt, int64_t ns) {
    constexpr int BB = BS * BS, GPW = 32 / BS, NS = 8 * GPW, CPS = BS / NS;
    __shared__ cplx red[NS][R][BS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int grp = lane / BS, row = lane - grp * BS, base = grp * BS;
    const int slot = warp * GPW + grp, c0 = slot * CPS;
    const int64_t neven = (N + 1) / 2;
    for (int64_t i = blockIdx.x; i < neven; i += gridDim.x) {
        const int64_t m = 2 * i;
        cplx acc[R], vp[R], vn[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
            acc[q] = mk(0.0, 0.0);
            vp[q] = m >= 1 ? rhs[q * rs + (m - 1) * BS + row] : mk(0.0, 0.0);
            vn[q] = m + 1 < N ? rhs[q * rs + (m + 1) * BS + row] : mk(0.0, 0.0);
        }
        slot_mv<BS, R, T>(acc, Alpha + i * BB, row, c0, CPS, vp, base, -1.0);
        slot_mv<BS, R, T>(acc, Beta + i * BB, row, c0, CPS, vn, base, -1.0);
#pragma unroll
        for (int q = 0; q < R; ++q) red[slot][q][row] = acc[q];
        __syncthreads();
        for (int e = threadIdx.x; e < R * BS; e += blockDim.x) {
            const int q = e / BS, rr = e - q * BS;
            cplx s = rhs[q * rs + m * BS + rr];
            for (int k = 0; k < NS; ++k) s = cadd(s, red[k][q][rr]);
            nxt[q * ns + i * BS + rr] = s;
        }
        __syncthreads();
    }
}

template <int BS, int R, typename T>
__global__ void __launch_bounds__(256) k_bcr_bwd_cta(int64_t N, const T *__restrict__ Dinv,
                                                     const T *__restrict__ DinvLo,
                                                     const T *__restrict__ DinvUp,
                                                     const cplx *__restrict__ rhs, int64_t rs,
                                                     const cplx *__restrict__ xup, int64_t us,
                                                     cplx *__restrict__ x, int64_t xs) {
    constexpr int BB = BS * BS, GPW = 32 / BS, NS = 8 * GPW, CPS = BS / NS;
    __shared__ cplx red[NS][R][BS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int grp = lane / BS, row = lane - grp * BS, base = grp * BS;
    const int slot = warp * GPW + grp, c0 = slot * CPS;
    const int64_t nodd = N / 2, neven = (N + 1) / 2;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < neven * BS;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t ie = e / BS, rr = e - ie * BS;
#pragma unroll
        for (int q = 0; q < R; ++q) x[q * xs + (2 * ie) * BS + rr] = xup[q * us + ie * BS + rr];
    }
    for (int64_t i = blockIdx.x; i < nodd; i += gridDim.x) {
        const int64_t m = 2 * i + 1;
        cplx acc[R], r[R], vp[R], vn[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
            acc[q] = mk(0.0, 0.0);
            r[q] = rhs[q * rs + m * BS + row];
            vp[q] = xup[q * us + i * BS + row];
            vn[q] = m + 1 < N ? xup[q * us + (i + 1) * BS + row] : mk(0.0, 0.0);
        }
        slot_mv<BS, R, T>(acc, Dinv + i * BB, row, c0, CPS, r, base, 1.0);
        slot_mv<BS, R, T>(acc, DinvLo + i * BB, row, c0, CPS, vp, base, -1.0);
        slot_mv<BS, R, T>(acc, DinvUp + i * BB, row, c0, CPS, vn, base, -1.0);
#pragma unroll
        for (int q = 0; q < R; ++q) red[slot][q][row] = acc[q];
        __syncthreads();
        for (int e = threadIdx.x; e < R * BS; e += blockDim.x) {
            const int q = e / BS, rr = e - q * BS;
            cplx s = red[0][q][rr];
            for (int k = 1; k < NS; ++k) s = cadd(s, red[k][q][rr]);
            x[q * xs + m * BS + rr] = s;
        }
        __syncthreads();
    }
}

// The reduced system's dense inverse applied to R right-hand sides, in two
// deterministic stages: part[c][q][i] = sum over the c-th chunk of columns j
// of Minv[i, j] rhs[q][j] (a thread per row i, the column-major Minv read
// coalesced), then x[q][i] = sum over c of part[c][q][i] in chunk order.
constexpr int MV_CHUNKS = 48;
template <int R>
__global__ void __launch_bounds__(256) k_dense_mv(int64_t m, const cplx *__restrict__ M,
                                                  const cplx *__restrict__ rhs, int64_t rs,
                                                  cplx *__restrict__ part) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t cc = (m + gridDim.y - 1) / gridDim.y;
    const int64_t j0 = (int64_t)blockIdx.y * cc, j1 = min(m, j0 + cc);
    if (i >= m) return;
    cplx acc[R];
#pragma unroll
    for (int q = 0; q < R; ++q) acc[q] = mk(0.0, 0.0);
    for (int64_t j = j0; j < j1; ++j) {
        const cplx a = ldg_stream(M + j * m + i);
#pragma unroll
        for (int q = 0; q < R; ++q) cfma(acc[q], a, __ldg(rhs + q * rs + j));
    }
#pragma unroll
    for (int q = 0; q < R; ++q) part[((int64_t)blockIdx.y * R + q) * m + i] = acc[q];
}

template <int R>
__global__ void __launch_bounds__(256) k_dense_mv_sum(int64_t m, int chunks, const cplx *__restrict__ part,
                                                      cplx *__restrict__ x, int64_t xs) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= R * m) return;
    const int q = (int)(e / m);
    const int64_t i = e - q * m;
    cplx s = mk(0.0, 0.0);
    for (int c = 0; c < chunks; ++c) s = cadd(s, part[((int64_t)c * R + q) * m + i]);
    x[q * xs + i] = s;
}

// Two right-hand sides of the reduced system at unit vectors: rhs[q] =
// e_(i0 + q) (zero when i0 + q = m), stride rs.
__global__ void k_unit_pair(int64_t m, int64_t i0, cplx *__restrict__ rhs, int64_t rs) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < 2 * m;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int q = (int)(e / m);
        const int64_t j = e - q * m;
        rhs[q * rs + j] = mk(j == i0 + q ? 1.0 : 0.0, 0.0);
    }
}

// Block-Jacobi apply: x_j = Dinv_j r_j for every interior block.
template <int BS, int R, typename T>
__global__ void __launch_bounds__(256) k_bjac(int64_t nblk, const T *__restrict__ Dinv,
                                              const cplx *__restrict__ r, int64_t rs,
                                              cplx *__restrict__ x, int64_t xs) {
    constexpr int BPW = 32 / BS, BB = BS * BS;
    const int lane = threadIdx.x & 31, hw = lane / BS, row = lane - hw * BS, base = hw * BS;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t g = gw; g * BPW < nblk; g += nw) {
        const int64_t j = g * BPW + hw;
        const bool valid = j < nblk;
        const int64_t jc = valid ? j : nblk - 1;
        cplx acc[R], v[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
            acc[q] = mk(0.0, 0.0);
            v[q] = r[q * rs + jc * BS + row];
        }
        bmv_add<BS, R, T>(acc, Dinv + jc * BB, row, v, base, 1.0);
        if (valid)
#pragma unroll
            for (int q = 0; q < R; ++q) x[q * xs + j * BS + row] = acc[q];
    }
}

// Border step 1: per-CTA partials of F1 y (t-vector per RHS); lane owns tau
// rows lane + 32 u (u < NQ).
template <int R, int NQ, typename T>
__global__ void __launch_bounds__(256) k_border_g(int64_t nb, int t, const T *__restrict__ FT,
                                                  const cplx *__restrict__ y, int64_t ys,
                                                  cplx *__restrict__ part) {
    extern __shared__ cplx wsm[];  // 8 warps x R x t
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    cplx acc[R][NQ];
#pragma unroll
    for (int q = 0; q < R; ++q)
#pragma unroll
        for (int u = 0; u < NQ; ++u) acc[q][u] = mk(0.0, 0.0);
    const int64_t ngroups = (nb + 31) / 32;
    const int64_t gw = (int64_t)blockIdx.x * 8 + warp, nw = (int64_t)gridDim.x * 8;
    for (int64_t g = gw; g < ngroups; g += nw) {
        const int64_t col = g * 32 + lane;
        cplx yv[R];
#pragma unroll
        for (int q = 0; q < R; ++q) yv[q] = col < nb ? y[q * ys + col] : mk(0.0, 0.0);
#pragma unroll 8
        for (int c = 0; c < 32; ++c) {
            const int64_t cc = min(g * 32 + c, nb - 1);
            cplx yc[R];
#pragma unroll
            for (int q = 0; q < R; ++q) yc[q] = shfl(yv[q], c);
#pragma unroll
            for (int u = 0; u < NQ; ++u) {
                const int tau = lane + 32 * u;
                if (tau < t) {
                    const cplx f = ldm(FT + cc * t + tau);
#pragma unroll
                    for (int q = 0; q < R; ++q) cfma(acc[q][u], f, yc[q]);
                }
            }
        }
    }
#pragma unroll
    for (int q = 0; q < R; ++q)
#pragma unroll
        for (int u = 0; u < NQ; ++u) {
            const int tau = lane + 32 * u;
            if (tau < t) wsm[(warp * R + q) * t + tau] = acc[q][u];
        }
    __syncthreads();
    for (int e = threadIdx.x; e < R * t; e += blockDim.x) {
        const int q = e / t, tau = e - q * t;
        cplx s = wsm[q * t + tau];
        for (int w = 1; w < 8; ++w) s = cadd(s, wsm[(w * R + q) * t + tau]);
        part[((int64_t)blockIdx.x * R + q) * t + tau] = s;
    }
}

// Border step 2a: g[q][tau] = r2[q][tau] - sum_g part[g][q][tau], one warp
// per (q, tau), lanes over the CTA partials (fixed order).
template <int R>
__global__ void __launch_bounds__(256) k_border_gsum(int64_t nb, int t, int G,
                                                     const cplx *__restrict__ part,
                                                     const cplx *__restrict__ rin, int64_t rs,
                                                     cplx *__restrict__ gbuf) {
    const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (w >= R * t) return;
    const int q = w / t, tau = w - q * t;
    cplx s = mk(0.0, 0.0);
    for (int k = lane; k < G; k += 32) s = cadd(s, part[((int64_t)k * R + q) * t + tau]);
    s = warp_sum(s);
    if (lane == 0) gbuf[q * t + tau] = csub(rin[q * rs + nb + tau], s);
}

// Border step 2b: x2 = Sinv g; written to out[nb:] and x2buf.
template <int R>
__global__ void __launch_bounds__(256) k_border_x2(int64_t nb, int t, const cplx *__restrict__ gbuf,
                                                   const cplx *__restrict__ Sinv,
                                                   cplx *__restrict__ out, int64_t os,
                                                   cplx *__restrict__ x2buf) {
    __shared__ cplx g[R][128];
    for (int e = threadIdx.x; e < R * t; e += blockDim.x) g[e / t][e % t] = gbuf[e];
    __syncthreads();
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= R * t) return;
    const int q = e / t, tau = e - q * t;
    cplx acc = mk(0.0, 0.0);
#pragma unroll 8
    for (int c = 0; c < t; ++c) cfma(acc, Sinv[(int64_t)c * t + tau], g[q][c]);
    out[q * os + nb + tau] = acc;
    x2buf[q * t + tau] = acc;
}

// Border step 3: x1 = y - Y x2 (in place in out[0:nb]).
template <int R, typename T>
__global__ void __launch_bounds__(256) k_border_x1(int64_t nb, int t, const T *__restrict__ Y,
                                                   const cplx *__restrict__ x2buf,
                                                   cplx *__restrict__ out, int64_t os) {
    __shared__ cplx xs[R][128];
    for (int e = threadIdx.x; e < R * t; e += blockDim.x) xs[e / t][e % t] = x2buf[e];
    __syncthreads();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += stride) {
        cplx acc[R];
#pragma unroll
        for (int q = 0; q < R; ++q) acc[q] = out[q * os + i];
#pragma unroll 8
        for (int tau = 0; tau < t; ++tau) {
            const cplx yv = ldm(Y + (int64_t)tau * nb + i);
#pragma unroll
            for (int q = 0; q < R; ++q) cfms(acc[q], yv, xs[q][tau]);
        }
#pragma unroll
        for (int q = 0; q < R; ++q) out[q * os + i] = acc[q];
    }
}

// Tau corner for block Jacobi: x2 = Ginv r2.
template <int R>
__global__ void k_corner(int64_t nb, int t, const cplx *__restrict__ Ginv,
                         const cplx *__restrict__ r, int64_t rs, cplx *__restrict__ x, int64_t xs) {
    for (int e = threadIdx.x; e < R * t; e += blockDim.x) {
        const int q = e / t, tau = e - q * t;
        cplx acc = mk(0.0, 0.0);
        for (int c = 0; c < t; ++c) cfma(acc, Ginv[(int64_t)c * t + tau], r[q * rs + nb + c]);
        x[q * xs + nb + tau] = acc;
    }
}

// S partial: part[g] (t x t col-major) = sum over the CTA's rows of F1[:, i] Y[i, :].
__global__ void __launch_bounds__(256) k_schur_part(int64_t nb, int t, const cplx *__restrict__ FT,
                                                    const cplx *__restrict__ Y, int64_t rpc,
                                                    cplx *__restrict__ part) {
    __shared__ cplx sF[8][128];
    __shared__ cplx sY[8][128];
    const int64_t r0 = (int64_t)blockIdx.x * rpc, r1 = min(nb, r0 + rpc);
    const int npairs = t * t;
    cplx acc[64];
    const int per = (npairs + blockDim.x - 1) / blockDim.x;  // <= 64 for t <= 128
#pragma unroll
    for (int u = 0; u < 64; ++u) acc[u] = mk(0.0, 0.0);
    for (int64_t rs = r0; rs < r1; rs += 8) {
        for (int e = threadIdx.x; e < 8 * t; e += blockDim.x) {
            const int rr = e / t, c = e - rr * t;
            const int64_t row = rs + rr;
            const bool ok = row < r1;
            sF[rr][c] = ok ? FT[row * t + c] : mk(0.0, 0.0);
            sY[rr][c] = ok ? Y[(int64_t)c * nb + row] : mk(0.0, 0.0);
        }
        __syncthreads();
        for (int u = 0; u < per && u < 64; ++u) {
            const int pidx = threadIdx.x + u * blockDim.x;
            if (pidx >= npairs) break;
            const int a = pidx % t, bcol = pidx / t;
            cplx s = acc[u];
            for (int rr = 0; rr < 8; ++rr) cfma(s, sF[rr][a], sY[rr][bcol]);
            acc[u] = s;
        }
        __syncthreads();
    }
    for (int u = 0; u < per && u < 64; ++u) {
        const int pidx = threadIdx.x + u * blockDim.x;
        if (pidx >= npairs) break;
        part[(int64_t)blockIdx.x * npairs + pidx] = acc[u];
    }
}

// ---------------------------------------------------------------------------
template <int BS>
static size_t odd_smem() { return sizeof(cplx) * (BS * Blk<BS>::LDA + 2 * BS * Blk<BS>::LD); }
template <int BS>
static size_t even_smem() { return sizeof(cplx) * 5 * BS * Blk<BS>::LD; }
template <int BS>
static size_t inv_smem() { return sizeof(cplx) * BS * Blk<BS>::LDA; }

template <int BS>
static bbjd_status set_attrs() {
    bbjd_status s;
    if ((s = raise_smem_limit((const void *)k_bcr_odd<BS>, odd_smem<BS>()))) return s;
    if ((s = raise_smem_limit((const void *)k_bcr_even<BS>, even_smem<BS>()))) return s;
    return raise_smem_limit((const void *)k_invert_blocks<BS>, inv_smem<BS>());
}

// Levels with at most this many blocks to process run one CTA per block.
constexpr int64_t kSmallLevel = 2048;

static unsigned grid_for(int64_t items, int per_cta, int cap);

// CTA-per-block launches exist for b >= 16 (b = 8 blocks are too small to split).
template <int BS, int R, typename T>
static bool fwd_cta(int64_t N, int64_t items, const T *Alpha, const T *Beta, const cplx *rhs,
                    int64_t rs, cplx *nxt, int64_t ns, int cap, cudaStream_t st) {
    if constexpr (BS >= 16) {
        if (items > kSmallLevel) return false;
        k_bcr_fwd_cta<BS, R, T><<<grid_for(items, 1, cap), 256, 0, st>>>(N, Alpha, Beta, rhs, rs, nxt, ns);
        return true;
    } else {
        return false;
    }
}
template <int BS, int R, typename T>
static bool bwd_cta(int64_t N, int64_t items, const T *Dinv, const T *DinvLo, const T *DinvUp,
                    const cplx *rhs, int64_t rs, const cplx *xup, int64_t us, cplx *x, int64_t xs,
                    int cap, cudaStream_t st) {
    if constexpr (BS >= 16) {
        if (items > kSmallLevel) return false;
        k_bcr_bwd_cta<BS, R, T><<<grid_for(std::max<int64_t>(items, 1), 1, cap), 256, 0, st>>>(
            N, Dinv, DinvLo, DinvUp, rhs, rs, xup, us, x, xs);
        return true;
    } else {
        return false;
    }
}

static unsigned grid_for(int64_t items, int per_cta, int cap) {
    int64_t g = (items + per_cta - 1) / per_cta;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (unsigned)g;
}

// Factor array of type T: the FP64 pool, or its complex64 copy at the same
// element offset (mixed precision; the FP64 pool is released after the copy).
template <typename T>
static const T *fac(const bbjd_precond *pc, const cplx *p64) {
    if constexpr (std::is_same<T, float2>::value)
        return pc->pool32 + (p64 - pc->pool_base);
    else
        return p64;
}

// Solve K x = r for the interior with R right-hand sides (input stride rs,
// output stride xs).  x may alias r.  T: factor element type.  From level
// `start` > 0 the right-hand sides are already in that level's buffer and
// the solution is left in its x buffer (the factorisation uses this to
// form Minv).  With use_cut, the levels from pc->cut on and the top block
// are replaced by the reduced system's dense inverse.
template <int BS, int R, typename T = cplx>
static bbjd_status bcr_solve(const bbjd_precond *pc, const cplx *r, int64_t rs, cplx *x, int64_t xs,
                             cudaStream_t st, int64_t start = 0, bool use_cut = true) {
    // Vectors: level 0 is the caller's r / x; level l >= 1 and the top block
    // live in lvl_rhs / lvl_x at levels[l].vec_off / top_off, per-RHS stride
    // lvl_total.
    const int cap = 16 * num_sms();
    const int64_t L = (int64_t)pc->levels.size();
    const int64_t tot = pc->lvl_total;
    const bool cut = use_cut && pc->Minv && pc->cut > start;
    const int64_t stop = cut ? pc->cut : L;          // forward levels [start, stop)
    auto rhs_at = [&](int64_t l) -> const cplx * {
        return l == 0 ? r : (l < L ? pc->lvl_rhs + pc->levels[l].vec_off : pc->lvl_rhs + pc->top_off);
    };
    auto rstride = [&](int64_t l) -> int64_t { return l == 0 ? rs : tot; };
    for (int64_t l = start; l < stop; ++l) {
        const auto &lv = pc->levels[l];
        cplx *nxt = (l + 1 < L) ? pc->lvl_rhs + pc->levels[l + 1].vec_off : pc->lvl_rhs + pc->top_off;
        const T *Alpha = fac<T>(pc, lv.Alpha), *Beta = fac<T>(pc, lv.Beta);
        if (!fwd_cta<BS, R, T>(lv.N, lv.n_even, Alpha, Beta, rhs_at(l), rstride(l), nxt, tot, cap, st)) {
            const int64_t items = (lv.n_even + (32 / BS) - 1) / (32 / BS);
            k_bcr_fwd<BS, R, T><<<grid_for(items, 8, cap), 256, 0, st>>>(lv.N, Alpha, Beta, rhs_at(l),
                                                                        rstride(l), nxt, tot);
        }
        BBJD_LAUNCH_CHECK();
    }
    if (cut) {
        const int64_t m = pc->mcut;
        cplx *xc = pc->lvl_x + pc->levels[pc->cut].vec_off;
        k_dense_mv<R><<<dim3((unsigned)((m + 255) / 256), MV_CHUNKS), 256, 0, st>>>(
            m, pc->Minv, rhs_at(pc->cut), tot, pc->mpart);
        BBJD_LAUNCH_CHECK();
        k_dense_mv_sum<R><<<(unsigned)((R * m + 255) / 256), 256, 0, st>>>(m, MV_CHUNKS, pc->mpart, xc, tot);
        BBJD_LAUNCH_CHECK();
    } else {
        cplx *tx = L ? pc->lvl_x + pc->top_off : x;
        const int64_t txs = L ? tot : xs;
        k_bcr_top<BS, R, T><<<1, 32, 0, st>>>(fac<T>(pc, pc->Dinv_top), rhs_at(L), rstride(L), tx, txs);
        BBJD_LAUNCH_CHECK();
    }
    for (int64_t l = stop - 1; l >= start; --l) {
        const auto &lv = pc->levels[l];
        const cplx *xup = (l + 1 < L) ? pc->lvl_x + pc->levels[l + 1].vec_off : pc->lvl_x + pc->top_off;
        cplx *xo = l == 0 ? x : pc->lvl_x + lv.vec_off;
        const int64_t xos = l == 0 ? xs : tot;
        const T *Dinv = fac<T>(pc, lv.Dinv), *DinvLo = fac<T>(pc, lv.DinvLo);
        const T *DinvUp = fac<T>(pc, lv.DinvUp);
        if (!bwd_cta<BS, R, T>(lv.N, lv.n_odd, Dinv, DinvLo, DinvUp, rhs_at(l), rstride(l), xup, tot, xo,
                               xos, cap, st)) {
            const int64_t items = std::max<int64_t>((lv.n_odd + (32 / BS) - 1) / (32 / BS),
                                                    (lv.n_even * BS + 255) / 256);
            k_bcr_bwd<BS, R, T><<<grid_for(items, 8, cap), 256, 0, st>>>(lv.N, Dinv, DinvLo, DinvUp,
                                                                        rhs_at(l), rstride(l), xup, tot,
                                                                        xo, xos);
        }
        BBJD_LAUNCH_CHECK();
    }
    return BBJD_SUCCESS;
}

template <int BS, int R, typename T>
static bbjd_status precond_apply(const bbjd_precond *pc, const cplx *r, cplx *x, int64_t stride,
                                 cudaStream_t st) {
    const int cap = 16 * num_sms();
    if (pc->kind == BBJD_PC_BLOCK_JACOBI) {
        const int64_t items = (pc->nblk + (32 / BS) - 1) / (32 / BS);
        k_bjac<BS, R, T><<<grid_for(items, 8, cap), 256, 0, st>>>(pc->nblk, fac<T>(pc, pc->pool_base), r,
                                                                 stride, x, stride);
        BBJD_LAUNCH_CHECK();
        if (pc->t > 0) {
            k_corner<R><<<1, 256, 0, st>>>(pc->nb, pc->t, pc->Ginv, r, stride, x, stride);
            BBJD_LAUNCH_CHECK();
        }
        return BBJD_SUCCESS;
    }
    bbjd_status s = bcr_solve<BS, R, T>(pc, r, stride, x, stride, st);
    if (s != BBJD_SUCCESS || pc->t == 0) return s;
    const size_t smem = sizeof(cplx) * 8 * R * (size_t)pc->t;
    const int nq = (pc->t + 31) / 32;
    const T *FT, *Y;
    if constexpr (std::is_same<T, float2>::value) {
        FT = pc->FT32;
        Y = pc->Y32;
    } else {
        FT = pc->FT;
        Y = pc->Y;
    }
    if (nq <= 1)
        k_border_g<R, 1, T><<<pc->G, 256, smem, st>>>(pc->nb, pc->t, FT, x, stride, pc->tau_part);
    else if (nq == 2)
        k_border_g<R, 2, T><<<pc->G, 256, smem, st>>>(pc->nb, pc->t, FT, x, stride, pc->tau_part);
    else
        k_border_g<R, 4, T><<<pc->G, 256, smem, st>>>(pc->nb, pc->t, FT, x, stride, pc->tau_part);
    BBJD_LAUNCH_CHECK();
    k_border_gsum<R><<<(unsigned)((R * pc->t + 7) / 8), 256, 0, st>>>(pc->nb, pc->t, pc->G,
                                                                       pc->tau_part, r, stride, pc->gbuf);
    BBJD_LAUNCH_CHECK();
    k_border_x2<R><<<(unsigned)((R * pc->t + 255) / 256), 256, 0, st>>>(pc->nb, pc->t, pc->gbuf,
                                                                         pc->Sinv, x, stride, pc->x2);
    BBJD_LAUNCH_CHECK();
    k_border_x1<R, T><<<grid_for(pc->nb, 256, 8 * num_sms()), 256, 0, st>>>(pc->nb, pc->t, Y, pc->x2,
                                                                           x, stride);
    BBJD_LAUNCH_CHECK();
    return BBJD_SUCCESS;
}

static bbjd_status precond_launch(const bbjd_precond *pc, int nrhs, const cplx *r, cplx *x, int64_t stride,
                                  cudaStream_t st) {
    const bool c64 = pc->precision == BBJD_MIXED;
#define BBJD_PC(BS)                                                                       \
    if (pc->b == BS) {                                                                    \
        if (nrhs == 1)                                                                    \
            return c64 ? precond_apply<BS, 1, float2>(pc, r, x, stride, st)               \
                       : precond_apply<BS, 1, cplx>(pc, r, x, stride, st);                \
        if (nrhs == 2)                                                                    \
            return c64 ? precond_apply<BS, 2, float2>(pc, r, x, stride, st)               \
                       : precond_apply<BS, 2, cplx>(pc, r, x, stride, st);                \
        return BBJD_ERR_INVALID;                                                          \
    }
    BBJD_PC(8)
    BBJD_PC(16)
    BBJD_PC(32)
#undef BBJD_PC
    return BBJD_ERR_INVALID;
}

// The BCR solve through a cached CUDA graph.  The first call with a given
// (r, x, stride, nrhs, stream) launches the kernels directly and records
// the key; the second captures them (stream capture, thread-local mode) and
// every call from then on launches the instantiated graph.  Block Jacobi
// (one or two kernels), the legacy default stream and a stream the caller
// is already capturing take the direct launches.  The kernels and their
// arguments are the same either way, so the results are.
constexpr size_t PC_GRAPH_MAX = 64;
bbjd_status precond_solve(const bbjd_precond *pc_in, int nrhs, const cplx *r, cplx *x, int64_t stride,
                          cudaStream_t st) {
    auto *pc = const_cast<bbjd_precond *>(pc_in);
    if (pc->kind != BBJD_PC_BBT_LU || st == nullptr || st == cudaStreamLegacy || st == cudaStreamPerThread)
        return precond_launch(pc, nrhs, r, x, stride, st);
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        return precond_launch(pc, nrhs, r, x, stride, st);
    }
    std::lock_guard<std::mutex> lock(pc->graph_mu);
    bbjd_precond::Graph *g = nullptr;
    for (auto &e : pc->graphs)
        if (e.r == r && e.x == x && e.stride == stride && e.nrhs == nrhs && e.st == st) g = &e;
    if (g && g->exec) {
        BBJD_CUDA_TRY(cudaGraphLaunch(g->exec, st));
        count_launch(g->launches);
        return BBJD_SUCCESS;
    }
    if (!g) {
        if (pc->graphs.size() < PC_GRAPH_MAX) {
            bbjd_precond::Graph e;
            e.r = r; e.x = x; e.stride = stride; e.nrhs = nrhs; e.st = st;
            pc->graphs.push_back(e);
        }
        return precond_launch(pc, nrhs, r, x, stride, st);
    }
    // second call with this key: capture the launches, instantiate, launch
    const long long l0 = g_launches.load();
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return precond_launch(pc, nrhs, r, x, stride, st);
    }
    const bbjd_status s = precond_launch(pc, nrhs, r, x, stride, st);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &graph);
    const long long nl = g_launches.load() - l0;
    g_launches.fetch_sub(nl);            // captured, not launched
    cudaGraphExec_t exec = nullptr;
    const bool ok = s == BBJD_SUCCESS && e == cudaSuccess && graph &&
                    cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    if (!ok) {
        cudaGetLastError();
        return precond_launch(pc, nrhs, r, x, stride, st);
    }
    g->exec = exec;
    g->launches = (int)nl;
    BBJD_CUDA_TRY(cudaGraphLaunch(exec, st));
    count_launch(g->launches);
    return BBJD_SUCCESS;
}

double precond_bytes(const bbjd_precond *pc, int nrhs) {
    const double es = pc->precision == BBJD_MIXED ? 8.0 : 16.0;  // bytes per stored factor entry
    const double bb = es * pc->b * pc->b;
    double bytes = 0.0;
    if (pc->kind == BBJD_PC_BLOCK_JACOBI) {
        bytes = bb * pc->nblk + 16.0 * pc->t * pc->t;
        bytes += 2.0 * 16.0 * nrhs * pc->n;
        return bytes;
    }
    for (const auto &lv : pc->levels) {
        bytes += bb * (3.0 * lv.n_odd + 2.0 * lv.n_even);
        // forward: read 3 rhs blocks per even, write 1; backward: read rhs + 2 x, write 1
        bytes += 16.0 * nrhs * pc->b * (4.0 * lv.n_even + 4.0 * lv.n_odd + 2.0 * lv.n_even);
    }
    if (pc->Minv) {
        // the levels from `cut` on and the top block are replaced by the
        // dense inverse (read once) and its partial products
        for (size_t l = (size_t)pc->cut; l < pc->levels.size(); ++l) {
            const auto &lv = pc->levels[l];
            bytes -= bb * (3.0 * lv.n_odd + 2.0 * lv.n_even);
            bytes -= 16.0 * nrhs * pc->b * (4.0 * lv.n_even + 4.0 * lv.n_odd + 2.0 * lv.n_even);
        }
        bytes += 16.0 * (double)pc->mcut * pc->mcut + 16.0 * nrhs * pc->mcut * (2.0 * MV_CHUNKS + 2.0);
    } else {
        bytes += bb;  // top
    }
    if (pc->t > 0) {
        bytes += es * (double)pc->nb * pc->t * 2.0;          // F1 and Y
        bytes += 16.0 * nrhs * (double)pc->nb * 3.0;         // y read twice, x1 written
    }
    return bytes;
}

// Host LAPACK inverse of a small t x t matrix (column-major).
static bool host_inverse(int t, std::vector<std::complex<double>> &A,
                         std::vector<std::complex<double>> &Ainv) {
    Ainv.assign((size_t)t * t, 0.0);
    for (int i = 0; i < t; ++i) Ainv[(size_t)i * t + i] = 1.0;
    std::vector<int> ipiv(t);
    int info = 0, n = t, nrhs = t;
    scipy_zgesv_(&n, &nrhs, A.data(), &n, ipiv.data(), Ainv.data(), &n, &info);
    return info == 0;
}

template <int BS>
static bbjd_status factor_bcr(bbjd_precond *pc, const bbjd_bbt_matrix *m, cplx sigma, cudaStream_t st) {
    BBJD_CUDA_TRY(cudaMemsetAsync(pc->err, 0, sizeof(int), st));
    constexpr int64_t BB = BS * BS;
    const int cap = 8 * num_sms();
    // level sizes and the factor pool
    int64_t N = pc->nblk, pool_blocks = 1, off = 0;
    pc->levels.clear();
    while (N > 1) {
        bbjd_precond::Level lv;
        lv.N = N;
        lv.n_odd = N / 2;
        lv.n_even = (N + 1) / 2;
        lv.vec_off = pc->levels.empty() ? 0 : off;  // level 0 vectors are the caller's
        if (!pc->levels.empty()) off += N * BS;
        pool_blocks += 3 * lv.n_odd + 2 * lv.n_even;
        pc->levels.push_back(lv);
        N = lv.n_even;
    }
    pc->top_off = off;
    pc->lvl_total = off + BS;
    BBJD_CUDA_TRY(cudaMalloc(&pc->pool, sizeof(cplx) * BB * pool_blocks));
    pc->pool_elems = BB * pool_blocks;
    pc->pool_base = pc->pool;
    BBJD_CUDA_TRY(cudaMalloc(&pc->lvl_rhs, sizeof(cplx) * 2 * pc->lvl_total));
    BBJD_CUDA_TRY(cudaMalloc(&pc->lvl_x, sizeof(cplx) * 2 * pc->lvl_total));
    cplx *p = pc->pool;
    for (auto &lv : pc->levels) {
        lv.Dinv = p; p += BB * lv.n_odd;
        lv.DinvLo = p; p += BB * lv.n_odd;
        lv.DinvUp = p; p += BB * lv.n_odd;
        lv.Alpha = p; p += BB * lv.n_even;
        lv.Beta = p; p += BB * lv.n_even;
    }
    pc->Dinv_top = p;
    // transient ping-pong for the current level's Dg, Lo, Up
    cplx *T0 = nullptr, *T1 = nullptr;
    const int64_t nb0 = pc->nblk, nb1 = (pc->nblk + 1) / 2;
    BBJD_CUDA_TRY(cudaMalloc(&T0, sizeof(cplx) * BB * 3 * nb0));
    BBJD_CUDA_TRY(cudaMalloc(&T1, sizeof(cplx) * BB * 3 * std::max<int64_t>(nb1, 1)));
    k_shift<<<grid_for(BB * nb0, 256, cap), 256, 0, st>>>(BB * nb0, m->Ad, m->Bd, sigma, T0);
    BBJD_LAUNCH_CHECK();
    BBJD_CUDA_TRY(cudaMemcpyAsync(T0 + BB * nb0, m->Al, sizeof(cplx) * BB * nb0, cudaMemcpyDeviceToDevice, st));
    BBJD_CUDA_TRY(cudaMemcpyAsync(T0 + 2 * BB * nb0, m->Au, sizeof(cplx) * BB * nb0, cudaMemcpyDeviceToDevice, st));
    cplx *cur = T0, *nxt = T1;
    int64_t cap_cur = nb0, cap_nxt = std::max<int64_t>(nb1, 1);
    for (auto &lv : pc->levels) {
        const cplx *Dg = cur, *Lo = cur + BB * cap_cur, *Up = cur + 2 * BB * cap_cur;
        k_bcr_odd<BS><<<grid_for(lv.n_odd, 1, 64 * num_sms()), 256, odd_smem<BS>(), st>>>(
            lv.N, Dg, Lo, Up, lv.Dinv, lv.DinvLo, lv.DinvUp, pc->err);
        BBJD_LAUNCH_CHECK();
        cplx *Dg2 = nxt, *Lo2 = nxt + BB * cap_nxt, *Up2 = nxt + 2 * BB * cap_nxt;
        k_bcr_even<BS><<<grid_for(lv.n_even, 1, 64 * num_sms()), 256, even_smem<BS>(), st>>>(
            lv.N, Dg, Lo, Up, lv.Dinv, lv.DinvLo, lv.DinvUp, lv.Alpha, lv.Beta, Dg2, Lo2, Up2);
        BBJD_LAUNCH_CHECK();
        std::swap(cur, nxt);
        std::swap(cap_cur, cap_nxt);
    }
    k_invert_blocks<BS><<<1, 256, inv_smem<BS>(), st>>>(1, cur, pc->Dinv_top, pc->err, nullptr);
    BBJD_LAUNCH_CHECK();
    BBJD_CUDA_TRY(cudaStreamSynchronize(st));
    cudaFree(T0);
    cudaFree(T1);
    int err = 0;
    BBJD_CUDA_TRY(cudaMemcpy(&err, pc->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) return BBJD_ERR_BREAKDOWN;

    // dense inverse of the reduced system at the first level with <= 64
    // blocks (levels from there on and the top block are ~13 dependent
    // latency-bound launches per solve): column pairs by sub-solves from
    // that level on unit right-hand sides
    pc->cut = -1;
    for (int64_t l = 1; l < (int64_t)pc->levels.size(); ++l)
        if (pc->levels[l].N <= 64) {
            pc->cut = l;
            break;
        }
    if (pc->cut > 0) {
        // only where the inverse is a small part of what a solve reads (large
        // pencils: 63 MB against 2.6 GB of factors at 31,250 blocks of 32)
        double factor_bytes = 0.0;
        for (const auto &lv : pc->levels) factor_bytes += 16.0 * BB * (3.0 * lv.n_odd + 2.0 * lv.n_even);
        const double m = (double)(pc->levels[pc->cut].N * BS);
        if (16.0 * m * m > 0.05 * factor_bytes) pc->cut = -1;
    }
    if (pc->cut > 0) {
        const int64_t m = pc->levels[pc->cut].N * BS, tot = pc->lvl_total;
        pc->mcut = m;
        BBJD_CUDA_TRY(cudaMalloc(&pc->Minv, sizeof(cplx) * (size_t)m * m));
        BBJD_CUDA_TRY(cudaMalloc(&pc->mpart, sizeof(cplx) * (size_t)MV_CHUNKS * 2 * m));
        cplx *rc = pc->lvl_rhs + pc->levels[pc->cut].vec_off;
        const cplx *xc = pc->lvl_x + pc->levels[pc->cut].vec_off;
        for (int64_t i0 = 0; i0 < m; i0 += 2) {
            k_unit_pair<<<grid_for(2 * m, 256, cap), 256, 0, st>>>(m, i0, rc, tot);
            BBJD_LAUNCH_CHECK();
            bbjd_status s = bcr_solve<BS, 2>(pc, nullptr, 0, nullptr, 0, st, pc->cut, false);
            if (s != BBJD_SUCCESS) return s;
            BBJD_CUDA_TRY(cudaMemcpy2DAsync(pc->Minv + i0 * m, sizeof(cplx) * m, xc, sizeof(cplx) * tot,
                                            sizeof(cplx) * m, (size_t)std::min<int64_t>(2, m - i0),
                                            cudaMemcpyDeviceToDevice, st));
        }
        BBJD_CUDA_TRY(cudaStreamSynchronize(st));
    }
    if (pc->t == 0) return BBJD_SUCCESS;

    // border: Y = K^-1 E (t right-hand sides, two at a time), S = G - F1 Y
    const int t = pc->t;
    BBJD_CUDA_TRY(cudaMalloc(&pc->Y, sizeof(cplx) * (size_t)pc->nb * t));
    for (int c = 0; c < t; c += 2) {
        bbjd_status s;
        if (c + 1 < t) s = bcr_solve<BS, 2>(pc, m->E + (int64_t)c * pc->nb, pc->nb, pc->Y + (int64_t)c * pc->nb, pc->nb, st);
        else s = bcr_solve<BS, 1>(pc, m->E + (int64_t)c * pc->nb, pc->nb, pc->Y + (int64_t)c * pc->nb, pc->nb, st);
        if (s != BBJD_SUCCESS) return s;
    }
    const int Gs = (int)std::max<int64_t>(1, std::min<int64_t>(2 * num_sms(), (pc->nb + 1023) / 1024));
    const int64_t rpc = ((pc->nb + Gs - 1) / Gs + 15) / 16 * 16;
    cplx *part = nullptr, *Sd = nullptr;
    BBJD_CUDA_TRY(cudaMalloc(&part, sizeof(cplx) * (size_t)Gs * t * t));
    BBJD_CUDA_TRY(cudaMalloc(&Sd, sizeof(cplx) * (size_t)t * t));
    k_schur_part<<<Gs, 256, 0, st>>>(pc->nb, t, m->FT, pc->Y, rpc, part);
    BBJD_LAUNCH_CHECK();
    {
        bbjd_status rs = reduce_partials(part, Gs, t * t, Sd, st);
        if (rs != BBJD_SUCCESS) return rs;
    }
    std::vector<std::complex<double>> S((size_t)t * t), G((size_t)t * t), Sinv;
    BBJD_CUDA_TRY(cudaMemcpyAsync(S.data(), Sd, sizeof(cplx) * t * t, cudaMemcpyDeviceToHost, st));
    // corner G[tau][c] = F[tau, nb + c] = FT[(nb + c) * t + tau]: column-major t x t
    BBJD_CUDA_TRY(cudaMemcpyAsync(G.data(), m->FT + pc->nb * t, sizeof(cplx) * t * t, cudaMemcpyDeviceToHost, st));
    BBJD_CUDA_TRY(cudaStreamSynchronize(st));
    cudaFree(part);
    cudaFree(Sd);
    // FT rows nb..n-1 hold F[:, nb + c] contiguous over tau: element (tau, c) at c*t + tau
    for (size_t e = 0; e < S.size(); ++e) S[e] = G[e] - S[e];
    if (!host_inverse(t, S, Sinv)) return BBJD_ERR_BREAKDOWN;
    BBJD_CUDA_TRY(cudaMalloc(&pc->Sinv, sizeof(cplx) * (size_t)t * t));
    BBJD_CUDA_TRY(cudaMemcpy(pc->Sinv, Sinv.data(), sizeof(cplx) * t * t, cudaMemcpyHostToDevice));
    return BBJD_SUCCESS;
}

template <int BS>
static bbjd_status factor_bjac(bbjd_precond *pc, const bbjd_bbt_matrix *m, cplx sigma, cudaStream_t st) {
    constexpr int64_t BB = BS * BS;
    BBJD_CUDA_TRY(cudaMemsetAsync(pc->err, 0, sizeof(int), st));
    BBJD_CUDA_TRY(cudaMalloc(&pc->pool, sizeof(cplx) * BB * pc->nblk));
    pc->pool_elems = BB * pc->nblk;
    pc->pool_base = pc->pool;
    cplx *D = nullptr;
    BBJD_CUDA_TRY(cudaMalloc(&D, sizeof(cplx) * BB * pc->nblk));
    k_shift<<<grid_for(BB * pc->nblk, 256, 8 * num_sms()), 256, 0, st>>>(BB * pc->nblk, m->Ad, m->Bd, sigma, D);
    BBJD_LAUNCH_CHECK();
    k_invert_blocks<BS><<<grid_for(pc->nblk, 1, 64 * num_sms()), 256, inv_smem<BS>(), st>>>(pc->nblk, D, pc->pool, pc->err, nullptr);
    BBJD_LAUNCH_CHECK();
    BBJD_CUDA_TRY(cudaStreamSynchronize(st));
    cudaFree(D);
    int err = 0;
    BBJD_CUDA_TRY(cudaMemcpy(&err, pc->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) return BBJD_ERR_BREAKDOWN;
    if (pc->t > 0) {
        const int t = pc->t;
        std::vector<std::complex<double>> G((size_t)t * t), Ginv;
        BBJD_CUDA_TRY(cudaMemcpy(G.data(), m->FT + pc->nb * t, sizeof(cplx) * t * t, cudaMemcpyDeviceToHost));
        if (!host_inverse(t, G, Ginv)) return BBJD_ERR_BREAKDOWN;
        BBJD_CUDA_TRY(cudaMalloc(&pc->Ginv, sizeof(cplx) * (size_t)t * t));
        BBJD_CUDA_TRY(cudaMemcpy(pc->Ginv, Ginv.data(), sizeof(cplx) * t * t, cudaMemcpyHostToDevice));
    }
    return BBJD_SUCCESS;
}

}  // namespace bbjd

namespace bbjd {
// Mixed precision: keep complex64 copies of the factor blocks, of Y = K^-1 E
// and of the tau rows (the solve reads them, widening to FP64 for the
// arithmetic), and release the FP64 factor blocks and Y.  The factorisation
// itself ran in FP64.
static bbjd_status to_complex64(bbjd_precond *pc, const bbjd_bbt_matrix *m) {
    const int cap = 8 * num_sms();
    BBJD_CUDA_TRY(cudaMalloc(&pc->pool32, sizeof(float2) * (size_t)pc->pool_elems));
    k_to_c64<<<grid_for(pc->pool_elems, 256, cap), 256>>>(pc->pool_elems, pc->pool, pc->pool32);
    BBJD_LAUNCH_CHECK();
    if (pc->Y) {
        const int64_t ny = pc->nb * pc->t, nf = m->n * m->t;
        BBJD_CUDA_TRY(cudaMalloc(&pc->Y32, sizeof(float2) * (size_t)ny));
        BBJD_CUDA_TRY(cudaMalloc(&pc->FT32, sizeof(float2) * (size_t)nf));
        k_to_c64<<<grid_for(ny, 256, cap), 256>>>(ny, pc->Y, pc->Y32);
        BBJD_LAUNCH_CHECK();
        k_to_c64<<<grid_for(nf, 256, cap), 256>>>(nf, m->FT, pc->FT32);
        BBJD_LAUNCH_CHECK();
    }
    BBJD_CUDA_TRY(cudaDeviceSynchronize());
    cudaFree(pc->pool);
    pc->pool = nullptr;   // pool_base keeps the offsets
    cudaFree(pc->Y);
    pc->Y = nullptr;
    return BBJD_SUCCESS;
}
}  // namespace bbjd

using namespace bbjd;

extern "C" bbjd_status bbjd_precond_create(const bbjd_bbt_matrix *m, bbjd_zomplex sigma, int kind,
                                           int precision, bbjd_precond **out) {
    if (!m || !out || (kind != BBJD_PC_BBT_LU && kind != BBJD_PC_BLOCK_JACOBI)) return BBJD_ERR_INVALID;
    if (precision != BBJD_FP64 && precision != BBJD_MIXED) return BBJD_ERR_INVALID;
    auto t0 = std::chrono::steady_clock::now();
    auto *pc = new bbjd_precond();
    pc->kind = kind;
    pc->precision = precision;
    pc->b = m->b;
    pc->t = m->t;
    pc->nblk = m->nblk;
    pc->nb = m->nb;
    pc->n = m->n;
    pc->FT = m->FT;
    const cplx sg = mk(sigma.real(), sigma.imag());
    cudaStream_t st = nullptr;
    bbjd_status s = BBJD_SUCCESS;
    if (cudaMalloc(&pc->err, sizeof(int)) != cudaSuccess) s = BBJD_ERR_ALLOC;
    // per device (raise_smem_limit keeps the largest value set on each)
    if (s == BBJD_SUCCESS) s = set_attrs<8>();
    if (s == BBJD_SUCCESS) s = set_attrs<16>();
    if (s == BBJD_SUCCESS) s = set_attrs<32>();
    if (s == BBJD_SUCCESS) {
        pc->G = (int)std::max<int64_t>(1, std::min<int64_t>(4 * num_sms(), (m->nb + 255) / 256));
        if (cudaMalloc(&pc->tau_part, sizeof(cplx) * (size_t)pc->G * 2 * std::max(1, m->t)) != cudaSuccess ||
            cudaMalloc(&pc->x2, sizeof(cplx) * 2 * std::max(1, m->t)) != cudaSuccess ||
            cudaMalloc(&pc->gbuf, sizeof(cplx) * 2 * std::max(1, m->t)) != cudaSuccess)
            s = BBJD_ERR_ALLOC;
    }
    if (s == BBJD_SUCCESS) {
        if (kind == BBJD_PC_BBT_LU) {
            if (m->b == 8) s = factor_bcr<8>(pc, m, sg, st);
            else if (m->b == 16) s = factor_bcr<16>(pc, m, sg, st);
            else s = factor_bcr<32>(pc, m, sg, st);
        } else {
            if (m->b == 8) s = factor_bjac<8>(pc, m, sg, st);
            else if (m->b == 16) s = factor_bjac<16>(pc, m, sg, st);
            else s = factor_bjac<32>(pc, m, sg, st);
        }
    }
    if (s == BBJD_SUCCESS && cudaDeviceSynchronize() != cudaSuccess) s = BBJD_ERR_CUDA;
    if (s == BBJD_SUCCESS && precision == BBJD_MIXED) s = to_complex64(pc, m);
    if (s != BBJD_SUCCESS) {
        bbjd_precond_free(pc);
        return s;
    }
    pc->factor_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *out = pc;
    return BBJD_SUCCESS;
}

extern "C" void bbjd_precond_free(bbjd_precond *pc) {
    if (!pc) return;
    for (auto &g : pc->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    cudaFree(pc->pool);
    cudaFree(pc->pool32);
    cudaFree(pc->Y);
    cudaFree(pc->Y32);
    cudaFree(pc->FT32);
    cudaFree(pc->Sinv);
    cudaFree(pc->Ginv);
    cudaFree(pc->lvl_rhs);
    cudaFree(pc->lvl_x);
    cudaFree(pc->tau_part);
    cudaFree(pc->x2);
    cudaFree(pc->gbuf);
    cudaFree(pc->Minv);
    cudaFree(pc->mpart);
    cudaFree(pc->err);
    delete pc;
}

extern "C" double bbjd_precond_solve_bytes(const bbjd_precond *pc, int nrhs) {
    return pc ? precond_bytes(pc, nrhs) : 0.0;
}

extern "C" double bbjd_precond_factor_seconds(const bbjd_precond *pc) {
    return pc ? pc->factor_seconds : 0.0;
}

extern "C" bbjd_status bbjd_precond_solve(const bbjd_precond *pc, int nrhs, const bbjd_zomplex *r,
                                          bbjd_zomplex *x, void *stream) {
    if (!pc || !r || !x || nrhs < 1 || nrhs > 2) return BBJD_ERR_INVALID;
    return precond_solve(pc, nrhs, reinterpret_cast<const cplx *>(r), reinterpret_cast<cplx *>(x),
                         pc->n, (cudaStream_t)stream);
}
