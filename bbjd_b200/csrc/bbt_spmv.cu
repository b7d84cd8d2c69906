// Fused A x / B x product of a block-bordered pencil (HBM-bound, sm_100a).
//
// Replaces the two operator callbacks the reference makes per Ritz vector
// and per expansion vector (reference jd_core.c:884-885, 1051-1054, through
// the scipy CSC closures of bbjd.py:183-205), and fuses the residual
// r = theta_b A u - theta_a B u with its norm (reference jd_core.c:887-892).
//
// Mapping: a warp owns 32/BS consecutive block rows per step (lane = one
// row of one block).  Blocks are column-major, so for each column c the
// lanes of a block row read 32 consecutive complex values (one 512-byte
// transaction); the three x segments a block row needs are held one value
// per lane and broadcast with shuffles.  The border columns E (column-major,
// ld nb) are read the same way against x's tail staged in shared memory.
// The tau rows are t dot products of length n: the warp that owns columns
// [32 g, 32 g + 32) adds F[:, those columns] x[those columns] into per-lane
// accumulators (lane = tau), reading F^T rows contiguously; the CTA reduces
// its warps in shared memory and a finalize kernel sums the CTAs in a fixed
// order and adds the corner block.
#include "bbt.cuh"

#include <algorithm>

namespace bbjd {

template <int BS, int NQ>
__global__ void __launch_bounds__(256, 2) k_bbt_spmv(
    int64_t nblk, int t, int64_t nb, const cplx *__restrict__ Ad, const cplx *__restrict__ Al,
    const cplx *__restrict__ Au, const cplx *__restrict__ Bd, const cplx *__restrict__ E,
    const cplx *__restrict__ FT, const cplx *__restrict__ x, cplx *__restrict__ yA,
    cplx *__restrict__ yB, cplx ta, cplx tb, cplx *__restrict__ r, cplx *__restrict__ tau_part,
    double *__restrict__ rn_part) {
    constexpr int BPW = 32 / BS;
    constexpr int BB = BS * BS;
    extern __shared__ cplx sm[];
    cplx *xtail = sm;           // t
    cplx *wtau = sm + t;        // 8 warps x t
    for (int i = threadIdx.x; i < t; i += blockDim.x) xtail[i] = x[nb + i];
    __syncthreads();

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int hw = lane / BS, row = lane - hw * BS, base = hw * BS;
    const int64_t gw = (int64_t)blockIdx.x * 8 + warp, nw = (int64_t)gridDim.x * 8;
    const int64_t ngroups = (nblk + BPW - 1) / BPW;
    // NQ = 0: t is a power of two below 32 and one load of F^T covers 32/t
    // columns (lane = column offset * t + tau); otherwise lane = tau and NQ
    // loads cover the t tau values of one column.
    constexpr int NA = NQ > 0 ? NQ : 1;
    cplx tacc[NA];
#pragma unroll
    for (int q = 0; q < NA; ++q) tacc[q] = mk(0.0, 0.0);
    double rn = 0.0;

    for (int64_t gi = gw; gi < ngroups; gi += nw) {
        const int64_t j = gi * BPW + hw;
        const bool valid = j < nblk;
        const int64_t jc = valid ? j : nblk - 1;
        const cplx xc = valid ? x[jc * BS + row] : mk(0.0, 0.0);
        const cplx xp = (valid && j > 0) ? x[(jc - 1) * BS + row] : mk(0.0, 0.0);
        const cplx xn = (valid && j + 1 < nblk) ? x[(jc + 1) * BS + row] : mk(0.0, 0.0);
        const cplx *pd = Ad + jc * BB + row;
        const cplx *pl = Al + jc * BB + row;
        const cplx *pu = Au + jc * BB + row;
        const cplx *pb = Bd + jc * BB + row;
        cplx a = mk(0.0, 0.0), bacc = mk(0.0, 0.0);
#pragma unroll 4
        for (int c = 0; c < BS; ++c) {
            const cplx xcc = shfl(xc, base + c), xpc = shfl(xp, base + c), xnc = shfl(xn, base + c);
            const cplx md = ldg_stream(pd + c * BS), ml = ldg_stream(pl + c * BS);
            const cplx mu = ldg_stream(pu + c * BS), mb = ldg_stream(pb + c * BS);
            cfma(a, md, xcc);
            cfma(a, ml, xpc);
            cfma(a, mu, xnc);
            cfma(bacc, mb, xcc);
        }
        if (t > 0) {
            const cplx *pe = E + jc * BS + row;
#pragma unroll 8
            for (int tau = 0; tau < t; ++tau) cfma(a, ldg_stream(pe + (int64_t)tau * nb), xtail[tau]);
            // tau-row partial sums over the 32 columns of this group
            const int64_t col0 = gi * 32;
            if constexpr (NQ == 0) {
                // element (tau, col0 + c) with c = k * 32/t + lane / t sits at
                // FT + col0 * t + 32 k + lane; columns past nb (last group) read
                // the last interior column and meet x = 0
                const int cpl = 32 / t, cc = lane / t;
                const int64_t last = (nb - 1) * t + (lane - cc * t);
                const cplx *pf = FT + col0 * t + lane;
#pragma unroll 1
                for (int k = 0; k < t; ++k) {
                    const cplx xv = shfl(xc, k * cpl + cc);
                    const int64_t off = col0 * t + 32 * k + lane;
                    cfma(tacc[0], ldg_stream(off <= last ? pf + 32 * k : FT + last), xv);
                }
            } else {
#pragma unroll 4
                for (int c = 0; c < 32; ++c) {
                    const cplx xv = shfl(xc, c);
                    const int64_t col = min(col0 + c, nb - 1);
                    const cplx *pf = FT + col * t;
#pragma unroll
                    for (int q = 0; q < NQ; ++q) {
                        const int tau = lane + 32 * q;
                        if (tau < t) cfma(tacc[q], ldg_stream(pf + tau), xv);
                    }
                }
            }
        }
        if (valid) {
            const int64_t i = j * BS + row;
            yA[i] = a;
            yB[i] = bacc;
            if (r) {
                cplx rr = cmul(tb, a);
                cfms(rr, ta, bacc);
                r[i] = rr;
                rn += cabs2(rr);
            }
        }
    }
    // CTA reduction of the tau partials (fixed order over warps)
    if constexpr (NQ == 0) {
        // lanes tau, tau + t, tau + 2t, ... hold the same tau row
        cplx v = tacc[0];
        for (int o = t; o < 32; o <<= 1) {
            v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
            v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
        }
        if (lane < t) wtau[warp * t + lane] = v;
    } else {
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            const int tau = lane + 32 * q;
            if (tau < t) wtau[warp * t + tau] = tacc[q];
        }
    }
    __shared__ double srn[8];
    rn = warp_sum(rn);
    if (lane == 0) srn[warp] = rn;
    __syncthreads();
    for (int tau = threadIdx.x; tau < t; tau += blockDim.x) {
        cplx s = wtau[tau];
        for (int w = 1; w < 8; ++w) s = cadd(s, wtau[w * t + tau]);
        tau_part[(int64_t)blockIdx.x * t + tau] = s;
    }
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < 8; ++w) s += srn[w];
        rn_part[blockIdx.x] = s;
    }
}

// Tau rows and the residual norm: y[nb + tau] = sum_g tau_part[g][tau] +
// F[tau, nb:] x[nb:], one warp per tau row (lanes over the CTA partials, a
// fixed order); B's tau rows are zero.  With a residual, the last CTA to
// finish adds the interior partial norms and the tau rows' |r|^2 in a fixed
// order and stores ||r||.
__global__ void __launch_bounds__(256) k_bbt_tau_finalize(
    int t, int64_t nb, int G, const cplx *__restrict__ tau_part, const cplx *__restrict__ FT,
    const cplx *__restrict__ x, cplx *__restrict__ yA, cplx *__restrict__ yB, cplx ta, cplx tb,
    cplx *__restrict__ r, const double *__restrict__ rn_part, double *__restrict__ rtau_nsq,
    unsigned *counter, double *__restrict__ rnorm) {
    const int lane = threadIdx.x & 31;
    const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (w < t) {
        cplx s = mk(0.0, 0.0);
        for (int g = lane; g < G; g += 32) s = cadd(s, tau_part[(int64_t)g * t + w]);
        for (int c = lane; c < t; c += 32) cfma(s, FT[(nb + c) * t + w], x[nb + c]);
        s = warp_sum(s);
        if (lane == 0) {
            yA[nb + w] = s;
            yB[nb + w] = mk(0.0, 0.0);
            if (r) {
                const cplx rr = cmul(tb, s);
                r[nb + w] = rr;
                rtau_nsq[w] = cabs2(rr);
            }
        }
    }
    if (!r) return;
    __shared__ bool last;
    __shared__ double red[8];
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!last) return;
    double acc = 0.0;
    for (int g = threadIdx.x; g < G; g += blockDim.x) acc += __ldcg(rn_part + g);
    for (int i = threadIdx.x; i < t; i += blockDim.x) acc += __ldcg(rtau_nsq + i);
    acc = warp_sum(acc);
    if (lane == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) tot += red[i];
        *rnorm = sqrt(tot);
        *counter = 0u;
    }
}

template <int BS>
static bbjd_status launch_spmv(const bbjd_bbt_matrix *m, const BBTScratch *sc, const cplx *x,
                               cplx *yA, cplx *yB, cplx ta, cplx tb, cplx *r, double *rnorm,
                               cudaStream_t st) {
    const size_t smem = sizeof(cplx) * (size_t)m->t * 9;
    const int nq = (m->t + 31) / 32;
#define BBJD_SPMV(NQ)                                                                   \
    k_bbt_spmv<BS, NQ><<<sc->G, 256, smem, st>>>(m->nblk, m->t, m->nb, m->Ad, m->Al, m->Au, \
                                                 m->Bd, m->E, m->FT, x, yA, yB, ta, tb, r,  \
                                                 sc->tau_part, sc->rn_part)
    const int t = m->t;
    if (t > 0 && t < 32 && (t & (t - 1)) == 0) BBJD_SPMV(0);
    else if (nq <= 1) BBJD_SPMV(1);
    else if (nq == 2) BBJD_SPMV(2);
    else if (nq <= 4) BBJD_SPMV(4);
    else return BBJD_ERR_INVALID;
#undef BBJD_SPMV
    BBJD_LAUNCH_CHECK();
    if (m->t > 0 || r) {
        const unsigned gf = (unsigned)std::max(1, (m->t + 7) / 8);
        k_bbt_tau_finalize<<<gf, 256, 0, st>>>(m->t, m->nb, sc->G, sc->tau_part, m->FT, x, yA, yB, ta,
                                               tb, r, sc->rn_part, sc->rtau_nsq, sc->counter, rnorm);
    }
    BBJD_LAUNCH_CHECK();
    return BBJD_SUCCESS;
}

bbjd_status bbt_scratch_alloc(const bbjd_bbt_matrix *m, BBTScratch *sc) {
    const int BPW = 32 / m->b;
    const int64_t groups = (m->nblk + BPW - 1) / BPW;
    const int t = m->t;
    sc->G = (int)std::max<int64_t>(1, std::min<int64_t>(4 * num_sms(), (groups + 7) / 8));
    BBJD_CUDA_TRY(cudaMalloc(&sc->tau_part, sizeof(cplx) * (size_t)sc->G * (t > 0 ? t : 1)));
    BBJD_CUDA_TRY(cudaMalloc(&sc->rn_part, sizeof(double) * (size_t)sc->G));
    BBJD_CUDA_TRY(cudaMalloc(&sc->rnorm, sizeof(double)));
    BBJD_CUDA_TRY(cudaMalloc(&sc->rtau_nsq, sizeof(double) * (size_t)(t > 0 ? t : 1)));
    BBJD_CUDA_TRY(cudaMalloc(&sc->counter, sizeof(unsigned)));
    BBJD_CUDA_TRY(cudaMemset(sc->counter, 0, sizeof(unsigned)));
    return BBJD_SUCCESS;
}

void bbt_scratch_free(BBTScratch *sc) {
    cudaFree(sc->tau_part);
    cudaFree(sc->rn_part);
    cudaFree(sc->rnorm);
    cudaFree(sc->rtau_nsq);
    cudaFree(sc->counter);
    *sc = BBTScratch();
}

bbjd_status bbt_apply(const bbjd_bbt_matrix *m, const BBTScratch *sc, const cplx *x, cplx *yA,
                      cplx *yB, cplx ta, cplx tb, cplx *r, double *rnorm, cudaStream_t st) {
    if (!sc) sc = &m->sc;
    if (!rnorm) rnorm = sc->rnorm;
    switch (m->b) {
        case 8: return launch_spmv<8>(m, sc, x, yA, yB, ta, tb, r, rnorm, st);
        case 16: return launch_spmv<16>(m, sc, x, yA, yB, ta, tb, r, rnorm, st);
        case 32: return launch_spmv<32>(m, sc, x, yA, yB, ta, tb, r, rnorm, st);
        default: return BBJD_ERR_INVALID;
    }
}

double bbt_bytes(const bbjd_bbt_matrix *m, bool with_residual) {
    const double bb = (double)m->b * m->b;
    double bytes = 16.0 * (4.0 * m->nblk * bb            // Ad, Al, Au, Bd
                           + 2.0 * (double)m->nb * m->t  // E and F's interior columns
                           + (double)m->t * m->t);       // corner
    bytes += 16.0 * 3.0 * m->n;                           // x read, yA and yB written
    if (with_residual) bytes += 16.0 * m->n;              // r written
    return bytes;
}

}  // namespace bbjd

// ===========================================================================
// C-ABI: device matrix lifetime and the stand-alone product
// ===========================================================================
using namespace bbjd;

extern "C" bbjd_status bbjd_bbt_create(bbjd_int b, bbjd_int nblk, bbjd_int t,
                                       const bbjd_zomplex *Ad, const bbjd_zomplex *Al,
                                       const bbjd_zomplex *Au, const bbjd_zomplex *E,
                                       const bbjd_zomplex *F, const bbjd_zomplex *Bd,
                                       int from_host, bbjd_bbt_matrix **out) {
    if (!out || (b != 8 && b != 16 && b != 32) || nblk < 1 || t < 0 || t > 128)
        return BBJD_ERR_INVALID;
    if (!Ad || !Al || !Au || !Bd || (t > 0 && (!E || !F))) return BBJD_ERR_INVALID;
    auto *m = new bbjd_bbt_matrix();
    m->b = (int)b;
    m->t = (int)t;
    m->nblk = nblk;
    m->nb = nblk * b;
    m->n = m->nb + t;
    const size_t bb = (size_t)nblk * b * b;
    const size_t ne = (size_t)m->nb * t, nf = (size_t)m->n * t;
    const size_t total = 4 * bb + ne + nf;
    cudaError_t e = cudaMalloc(&m->mem, sizeof(cplx) * total);
    if (e != cudaSuccess) { delete m; return BBJD_ERR_ALLOC; }
    m->Ad = m->mem;
    m->Al = m->Ad + bb;
    m->Au = m->Al + bb;
    m->Bd = m->Au + bb;
    m->E = m->Bd + bb;
    m->FT = m->E + ne;
    const cudaMemcpyKind kind = from_host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    const size_t blk = sizeof(cplx) * b * b;
    bool ok = cudaMemcpy(m->Ad, Ad, blk * nblk, kind) == cudaSuccess &&
              cudaMemcpy(m->Al, Al, blk * nblk, kind) == cudaSuccess &&
              cudaMemcpy(m->Au, Au, blk * nblk, kind) == cudaSuccess &&
              cudaMemcpy(m->Bd, Bd, blk * nblk, kind) == cudaSuccess;
    if (ok && t > 0)
        ok = cudaMemcpy(m->E, E, sizeof(cplx) * ne, kind) == cudaSuccess &&
             cudaMemcpy(m->FT, F, sizeof(cplx) * nf, kind) == cudaSuccess;
    // the couplings outside the matrix are zero by definition
    ok = ok && cudaMemset(m->Al, 0, blk) == cudaSuccess &&
         cudaMemset(m->Au + (size_t)(nblk - 1) * b * b, 0, blk) == cudaSuccess;
    ok = ok && bbt_scratch_alloc(m, &m->sc) == BBJD_SUCCESS;
    if (!ok) {
        bbjd_bbt_free(m);
        return BBJD_ERR_CUDA;
    }
    *out = m;
    return BBJD_SUCCESS;
}

extern "C" void bbjd_bbt_free(bbjd_bbt_matrix *m) {
    if (!m) return;
    cudaFree(m->mem);
    bbt_scratch_free(&m->sc);
    delete m;
}

extern "C" bbjd_int bbjd_bbt_n(const bbjd_bbt_matrix *m) { return m ? m->n : 0; }

extern "C" double bbjd_bbt_matvec_bytes(const bbjd_bbt_matrix *m) {
    return m ? bbt_bytes(m, false) : 0.0;
}

extern "C" bbjd_status bbjd_bbt_matvec(const bbjd_bbt_matrix *m, const bbjd_zomplex *x,
                                       bbjd_zomplex *yA, bbjd_zomplex *yB, void *stream) {
    if (!m || !x || !yA || !yB) return BBJD_ERR_INVALID;
    return bbt_apply(m, nullptr, reinterpret_cast<const cplx *>(x), reinterpret_cast<cplx *>(yA),
                     reinterpret_cast<cplx *>(yB), mk(0, 0), mk(0, 0), nullptr, nullptr,
                     (cudaStream_t)stream);
}
