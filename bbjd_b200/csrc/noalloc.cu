// CGS + DGKS orthogonalisation that allocates nothing.
//
// Some callers cannot call cudaMalloc at the point where they orthogonalise:
// a host framework that owns all device memory and forbids allocation after
// start-up, or a pipeline that must not stall the device (cudaMalloc and
// cudaFree synchronise implicitly).  bbjd_dev_orthogonalize_static serves
// them: its reduction scratch is the file-scope device array below, so the
// call itself issues no allocation or free of any kind.
//
// The array (~2.7 MB) is held until the process exits by every GPU on which
// the module holding it is loaded.  With CUDA's lazy module loading (the
// default since CUDA 12.2) that happens at the first call on each device:
// that call loads the module, which allocates the array and may synchronise
// the device, so callers make one warm-up call (k = 0 will do) per device at
// start-up, before any stream capture.  Every call shares it and it keeps the last call's
// contents, so the call clears what must start at zero (the completion
// counter of the norm reduction) before it launches, and two calls that
// overlap on the GPU (different streams, or different host threads on one
// device) race on it: serialise them.
#include <cstdio>
#include <mutex>

#include "dense.cuh"

namespace bbjd {

// sizes of the static scratch (see include/bbjd_gpu.h for the call limits)
constexpr int ST_G_MAX = 640;                        // CTAs of the dot kernel
constexpr int ST_G2_MAX = 1280;                      // CTAs of the update kernel
constexpr int ST_X_MAX = BBJD_STATIC_ORTH_MAX_K + 1; // k dots + ||v||^2
constexpr size_t ST_PARTIAL = (size_t)ST_G_MAX * ST_X_MAX;     // complex
constexpr size_t ST_RED = 2 * (size_t)ST_X_MAX;                // complex: pass 1, pass 2
constexpr size_t ST_BYTES = 16 * (ST_PARTIAL + ST_RED) + 8 * ST_G2_MAX + 256;

// [partial | red | nrm_part | counter, flag, norm]
static __device__ __align__(256) unsigned char g_orth_scratch[ST_BYTES];

namespace {
constexpr int MAX_DEV = 64;
std::mutex g_mu;
unsigned char *g_addr[MAX_DEV] = {nullptr};
}  // namespace

// Device address of the static scratch on the current device.  In host code
// g_orth_scratch names a host-side stand-in, not device memory; the device
// address comes from cudaGetSymbolAddress, once per device, with that device
// current.
static bbjd_status scratch_address(unsigned char **out) {
    int dev = 0;
    BBJD_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEV) return BBJD_ERR_INVALID;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        BBJD_CUDA_TRY(cudaGetSymbolAddress(&p, g_orth_scratch));
        g_addr[dev] = static_cast<unsigned char *>(p);
    }
    *out = g_addr[dev];
    return BBJD_SUCCESS;
}

}  // namespace bbjd

using namespace bbjd;

extern "C" bbjd_status bbjd_dev_orthogonalize_static(bbjd_int n, bbjd_int k, const bbjd_zomplex *Q,
                                                     bbjd_int ldq, bbjd_zomplex *v,
                                                     double *norm_out, int *second_pass_out,
                                                     void *stream) {
    if (n < 1 || k < 0 || !v || (k > 0 && (!Q || ldq < n))) return BBJD_ERR_INVALID;
    if (n > BBJD_STATIC_ORTH_MAX_N || k > BBJD_STATIC_ORTH_MAX_K) {
        fprintf(stderr,
                "bbjd_dev_orthogonalize_static: n = %lld, k = %lld exceeds the static scratch "
                "(n <= %d, k <= %d); use bbjd_dev_orthogonalize\n",
                (long long)n, (long long)k, BBJD_STATIC_ORTH_MAX_N, BBJD_STATIC_ORTH_MAX_K);
        return BBJD_ERR_INVALID;
    }
    unsigned char *base = nullptr;
    bbjd_status s = scratch_address(&base);
    if (s) return s;
    cudaStream_t st = (cudaStream_t)stream;

    // the same launch shapes as the allocating variant, capped to the array
    Scratch S;
    S.n = n;
    const int sms = num_sms();
    int G = (int)std::max<int64_t>(1, std::min<int64_t>(std::min(4 * sms, ST_G_MAX), (n + 255) / 256));
    // the dot kernel stages its rows' v in shared memory (16 B a row): on a
    // device with few SMs visible (MPS, green contexts) use all ST_G_MAX CTAs,
    // which keeps n <= BBJD_STATIC_ORTH_MAX_N under 205 KB whatever the SM count
    if (16 * (((n + G - 1) / G + 31) / 32 * 32) > 200 * 1024)
        G = (int)std::max<int64_t>(1, std::min<int64_t>(ST_G_MAX, (n + 255) / 256));
    S.rpc = ((n + G - 1) / G + 31) / 32 * 32;
    S.G = (int)((n + S.rpc - 1) / S.rpc);
    S.G2 = (int)std::max<int64_t>(1, std::min<int64_t>(std::min(8 * sms, ST_G2_MAX), (n + 255) / 256));
    S.maxX = ST_X_MAX;
    S.partial = reinterpret_cast<cplx *>(base);
    S.red = S.partial + ST_PARTIAL;
    S.nrm_part = reinterpret_cast<double *>(S.red + ST_RED);
    unsigned char *tail = reinterpret_cast<unsigned char *>(S.nrm_part + ST_G2_MAX);
    S.counter = reinterpret_cast<unsigned *>(tail);
    S.flags = reinterpret_cast<int *>(tail + 64);
    S.scal = reinterpret_cast<double *>(tail + 128);
    if ((s = tsdot_allow_smem(sizeof(cplx) * (size_t)S.rpc))) return s;
    // the norm reduction's completion counter must start at zero
    BBJD_CUDA_TRY(cudaMemsetAsync(S.counter, 0, sizeof(unsigned), st));

    const cplx *dQ = reinterpret_cast<const cplx *>(Q);
    cplx *dv = reinterpret_cast<cplx *>(v);
    cplx *h1 = S.red, *h2 = S.red + ST_X_MAX;
    if (k == 0) {
        s = update(S, 0, n, nullptr, nullptr, nullptr, mk(0, 0), mk(0, 0), mk(1, 0), dv, mk(0, 0),
                   nullptr, dv, S.scal, nullptr, nullptr, nullptr, nullptr, st);
    } else {
        s = tsdot(S, 1, 1, (int)k, ldq, dQ, nullptr, dv, nullptr, h1, nullptr, st);
        if (!s) s = update(S, (int)k, ldq, dQ, h1, nullptr, mk(1, 0), mk(0, 0), mk(1, 0), dv, mk(0, 0),
                           nullptr, dv, S.scal, h1 + k, nullptr, S.flags, nullptr, st);
        if (!s) s = tsdot(S, 1, 1, (int)k, ldq, dQ, nullptr, dv, nullptr, h2, S.flags, st);
        if (!s) s = update(S, (int)k, ldq, dQ, h2, nullptr, mk(1, 0), mk(0, 0), mk(1, 0), dv, mk(0, 0),
                           nullptr, dv, S.scal, nullptr, nullptr, nullptr, S.flags, st);
    }
    double nrm = 0.0;
    int flag = 0;
    if (!s && cudaMemcpyAsync(&nrm, S.scal, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        s = BBJD_ERR_CUDA;
    if (!s && k > 0 && cudaMemcpyAsync(&flag, S.flags, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        s = BBJD_ERR_CUDA;
    if (!s && cudaStreamSynchronize(st) != cudaSuccess) s = BBJD_ERR_CUDA;
    if (norm_out) *norm_out = nrm;
    if (second_pass_out) *second_pass_out = flag;
    return s;
}
