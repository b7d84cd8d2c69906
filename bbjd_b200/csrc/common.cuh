// Shared device helpers for the B200 JDQZ engine (sm_100a).
//
// Complex128 values are double2 (x = real, y = imaginary), the same bytes
// as C's double complex and std::complex<double>.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <atomic>

#include "../../include/bbjd_gpu.h"

namespace bbjd {

typedef double2 cplx;

__host__ __device__ __forceinline__ cplx mk(double re, double im) { return make_double2(re, im); }
__host__ __device__ __forceinline__ cplx cadd(cplx a, cplx b) { return mk(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ cplx csub(cplx a, cplx b) { return mk(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ cplx cmul(cplx a, cplx b) {
    return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// conj(a) * b
__host__ __device__ __forceinline__ cplx cmulc(cplx a, cplx b) {
    return mk(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ cplx cscale(cplx a, double s) { return mk(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ double cabs2(cplx a) { return a.x * a.x + a.y * a.y; }

// acc += a * b
__device__ __forceinline__ void cfma(cplx &acc, cplx a, cplx b) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
}
// acc += conj(a) * b
__device__ __forceinline__ void cfmac(cplx &acc, cplx a, cplx b) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(-a.y, b.x, acc.y);
}
// acc -= a * b
__device__ __forceinline__ void cfms(cplx &acc, cplx a, cplx b) {
    acc.x = fma(-a.x, b.x, acc.x);
    acc.x = fma(a.y, b.y, acc.x);
    acc.y = fma(-a.x, b.y, acc.y);
    acc.y = fma(-a.y, b.x, acc.y);
}

__device__ __forceinline__ cplx shfl(cplx v, int src, int width = 32) {
    return mk(__shfl_sync(0xffffffffu, v.x, src, width), __shfl_sync(0xffffffffu, v.y, src, width));
}
__device__ __forceinline__ cplx warp_sum(cplx v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Read-only streaming load (data read once per pass: bypass L1 allocation).
__device__ __forceinline__ cplx ldg_stream(const cplx *p) { return __ldcs(p); }

// Launch bookkeeping: every kernel launch of this library is counted so the
// device solve can report how many kernels it ran.
extern std::atomic<long long> g_launches;
inline void count_launch(int n = 1) { g_launches.fetch_add(n, std::memory_order_relaxed); }

int num_sms();
bbjd_status raise_smem_limit(const void *func, size_t bytes);

}  // namespace bbjd

#define BBJD_CUDA_TRY(expr)                                                  \
    do {                                                                     \
        cudaError_t _e = (expr);                                             \
        if (_e != cudaSuccess) {                                             \
            bbjd::set_last_error(_e, #expr, __FILE__, __LINE__);             \
            return BBJD_ERR_CUDA;                                            \
        }                                                                    \
    } while (0)

#define BBJD_LAUNCH_CHECK()                                                  \
    do {                                                                     \
        bbjd::count_launch();                                                \
        cudaError_t _e = cudaGetLastError();                                 \
        if (_e != cudaSuccess) {                                             \
            bbjd::set_last_error(_e, "kernel launch", __FILE__, __LINE__);   \
            return BBJD_ERR_CUDA;                                            \
        }                                                                    \
    } while (0)

namespace bbjd {
void set_last_error(cudaError_t e, const char *what, const char *file, int line);
}
