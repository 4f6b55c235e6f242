// intpeak.cu - the measured int32 ALU rate of this GPU for the DP's own
// operation pattern, the denominator of the integer roofline.
//
// The band recurrence is a stream of int32 additions each followed by a
// maximum (M = max(M, M_p + s); D = max(D_p + e1, M_p + o1); the horizontal
// scan keys), so the kernel runs 16 independent chains per thread of
// v = max(v + inc, floor) and counts 2 operations per step (one add, one
// max), whatever instructions the compiler picks for them. Grid: 4 blocks of
// 256 threads per SM, enough warps to keep every scheduler issuing.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/poa_b200.h"

namespace {

constexpr int kChains = 16;

__global__ void __launch_bounds__(256) k_int_peak(int32_t* sink, int iters, int32_t seed) {
    int32_t v[kChains], inc[kChains];
    const int32_t floor_v = seed - (int32_t)threadIdx.x;
#pragma unroll
    for (int k = 0; k < kChains; k++) {
        v[k] = (int32_t)(threadIdx.x * 7u + blockIdx.x * 3u) + k;
        inc[k] = ((seed ^ (k * 2654435761u)) & 31) - 15;
    }
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int k = 0; k < kChains; k++) v[k] = max(v[k] + inc[k], floor_v);
    }
    int32_t r = 0;
#pragma unroll
    for (int k = 0; k < kChains; k++) r ^= v[k];
    if (r == seed) sink[blockIdx.x] = r;  // keeps the chains live; practically never taken
}

}  // namespace

extern "C" int poa_int_peak(int device, int iters, double* ops_per_s, double* ms) {
    if (!ops_per_s || iters <= 0) return POA_BAD_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return POA_CUDA;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return POA_CUDA;
    const int blocks = sms * 4, threads = 256;
    int32_t* sink = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = POA_CUDA;
    float t = 0.f;
    if (cudaMalloc((void**)&sink, sizeof(int32_t) * blocks) != cudaSuccess) return POA_CUDA;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) goto done;
    k_int_peak<<<blocks, threads>>>(sink, iters / 4 + 1, 12345);  // warm-up
    cudaEventRecord(e0);
    k_int_peak<<<blocks, threads>>>(sink, iters, 12345);
    cudaEventRecord(e1);
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) goto done;
    cudaEventElapsedTime(&t, e0, e1);
    if (t > 0.f) {
        *ops_per_s = (double)blocks * threads * (double)iters * kChains * 2.0 / (t * 1e-3);
        if (ms) *ms = t;
        rc = POA_OK;
    }
done:
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(sink);
    return rc;
}
