// FMA-rate probe of include/tcp_probe.h: the arithmetic ceiling that the MVP
// kernels' roofline is reported against.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "../../include/tcp_mvp.h"
#include "../../include/tcp_probe.h"
#include "tcp_internal.h"

namespace {

constexpr int kProbeThreads = 256;
constexpr int kProbeChains = 8;   // independent FMA chains per thread
constexpr int kProbeIters = 8192;

// v <- v * a + b on kProbeChains independent chains; the sum is stored so the
// loop cannot be removed.  With |a| < 1 the chains converge to b / (1 - a).
template <typename R>
__global__ void __launch_bounds__(kProbeThreads) k_fma_probe(R a, R b, R *out) {
    R v[kProbeChains];
#pragma unroll
    for (int j = 0; j < kProbeChains; ++j) v[j] = static_cast<R>(threadIdx.x + j) * static_cast<R>(1e-3);
    for (int it = 0; it < kProbeIters; ++it) {
#pragma unroll
        for (int j = 0; j < kProbeChains; ++j) v[j] = fma(v[j], a, b);
    }
    R s = 0;
#pragma unroll
    for (int j = 0; j < kProbeChains; ++j) s += v[j];
    out[static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x] = s;
}

template <typename R>
int probe(uint32_t repeats, double *rate, double *ms_out) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fma_probe<R>, kProbeThreads, 0);
    const int grid = std::max(sms, 1) * std::max(per_sm, 1);
    R *out = nullptr;
    cudaError_t e = cudaMalloc(&out, sizeof(R) * static_cast<size_t>(grid) * kProbeThreads);
    if (e != cudaSuccess) return tcp::fail(TCP_ERR_ALLOCATION, std::string("probe allocation: ") + cudaGetErrorString(e));
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    float best = 1e30f;
    k_fma_probe<R><<<grid, kProbeThreads>>>(static_cast<R>(0.999), static_cast<R>(1e-3), out);  // warm-up
    for (uint32_t r = 0; r < std::max(repeats, 1u); ++r) {
        cudaEventRecord(t0);
        k_fma_probe<R><<<grid, kProbeThreads>>>(static_cast<R>(0.999), static_cast<R>(1e-3), out);
        cudaEventRecord(t1);
        cudaEventSynchronize(t1);
        float ms = 0;
        cudaEventElapsedTime(&ms, t0, t1);
        best = std::min(best, ms);
    }
    e = cudaGetLastError();
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    cudaFree(out);
    if (e != cudaSuccess) return tcp::fail(TCP_ERR_CUDA, std::string("probe kernel: ") + cudaGetErrorString(e));
    const double flops = 2.0 * kProbeChains * kProbeIters * static_cast<double>(grid) * kProbeThreads;
    *rate = flops / (best * 1e-3);
    if (ms_out) *ms_out = best;
    return TCP_OK;
}

}  // namespace

extern "C" int tcp_probe_fma_rate(int dtype, uint32_t repeats, double *out_flops_per_s, double *out_ms) {
    if (out_flops_per_s == nullptr) return tcp::fail(TCP_ERR_INVALID_ARGUMENT, "null output");
    if (dtype == TCP_DTYPE_C128) return probe<double>(repeats, out_flops_per_s, out_ms);
    if (dtype == TCP_DTYPE_C64) return probe<float>(repeats, out_flops_per_s, out_ms);
    return tcp::fail(TCP_ERR_INVALID_ARGUMENT, "unknown dtype");
}
