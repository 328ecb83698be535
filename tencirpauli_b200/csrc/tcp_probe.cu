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

// Shared-memory operand rate: 512 threads per CTA read 16-byte values from a
// 64 KiB tile in the MVP kernels' pattern -- lane t of a warp reads row
// (t ^ m) of an aligned 32-row block, 8 independent rows per thread, m
// changing every round -- and fold them into registers that are stored at
// the end.  One CTA per SM (the tile plus the launch bound keep it so).
constexpr int kSmemThreads = 512;
constexpr int kSmemRounds = 2048;
constexpr uint32_t kSmemRows = 4096;  // 64 KiB of 16-byte rows

__global__ void __launch_bounds__(kSmemThreads, 1) k_smem_probe(uint4 *out) {
    extern __shared__ __align__(128) uint4 tile[];
    const uint32_t t = threadIdx.x;
    for (uint32_t r = t; r < kSmemRows; r += kSmemThreads) tile[r] = make_uint4(r, r * 3u, r * 5u, r * 7u);
    __syncthreads();
    uint4 acc = make_uint4(0, 0, 0, 0);
    for (int it = 0; it < kSmemRounds; ++it) {
        const uint32_t m = (static_cast<uint32_t>(it) * 0x9e37u) & (kSmemThreads - 1u);
        const uint32_t base = t ^ m;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const uint4 v = tile[base + (static_cast<uint32_t>(j) << 9)];
            acc.x ^= v.x;
            acc.y += v.y;
            acc.z ^= v.z;
            acc.w += v.w;
        }
    }
    out[static_cast<size_t>(blockIdx.x) * blockDim.x + t] = acc;
}

int probe_smem(uint32_t repeats, double *rate, double *ms_out) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t smem = kSmemRows * sizeof(uint4);
    cudaError_t e = cudaFuncSetAttribute(k_smem_probe, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return tcp::fail(TCP_ERR_CUDA, std::string("probe attribute: ") + cudaGetErrorString(e));
    const int grid = std::max(sms, 1);
    uint4 *out = nullptr;
    e = cudaMalloc(&out, sizeof(uint4) * static_cast<size_t>(grid) * kSmemThreads);
    if (e != cudaSuccess) return tcp::fail(TCP_ERR_ALLOCATION, std::string("probe allocation: ") + cudaGetErrorString(e));
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    float best = 1e30f;
    k_smem_probe<<<grid, kSmemThreads, smem>>>(out);  // warm-up
    for (uint32_t r = 0; r < std::max(repeats, 1u); ++r) {
        cudaEventRecord(t0);
        k_smem_probe<<<grid, kSmemThreads, smem>>>(out);
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
    const double bytes = 16.0 * 8.0 * kSmemRounds * static_cast<double>(grid) * kSmemThreads;
    *rate = bytes / (best * 1e-3);
    if (ms_out) *ms_out = best;
    return TCP_OK;
}

}  // namespace

extern "C" int tcp_probe_smem_rate(uint32_t repeats, double *out_bytes_per_s, double *out_ms) {
    if (out_bytes_per_s == nullptr) return tcp::fail(TCP_ERR_INVALID_ARGUMENT, "null output");
    return probe_smem(repeats, out_bytes_per_s, out_ms);
}

extern "C" int tcp_probe_fma_rate(int dtype, uint32_t repeats, double *out_flops_per_s, double *out_ms) {
    if (out_flops_per_s == nullptr) return tcp::fail(TCP_ERR_INVALID_ARGUMENT, "null output");
    if (dtype == TCP_DTYPE_C128) return probe<double>(repeats, out_flops_per_s, out_ms);
    if (dtype == TCP_DTYPE_C64) return probe<float>(repeats, out_flops_per_s, out_ms);
    return tcp::fail(TCP_ERR_INVALID_ARGUMENT, "unknown dtype");
}
