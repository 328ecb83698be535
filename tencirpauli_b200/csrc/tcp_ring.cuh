// Device building blocks of the ring kernels (k_ring in tcp_mvp.cu,
// k_ring_batched in tcp_batched.cu): ring geometry, the accumulator of a
// thread's 8 rows, and the walk of one group's term records.  The block
// layout they read is tcp::RingSchedule's.
#pragma once

#include "tcp_device.cuh"

namespace tcpdev {

constexpr uint32_t kRingWarps = kThreads / 32;  // warps that own the tile's rows
constexpr uint32_t kRingCompensateGroups = 16;  // FP32: groups per Kahan fold

// Who refills the ring.  complex128: a dedicated producer warp waits on the
// stages' "empty" barriers and issues the fills (measured faster for FP64,
// whose row warps fit the 96 registers a 544-thread block leaves them).
// complex64: no extra warp -- the row warp that releases a stage last issues
// its refill -- so the 512 threads keep 128 registers for the paired FP32
// accumulators.
template <typename R> struct RingShape;
template <> struct RingShape<double> {
    static constexpr bool kProducerWarp = true;
    static constexpr int kThreadsPerCta = kThreads + 32;
};
template <> struct RingShape<float> {
    static constexpr bool kProducerWarp = false;
    static constexpr int kThreadsPerCta = kThreads;
};

template <typename R> struct RingDepth;
template <> struct RingDepth<double> { static constexpr uint32_t K = 3; };  // 3 x (64 + 8) KiB
template <> struct RingDepth<float> { static constexpr uint32_t K = 4; };   // 4 x (32 + 8) KiB

template <typename R> constexpr uint32_t ring_tile_bytes() {
    return (1u << kTileBitsC128) * static_cast<uint32_t>(sizeof(typename Cx<R>::T));
}
template <typename R> constexpr uint32_t ring_stage_bytes() { return ring_tile_bytes<R>() + tcp::kRingBlockBytes; }
template <typename R> constexpr size_t ring_smem_bytes() {
    return static_cast<size_t>(RingDepth<R>::K) * ring_stage_bytes<R>();
}

template <typename R> __device__ __forceinline__ const unsigned char *ring_blocks(const DevSchedule &s);
template <> __device__ __forceinline__ const unsigned char *ring_blocks<double>(const DevSchedule &s) {
    return s.ring128;
}
template <> __device__ __forceinline__ const unsigned char *ring_blocks<float>(const DevSchedule &s) {
    return s.ring64;
}

// Weight of a ring term record: one f64 (bytes 8..15) or one f32 (bytes 8..11).
template <typename R> __device__ __forceinline__ R ring_weight(uint4 rec);
template <> __device__ __forceinline__ double ring_weight<double>(uint4 rec) {
    return __hiloint2double(static_cast<int>(rec.w), static_cast<int>(rec.z));
}
template <> __device__ __forceinline__ float ring_weight<float>(uint4 rec) { return __uint_as_float(rec.z); }

// One term record applied to the thread's 8 rows, row j reading loaded value
// j ^ A.  Sign of row j: parity(zlo & t) ^ parity(zt & tile) ^ bit j of the
// pattern (the rest is folded into the weight).  meta & t keeps only the zlo
// bits because t < 512.
template <int A, typename R>
__device__ __forceinline__ void ring_term(uint4 rec, uint32_t tid, uint32_t tile32,
                                          const typename Cx<R>::T (&xv)[8], RingAcc<R> (&acc)[8]) {
    const uint32_t meta = rec.x;
    const uint32_t base = __popc((meta & tid) ^ (rec.y & tile32)) & 1u;
    const uint32_t pattern = (meta >> 9) & 0xffu;
    const bool imag = ((meta >> 17) & 1u) != 0u;
    const R w = ring_weight<R>(rec);
    if (pattern == 0u) {
        const R ws = flip_by(w, base);
        if (!imag) {
#pragma unroll
            for (int j = 0; j < 8; ++j) acc[j].add_real(ws, xv[j ^ A]);
        } else {
#pragma unroll
            for (int j = 0; j < 8; ++j) acc[j].add_imag(ws, xv[j ^ A]);
        }
    } else {
        const uint32_t pat = (pattern ^ (0u - base)) & 0xffu;
        if (!imag) {
#pragma unroll
            for (int j = 0; j < 8; ++j) acc[j].add_real(flip_if(w, pat, j), xv[j ^ A]);
        } else {
#pragma unroll
            for (int j = 0; j < 8; ++j) acc[j].add_imag(flip_if(w, pat, j), xv[j ^ A]);
        }
    }
}

// The `nt` records of one group, two per iteration so that the integer work of
// one overlaps the multiply-adds of the other.
template <int A, typename R>
__device__ __forceinline__ void ring_group(const uint4 *__restrict__ trm, uint32_t nt, uint32_t tid, uint32_t tile32,
                                           const typename Cx<R>::T (&xv)[8], RingAcc<R> (&acc)[8]) {
    uint32_t k = 0;
    for (; k + 2u <= nt; k += 2u) {
        const uint4 r0 = trm[k], r1 = trm[k + 1];
        ring_term<A, R>(r0, tid, tile32, xv, acc);
        ring_term<A, R>(r1, tid, tile32, xv, acc);
    }
    if (k < nt) ring_term<A, R>(trm[k], tid, tile32, xv, acc);
}


}  // namespace tcpdev
