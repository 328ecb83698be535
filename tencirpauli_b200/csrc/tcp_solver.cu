// libtcpmvp.so -- eigensolver kernels built on the MVP: FP64 block
// inner products and block combinations over complex64 or complex128 vector
// storage, per-basis-state features, the Jacobi and learned (MLP)
// preconditioners, and the MLP's training kernels (forward, backward, Adam).
//
// Vectors are stored RHS-major (vector v at offset v * n) as complex64 or
// complex128; every reduction and combination accumulates in FP64.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <type_traits>
#include <string>
#include <vector>

#include "../../include/tcp_solver.h"
#include "tcp_device.cuh"
#include "tcp_plan_impl.h"

using namespace tcpdev;
using tcp::cuda_fail;
using tcp::fail;

namespace {

constexpr int kGramThreads = 512;      // 16 warps, one CTA per SM
constexpr int kGramWarps = kGramThreads / 32;
constexpr int kGramPairs = 16;         // (i, j) pairs of one warp tile
constexpr int kGramMaxVectors = 96;    // p + q
constexpr int kGramMaxPairs = 512;     // p * q
constexpr int kGramBlocks = 296;       // partial-sum slots in the work buffer
constexpr int kGramGrid = 148;         // CTAs launched (<= kGramBlocks)
constexpr int kGramRedBytes = 96 * 1024;  // shared memory for the row-group sums
constexpr int kGramStages = 4;            // TMA pipeline depth (chunks)
constexpr uint32_t kGramStageBytes = 48 * 1024;  // one chunk of every vector

constexpr int kCombineThreads = 256;
constexpr int kCombineTile = 4;        // output vectors per thread
constexpr int kCombineUnroll = 8;      // complex128 source vectors loaded ahead (16 for complex64)
constexpr int kCombineMaxK = 32;       // output vectors per launch

__device__ __forceinline__ double2 load_c(const void *base, int c64, uint64_t idx) {
    if (c64) {
        const float2 v = static_cast<const float2 *>(base)[idx];
        return make_double2(v.x, v.y);
    }
    return static_cast<const double2 *>(base)[idx];
}
__device__ __forceinline__ void store_c(void *base, int c64, uint64_t idx, double2 v) {
    if (c64) {
        static_cast<float2 *>(base)[idx] = make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
    } else {
        static_cast<double2 *>(base)[idx] = v;
    }
}
template <bool C64> __device__ __forceinline__ double2 load_v(const void *base, uint64_t idx) {
    if constexpr (C64) {
        const float2 v = __ldg(static_cast<const float2 *>(base) + idx);
        return make_double2(v.x, v.y);
    } else {
        return __ldg(static_cast<const double2 *>(base) + idx);
    }
}

__device__ __forceinline__ uint64_t umin64(uint64_t a, uint64_t b) { return a < b ? a : b; }

// t += conj(a) * b in FP64.
__device__ __forceinline__ void cmac(double2 &t, double2 a, double2 b) {
    t.x = fma(a.x, b.x, fma(a.y, b.y, t.x));
    t.y = fma(a.x, b.y, fma(-a.y, b.x, t.y));
}

// Per-CTA partial sums of G = A^H B.  The p x q pairs are cut into warp
// tiles of PI x QJ pairs (PI vectors of A, QJ of B: 8 x 1, 8 x 2 or 4 x 4,
// at most kGramPairs).  The CTA's rows are dealt to `groups` row groups, and
// its 16 warps take the (tile, row group) slots in turn: with groups chosen so
// that slots is a multiple of 16, every warp does the same work.  Warps walk
// the same 32-row chunks, so the B rows one tile reads are shared through L1
// by the warps of the other tiles and every vector crosses HBM once.  Each
// lane keeps its pair sums in FP64 registers; the warp reduces them by a
// fixed butterfly (commutative steps, so every lane holds the same bits), the
// row groups of a tile are summed in a fixed order from shared memory, and
// the CTA writes partial[block][i + p*j].  RPL = 2 (both blocks complex64,
// n even, 16-byte aligned) gives each lane two rows per chunk.
template <int QJ, bool A64, bool B64, int RPL>
__global__ void __launch_bounds__(kGramThreads, 1)
    k_gram_tiles(const void *__restrict__ A, uint32_t p, const void *__restrict__ B, uint32_t q, uint64_t n,
                 uint32_t groups, double2 *__restrict__ partial) {
    constexpr int PI = QJ == 4 ? 4 : 8;
    constexpr int TP = PI * QJ;
    static_assert(TP <= kGramPairs, "tile shape");
    extern __shared__ double2 red[];  // [slot][TP] when groups > 1
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t ni = (p + PI - 1) / PI, nj = (q + QJ - 1) / QJ, ntiles = ni * nj;
    const uint32_t slots = groups * ntiles;
    const uint32_t pairs = p * q;
    const uint64_t chunks = (n + 32 * RPL - 1) / (32 * RPL);
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * groups;
    for (uint32_t s = warp; s < slots; s += kGramWarps) {
        const uint32_t tile = s % ntiles, rg = s / ntiles;
        const uint32_t i0 = (tile % ni) * PI, j0 = (tile / ni) * QJ;
        double2 acc[TP];
#pragma unroll
        for (int e = 0; e < TP; ++e) acc[e] = make_double2(0.0, 0.0);
        for (uint64_t c = static_cast<uint64_t>(blockIdx.x) * groups + rg; c < chunks; c += stride) {
            if constexpr (RPL == 1) {
                const uint64_t row = c * 32 + lane;
                if (row < n) {
                    double2 b[QJ], a[PI];
#pragma unroll
                    for (int jj = 0; jj < QJ; ++jj)
                        b[jj] = j0 + jj < q ? load_v<B64>(B, static_cast<uint64_t>(j0 + jj) * n + row)
                                            : make_double2(0.0, 0.0);
#pragma unroll
                    for (int ii = 0; ii < PI; ++ii)
                        a[ii] = i0 + ii < p ? load_v<A64>(A, static_cast<uint64_t>(i0 + ii) * n + row)
                                            : make_double2(0.0, 0.0);
#pragma unroll
                    for (int ii = 0; ii < PI; ++ii) {
#pragma unroll
                        for (int jj = 0; jj < QJ; ++jj) cmac(acc[ii * QJ + jj], a[ii], b[jj]);
                    }
                }
            } else {
                // complex64 storage, n even: a lane loads rows 2 lane and
                // 2 lane + 1 of every vector as one 16-byte float4
                const uint64_t row = c * 64 + 2 * lane;
                if (row < n) {
                    const float4 *A4 = static_cast<const float4 *>(A), *B4 = static_cast<const float4 *>(B);
                    float4 b[QJ], a[PI];
#pragma unroll
                    for (int jj = 0; jj < QJ; ++jj)
                        b[jj] = j0 + jj < q ? __ldg(B4 + (static_cast<uint64_t>(j0 + jj) * n + row) / 2)
                                            : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                    for (int ii = 0; ii < PI; ++ii)
                        a[ii] = i0 + ii < p ? __ldg(A4 + (static_cast<uint64_t>(i0 + ii) * n + row) / 2)
                                            : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                    for (int ii = 0; ii < PI; ++ii) {
#pragma unroll
                        for (int jj = 0; jj < QJ; ++jj) {
                            cmac(acc[ii * QJ + jj], make_double2(a[ii].x, a[ii].y), make_double2(b[jj].x, b[jj].y));
                            cmac(acc[ii * QJ + jj], make_double2(a[ii].z, a[ii].w), make_double2(b[jj].z, b[jj].w));
                        }
                    }
                }
            }
        }
#pragma unroll
        for (int e = 0; e < TP; ++e) {
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                acc[e].x += __shfl_xor_sync(0xffffffffu, acc[e].x, off);
                acc[e].y += __shfl_xor_sync(0xffffffffu, acc[e].y, off);
            }
        }
#pragma unroll
        for (int e = 0; e < TP; ++e) {
            if (lane == static_cast<uint32_t>(e)) {
                if (groups == 1u) {
                    const uint32_t i = i0 + e / QJ, j = j0 + e % QJ;
                    if (i < p && j < q) partial[static_cast<size_t>(blockIdx.x) * pairs + i + p * j] = acc[e];
                } else {
                    red[s * TP + e] = acc[e];
                }
            }
        }
    }
    if (groups > 1u) {
        __syncthreads();
        for (uint32_t t = threadIdx.x; t < ntiles * TP; t += blockDim.x) {
            const uint32_t tile = t / TP, e = t % TP;
            double2 sum = make_double2(0.0, 0.0);
            for (uint32_t rg = 0; rg < groups; ++rg) {
                const double2 v = red[(rg * ntiles + tile) * TP + e];
                sum.x += v.x;
                sum.y += v.y;
            }
            const uint32_t i = (tile % ni) * PI + e / QJ, j = (tile / ni) * QJ + e % QJ;
            if (i < p && j < q) partial[static_cast<size_t>(blockIdx.x) * pairs + i + p * j] = sum;
        }
    }
}

// 2-D tiled TMA load of one box (x: innermost coordinate in 8-byte units,
// y: vector index) into shared memory; completes the box bytes on `bar`.
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// G = A^H B for two blocks of the same storage type, fed by the TMA engine.
// The blocks are described by two 2-D tensor maps (vectors x 8-byte units),
// and a chunk is one box of each: `rows` rows of every vector.  A CTA walks
// its full chunks (chunk c = blockIdx.x + k * gridDim.x) through a
// kGramStages-deep ring in shared memory; thread 0 issues the two box loads
// of a chunk onto the stage's mbarrier kGramStages - 1 chunks ahead of the
// consumers, so the loads in flight hold no registers.  The last n % rows
// rows are read straight from global memory by the CTA next in turn.  Warp w
// takes tile w % ntiles and row group w / ntiles (ntiles * groups <= 16); its
// lanes keep the tile's pair sums in FP64 registers.  The reduction order is
// fixed (warp butterfly, row groups, then k_gram_reduce over CTAs).  A box
// that does not land within the bounded wait poisons this CTA's partial sums
// with NaN, after a bounded wait for the boxes still in flight, so the caller
// sees a non-finite Gram matrix.
template <int QJ, bool C64>
__global__ void __launch_bounds__(kGramThreads, 1)
    k_gram_tma(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb,
               const void *__restrict__ A, uint32_t p, const void *__restrict__ B, uint32_t q, uint64_t n,
               uint32_t rows, uint32_t groups, double2 *__restrict__ partial) {
    using E = std::conditional_t<C64, float2, double2>;
    constexpr int PI = QJ == 4 ? 4 : 8;
    constexpr int TP = PI * QJ;
    constexpr int UNITS = sizeof(E) / 8;  // 8-byte units per element
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[kGramStages];
    __shared__ double2 red[kGramWarps][kGramPairs];
    E *ring = reinterpret_cast<E *>(smem_raw);
    const uint32_t vecs = p + q;
    const size_t stage_elems = static_cast<size_t>(vecs) * rows;
    const uint32_t stage_bytes = static_cast<uint32_t>(stage_elems * sizeof(E));
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    const uint32_t ni = (p + PI - 1) / PI, nj = (q + QJ - 1) / QJ, ntiles = ni * nj;
    const uint32_t pairs = p * q;
    const uint64_t chunks = n / rows;  // full chunks only
    const uint64_t mine = chunks > blockIdx.x ? (chunks - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;

    if (tid == 0) {
        for (int st = 0; st < kGramStages; ++st) mbar_init(&full[st], 1);
        fence_mbar_init();
    }
    __syncthreads();
    // chunk k of this CTA -> stage k % kGramStages
    auto issue = [&](uint64_t k) {
        const uint64_t r0 = (blockIdx.x + k * gridDim.x) * static_cast<uint64_t>(rows);
        uint64_t *bar = &full[k % kGramStages];
        E *dst = ring + (k % kGramStages) * stage_elems;
        mbar_arrive_expect_tx(bar, stage_bytes);
        tma_load_2d(dst, &ta, static_cast<int>(r0 * UNITS), 0, bar);
        tma_load_2d(dst + static_cast<size_t>(p) * rows, &tb, static_cast<int>(r0 * UNITS), 0, bar);
    };
    if (tid == 0) {
        for (uint64_t k = 0; k < mine && k + 1 < static_cast<uint64_t>(kGramStages); ++k) issue(k);
    }

    const bool active = warp < ntiles * groups;
    const uint32_t tile = warp % ntiles, rg = warp / ntiles;
    const uint32_t i0 = (tile % ni) * PI, j0 = (tile / ni) * QJ;
    double2 acc[TP];
#pragma unroll
    for (int e = 0; e < TP; ++e) acc[e] = make_double2(0.0, 0.0);
    // one row of the tile's vectors, from shared memory or from global memory
    auto accumulate = [&](const E *sa, const E *sb, size_t stride, uint64_t r) {
        double2 a[PI], b[QJ];
#pragma unroll
        for (int jj = 0; jj < QJ; ++jj) {
            if (j0 + jj < q) {
                const E v = sb[(j0 + jj) * stride + r];
                b[jj] = make_double2(v.x, v.y);
            } else {
                b[jj] = make_double2(0.0, 0.0);
            }
        }
#pragma unroll
        for (int ii = 0; ii < PI; ++ii) {
            if (i0 + ii < p) {
                const E v = sa[(i0 + ii) * stride + r];
                a[ii] = make_double2(v.x, v.y);
            } else {
                a[ii] = make_double2(0.0, 0.0);
            }
        }
#pragma unroll
        for (int ii = 0; ii < PI; ++ii) {
#pragma unroll
            for (int jj = 0; jj < QJ; ++jj) cmac(acc[ii * QJ + jj], a[ii], b[jj]);
        }
    };
    for (uint64_t k = 0; k < mine; ++k) {
        const uint32_t st = static_cast<uint32_t>(k % kGramStages);
        const bool ok = mbar_wait_bounded(&full[st], static_cast<uint32_t>(k / kGramStages) & 1u);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                // let the boxes already issued land before the CTA exits
                const uint64_t issued = umin64(mine, k + kGramStages - 1);
                for (uint64_t kk = k; kk < issued; ++kk)
                    mbar_wait_bounded(&full[kk % kGramStages], static_cast<uint32_t>(kk / kGramStages) & 1u,
                                      kWaitLimitNs / 4);
            }
            const double nan = __longlong_as_double(0x7ff8000000000000ll);
            for (uint32_t pr = tid; pr < pairs; pr += blockDim.x)
                partial[static_cast<size_t>(blockIdx.x) * pairs + pr] = make_double2(nan, nan);
            return;
        }
        // every thread has finished chunk k - 1, so its stage can be refilled
        if (tid == 0 && k + kGramStages - 1 < mine) {
            fence_proxy_async_smem();
            issue(k + kGramStages - 1);
        }
        if (active) {
            const E *sa = ring + st * stage_elems;
            for (uint32_t r = rg * 32 + lane; r < rows; r += groups * 32) accumulate(sa, sa + static_cast<size_t>(p) * rows, rows, r);
        }
    }
    const uint64_t tail0 = chunks * rows;
    if (active && tail0 < n && blockIdx.x == chunks % gridDim.x) {
        for (uint64_t r = tail0 + rg * 32 + lane; r < n; r += groups * 32)
            accumulate(static_cast<const E *>(A), static_cast<const E *>(B), n, r);
    }
#pragma unroll
    for (int e = 0; e < TP; ++e) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            acc[e].x += __shfl_xor_sync(0xffffffffu, acc[e].x, off);
            acc[e].y += __shfl_xor_sync(0xffffffffu, acc[e].y, off);
        }
    }
    if (active) {
#pragma unroll
        for (int e = 0; e < TP; ++e)
            if (lane == static_cast<uint32_t>(e)) red[warp][e] = acc[e];
    }
    __syncthreads();
    for (uint32_t t = tid; t < ntiles * TP; t += blockDim.x) {
        const uint32_t tl = t / TP, e = t % TP;
        double2 sum = make_double2(0.0, 0.0);
        for (uint32_t g = 0; g < groups; ++g) {
            const double2 v = red[g * ntiles + tl][e];
            sum.x += v.x;
            sum.y += v.y;
        }
        const uint32_t i = (tl % ni) * PI + e / QJ, j = (tl / ni) * QJ + e % QJ;
        if (i < p && j < q) partial[static_cast<size_t>(blockIdx.x) * pairs + i + p * j] = sum;
    }
}

// Deterministic reduction of the per-block partials (fixed order).
__global__ void k_gram_reduce(const double2 *__restrict__ partial, uint32_t blocks, uint32_t pairs,
                              double2 *__restrict__ out) {
    const uint32_t pr = blockIdx.x * blockDim.x + threadIdx.x;
    if (pr >= pairs) return;
    double re = 0.0, im = 0.0;
    for (uint32_t b = 0; b < blocks; ++b) {
        const double2 v = partial[static_cast<size_t>(b) * pairs + pr];
        re += v.x;
        im += v.y;
    }
    out[pr] = make_double2(re, im);
}

// out[:, j] = alpha * sum_i A[:, i] S[i, j] + beta * out[:, j]  (FP64 arithmetic).
// A CTA covers rb = 256 / njp consecutive rows for njp tiles of kCombineTile
// output vectors (njp: the tile count rounded up to a power of two); the
// tiles of the same rows sit in one CTA, so each source row is fetched from
// HBM once and re-read from L1.  Source values are loaded 8 (complex128) or
// 16 (complex64) ahead of their multiply-adds, and every output sums
// i = 0..p-1 in order.
// S is staged column-major as p x (njp * kCombineTile), zero beyond k.
template <bool A64, bool O64>
__global__ void __launch_bounds__(kCombineThreads)
    k_combine_tiles(const void *__restrict__ A, uint32_t p, const double2 *__restrict__ S, uint32_t k, uint32_t njp,
                    uint64_t n, double alpha, double beta, void *__restrict__ out) {
    extern __shared__ double2 ss[];
    const uint32_t kpad = njp * kCombineTile;
    for (uint32_t e = threadIdx.x; e < p * kpad; e += blockDim.x) {
        const uint32_t j = e / p;
        ss[e] = j < k ? S[e] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    const uint32_t rb = kCombineThreads / njp;
    const uint32_t jt = threadIdx.x / rb;
    if (jt * kCombineTile >= k) return;  // padding tile: no further barrier below
    constexpr int U = A64 ? 2 * kCombineUnroll : kCombineUnroll;
    const double2 *sj = ss + static_cast<size_t>(p) * jt * kCombineTile;
    for (uint64_t r = static_cast<uint64_t>(blockIdx.x) * rb + threadIdx.x % rb; r < n;
         r += static_cast<uint64_t>(gridDim.x) * rb) {
        double2 acc[kCombineTile];
#pragma unroll
        for (int jj = 0; jj < kCombineTile; ++jj) acc[jj] = make_double2(0.0, 0.0);
        uint32_t i = 0;
        for (; i + U <= p; i += U) {
            double2 a[U];
#pragma unroll
            for (int u = 0; u < U; ++u) a[u] = load_v<A64>(A, static_cast<uint64_t>(i + u) * n + r);
#pragma unroll
            for (int u = 0; u < U; ++u) {
#pragma unroll
                for (int jj = 0; jj < kCombineTile; ++jj) {
                    const double2 sv = sj[i + u + p * jj];
                    acc[jj].x = fma(a[u].x, sv.x, fma(-a[u].y, sv.y, acc[jj].x));
                    acc[jj].y = fma(a[u].x, sv.y, fma(a[u].y, sv.x, acc[jj].y));
                }
            }
        }
        for (; i < p; ++i) {
            const double2 a = load_v<A64>(A, static_cast<uint64_t>(i) * n + r);
#pragma unroll
            for (int jj = 0; jj < kCombineTile; ++jj) {
                const double2 sv = sj[i + p * jj];
                acc[jj].x = fma(a.x, sv.x, fma(-a.y, sv.y, acc[jj].x));
                acc[jj].y = fma(a.x, sv.y, fma(a.y, sv.x, acc[jj].y));
            }
        }
#pragma unroll
        for (int jj = 0; jj < kCombineTile; ++jj) {
            const uint32_t j = jt * kCombineTile + jj;
            if (j < k) {
                double2 v = make_double2(alpha * acc[jj].x, alpha * acc[jj].y);
                if (beta != 0.0) {
                    const double2 o = load_c(out, O64, static_cast<uint64_t>(j) * n + r);
                    v.x = fma(beta, o.x, v.x);
                    v.y = fma(beta, o.y, v.y);
                }
                store_c(out, O64, static_cast<uint64_t>(j) * n + r, v);
            }
        }
    }
}

// Jacobi correction t = -r / (d - theta), |d - theta| clamped below by eps.
__global__ void k_jacobi(const void *__restrict__ R, int r64, uint64_t n, uint32_t k, const double2 *__restrict__ diag,
                         const double *__restrict__ theta, double eps, void *__restrict__ T, int t64) {
    for (uint64_t r = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; r < n;
         r += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const double d = diag[r].x;
        for (uint32_t j = 0; j < k; ++j) {
            double den = d - theta[j];
            if (fabs(den) < eps) den = den < 0.0 ? -eps : eps;
            const double2 v = load_c(R, r64, j * n + r);
            store_c(T, t64, j * n + r, make_double2(-v.x / den, -v.y / den));
        }
    }
}

// Per-basis-state features that do not depend on the Ritz value (see
// tcp_solver.h): H_ii, the mean and minimum diagonal of the states the row
// couples to, sum |H_ij|, sum |H_ij|^2, the number of couplings, and the
// normalised Hamming weight of the basis state.
__global__ void k_features(DevSchedule s, uint32_t gzero, uint32_t nqubits, uint64_t n, float *__restrict__ feat) {
    for (uint64_t r = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; r < n;
         r += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        auto diag_at = [&](uint64_t c) -> double {
            double re = 0.0;
            if (gzero != 0xffffffffu) {
                for (uint32_t t = s.g_tbeg[gzero]; t < s.g_tbeg[gzero + 1]; ++t) {
                    const double2 w = s.t_w[t];
                    re += (__popcll(s.t_z[t] & c) & 1) ? -w.x : w.x;
                }
            }
            return re;
        };
        const double hii = diag_at(r);
        double sum_abs = 0.0, sum_sq = 0.0, sum_nd = 0.0, min_nd = 1e300;
        uint32_t count = 0;
        for (uint32_t g = 0; g < s.ngroups; ++g) {
            if (g == gzero) continue;
            const uint64_t c = r ^ s.g_mask[g];
            double dre = 0.0, dim = 0.0;
            for (uint32_t t = s.g_tbeg[g]; t < s.g_tbeg[g + 1]; ++t) {
                const double2 w = s.t_w[t];
                const bool neg = __popcll(s.t_z[t] & c) & 1;
                dre += neg ? -w.x : w.x;
                dim += neg ? -w.y : w.y;
            }
            const double a2 = dre * dre + dim * dim;
            if (a2 == 0.0) continue;
            const double dj = diag_at(c);
            sum_abs += sqrt(a2);
            sum_sq += a2;
            sum_nd += dj;
            min_nd = fmin(min_nd, dj);
            ++count;
        }
        float *f = feat + r * TCP_FEATURES;
        f[0] = static_cast<float>(hii);
        f[1] = static_cast<float>(count ? sum_nd / count : hii);
        f[2] = static_cast<float>(count ? min_nd : hii);
        f[3] = static_cast<float>(sum_abs);
        f[4] = static_cast<float>(sum_sq);
        f[5] = static_cast<float>(count);
        f[6] = static_cast<float>(static_cast<double>(__popcll(r)) / fmax(1.0, static_cast<double>(nqubits)) - 0.5);
        f[7] = 0.f;
    }
}

// ---------------------------------- MLP -------------------------------------
// Network: x (TCP_MLP_IN inputs, built from the features and the Ritz value)
// -> tanh(W1 x + b1) (TCP_MLP_HIDDEN) -> tanh(W2 h1 + b2) (TCP_MLP_HIDDEN)
// -> c = w3 . h2 + b3.  The correction is t = -exp(c) r / max(d - theta, eps):
// c = 0 is the Jacobi correction, and the network learns a per-state factor.
constexpr int IN = TCP_MLP_IN, HID = TCP_MLP_HIDDEN;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + HID * IN, OFF_W2 = OFF_B1 + HID, OFF_B2 = OFF_W2 + HID * HID,
              OFF_W3 = OFF_B2 + HID, OFF_B3 = OFF_W3 + HID, NPARAM = OFF_B3 + 1;
static_assert(NPARAM == TCP_MLP_PARAMS, "parameter count mismatch");

// Network inputs of one basis state for Ritz value theta; `scale` normalises
// energies (a spread of the spectrum).  Also returns den = max(d - theta, eps).
__device__ __forceinline__ void mlp_inputs(const float *__restrict__ f, double theta, double scale, double eps,
                                           float (&x)[IN], double &den) {
    const double inv = 1.0 / scale;
    double d = static_cast<double>(f[0]) - theta;
    den = fabs(d) < eps ? (d < 0.0 ? -eps : eps) : d;
    x[0] = static_cast<float>(d * inv);
    x[1] = static_cast<float>((static_cast<double>(f[1]) - theta) * inv);
    x[2] = static_cast<float>((static_cast<double>(f[2]) - theta) * inv);
    x[3] = static_cast<float>(static_cast<double>(f[3]) * inv);
    x[4] = static_cast<float>(static_cast<double>(f[4]) * inv * inv);
    x[5] = static_cast<float>(static_cast<double>(f[5]) * 0.05);
    x[6] = f[6];
    // size of the second-order (one coupling out and back) term relative to the
    // first-order denominator, squashed to [0, 1)
    const double ratio = static_cast<double>(f[4]) / (fabs(den) * fmax(fabs(static_cast<double>(f[1]) - theta), eps));
    x[7] = static_cast<float>(ratio / (1.0 + ratio));
}

// tanh(a) = 1 - 2 / (exp(2a) + 1), an exact identity, evaluated with the
// fast exponential and division intrinsics: a handful of instructions, about
// 1e-7 absolute error (all the activations need), and it saturates to +-1 for
// large |a| (the exponential overflows to inf or underflows to 0).
__device__ __forceinline__ float act_tanh(float a) { return 1.f - __fdividef(2.f, __expf(2.f * a) + 1.f); }

__device__ __forceinline__ float mlp_forward(const float *__restrict__ w, const float (&x)[IN], float (&h1)[HID],
                                             float (&h2)[HID]) {
#pragma unroll 4
    for (int o = 0; o < HID; ++o) {
        float a = w[OFF_B1 + o];
#pragma unroll
        for (int i = 0; i < IN; ++i) a = fmaf(w[OFF_W1 + o * IN + i], x[i], a);
        h1[o] = act_tanh(a);
    }
#pragma unroll 4
    for (int o = 0; o < HID; ++o) {
        float a = w[OFF_B2 + o];
#pragma unroll 8
        for (int i = 0; i < HID; ++i) a = fmaf(w[OFF_W2 + o * HID + i], h1[i], a);
        h2[o] = act_tanh(a);
    }
    float c = w[OFF_B3];
#pragma unroll 8
    for (int i = 0; i < HID; ++i) c = fmaf(w[OFF_W3 + i], h2[i], c);
    return c;
}

// Network output c for one input row without the activations: layer 1 is
// evaluated unit by unit with the layer-2 sums accumulated alongside, so no
// activation array is indexed at run time (mlp_forward's arrays, indexed in
// partly unrolled loops, live in local memory).  The same operations in the
// same order as mlp_forward, so the output is identical.
__device__ __forceinline__ float mlp_eval(const float *__restrict__ w, const float (&x)[IN]) {
    float a2[HID];
#pragma unroll
    for (int p = 0; p < HID; ++p) a2[p] = w[OFF_B2 + p];
#pragma unroll 2
    for (int o = 0; o < HID; ++o) {
        float a = w[OFF_B1 + o];
#pragma unroll
        for (int i = 0; i < IN; ++i) a = fmaf(w[OFF_W1 + o * IN + i], x[i], a);
        const float h = act_tanh(a);
#pragma unroll
        for (int p = 0; p < HID; ++p) a2[p] = fmaf(w[OFF_W2 + p * HID + o], h, a2[p]);
    }
    float c = w[OFF_B3];
#pragma unroll
    for (int p = 0; p < HID; ++p) c = fmaf(w[OFF_W3 + p], act_tanh(a2[p]), c);
    return c;
}

// Learned correction for k residual vectors: t_j = -exp(c) r_j / den with
// den = H_ii - theta_j (FP64 diagonal, clamped by eps, exactly as k_jacobi).
__global__ void k_mlp_precond(const void *__restrict__ R, int r64, uint64_t n, uint32_t k,
                              const float *__restrict__ feat, const double2 *__restrict__ diag,
                              const double *__restrict__ theta, double scale, double eps, float clamp,
                              const float *__restrict__ wglob, void *__restrict__ T, int t64) {
    __shared__ float w[NPARAM];
    for (int e = threadIdx.x; e < NPARAM; e += blockDim.x) w[e] = wglob[e];
    __syncthreads();
    for (uint64_t r = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; r < n;
         r += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const float *f = feat + r * TCP_FEATURES;
        const double d = diag[r].x;
        for (uint32_t j = 0; j < k; ++j) {
            float x[IN];
            double den_f;
            mlp_inputs(f, theta[j], scale, eps, x, den_f);
            double den = d - theta[j];
            if (fabs(den) < eps) den = den < 0.0 ? -eps : eps;
            const float c = fminf(fmaxf(mlp_eval(w, x), -clamp), clamp);
            const double2 v = load_c(R, r64, j * n + r);
            if (c == 0.f) {  // the Jacobi correction, rounded exactly as k_jacobi
                store_c(T, t64, j * n + r, make_double2(-v.x / den, -v.y / den));
            } else {
                const double g = -static_cast<double>(__expf(c)) / den;  // |c| <= clamp
                store_c(T, t64, j * n + r, make_double2(g * v.x, g * v.y));
            }
        }
    }
}

// Training: per sample s the network sees inputs X[s] (TCP_MLP_IN floats) and
// predicts c; the correction is g = -exp(c) / den[s].  With a = |r|^2 and
// b = Re(conj(e) r) (e: the exact correction), the sample loss is
// wt[s] * (g^2 a - 2 g b + |e|^2).  A block takes kTrainChunk samples at a
// time: each thread runs one sample forward and back to the hidden layers and
// stages its activations in shared memory, then every thread accumulates the
// weight gradients of the parameters it owns over the chunk (no atomics; the
// result is deterministic).  Each block writes its gradient partial sum.
constexpr int kTrainChunk = 128;
constexpr int kTrainStride = IN + 4 * HID + 1;  // x, h1, h2, dh1, dh2, dc
__global__ void __launch_bounds__(kTrainChunk)
    k_mlp_train(const float *__restrict__ X, const float *__restrict__ den, const float *__restrict__ a,
                const float *__restrict__ b, const float *__restrict__ e2, const float *__restrict__ wt,
                const float *__restrict__ dc_in, uint32_t count, const float *__restrict__ wglob,
                float *__restrict__ grad_partial, float *__restrict__ loss_partial) {
    __shared__ float w[NPARAM];
    __shared__ float act[kTrainChunk][kTrainStride];
    __shared__ float lsum[kTrainChunk];
    constexpr int kOwn = (NPARAM + kTrainChunk - 1) / kTrainChunk;
    for (int e = threadIdx.x; e < NPARAM; e += blockDim.x) w[e] = wglob[e];
    float gacc[kOwn];
#pragma unroll
    for (int q = 0; q < kOwn; ++q) gacc[q] = 0.f;
    float loss = 0.f;
    __syncthreads();
    const uint32_t chunks = (count + kTrainChunk - 1) / kTrainChunk;
    for (uint32_t ch = blockIdx.x; ch < chunks; ch += gridDim.x) {
        const uint32_t sidx = ch * kTrainChunk + threadIdx.x;
        float *my = act[threadIdx.x];
        if (sidx < count) {
            float x[IN], h1[HID], h2[HID];
#pragma unroll
            for (int i = 0; i < IN; ++i) x[i] = X[static_cast<size_t>(sidx) * IN + i];
            const float c = mlp_forward(w, x, h1, h2);
            float dc;
            if (dc_in != nullptr) {  // caller-supplied dL/dc (any loss on the outputs)
                dc = dc_in[sidx];
            } else {
                const float g = -expf(c) / den[sidx];
                const float as = a[sidx], bs = b[sidx], ws = wt[sidx];
                loss += ws * (g * g * as - 2.f * g * bs + e2[sidx]);
                dc = ws * (2.f * g * as - 2.f * bs) * g;  // dL/dc
            }
            float dh2[HID];
#pragma unroll
            for (int i = 0; i < HID; ++i) dh2[i] = dc * w[OFF_W3 + i] * (1.f - h2[i] * h2[i]);
#pragma unroll
            for (int i = 0; i < IN; ++i) my[i] = x[i];
#pragma unroll
            for (int i = 0; i < HID; ++i) {
                float d1 = 0.f;
#pragma unroll
                for (int o = 0; o < HID; ++o) d1 = fmaf(dh2[o], w[OFF_W2 + o * HID + i], d1);
                my[IN + i] = h1[i];
                my[IN + HID + i] = h2[i];
                my[IN + 2 * HID + i] = d1 * (1.f - h1[i] * h1[i]);
                my[IN + 3 * HID + i] = dh2[i];
            }
            my[IN + 4 * HID] = dc;
        } else {
            for (int i = 0; i < kTrainStride; ++i) my[i] = 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < kOwn; ++q) {
            const int pidx = threadIdx.x + q * kTrainChunk;
            if (pidx >= NPARAM) break;
            float acc = 0.f;
            if (pidx < OFF_B1) {  // W1[o][i] += dh1[o] * x[i]
                const int o = pidx / IN, i = pidx % IN;
                for (int r = 0; r < kTrainChunk; ++r) acc = fmaf(act[r][IN + 2 * HID + o], act[r][i], acc);
            } else if (pidx < OFF_W2) {  // b1[o]
                const int o = pidx - OFF_B1;
                for (int r = 0; r < kTrainChunk; ++r) acc += act[r][IN + 2 * HID + o];
            } else if (pidx < OFF_B2) {  // W2[o][i] += dh2[o] * h1[i]
                const int o = (pidx - OFF_W2) / HID, i = (pidx - OFF_W2) % HID;
                for (int r = 0; r < kTrainChunk; ++r) acc = fmaf(act[r][IN + 3 * HID + o], act[r][IN + i], acc);
            } else if (pidx < OFF_W3) {  // b2[o]
                const int o = pidx - OFF_B2;
                for (int r = 0; r < kTrainChunk; ++r) acc += act[r][IN + 3 * HID + o];
            } else if (pidx < OFF_B3) {  // w3[i] += dc * h2[i]
                const int i = pidx - OFF_W3;
                for (int r = 0; r < kTrainChunk; ++r) acc = fmaf(act[r][IN + 4 * HID], act[r][IN + HID + i], acc);
            } else {  // b3
                for (int r = 0; r < kTrainChunk; ++r) acc += act[r][IN + 4 * HID];
            }
            gacc[q] += acc;
        }
        __syncthreads();
    }
#pragma unroll
    for (int q = 0; q < kOwn; ++q) {
        const int pidx = threadIdx.x + q * kTrainChunk;
        if (pidx < NPARAM) grad_partial[static_cast<size_t>(blockIdx.x) * NPARAM + pidx] = gacc[q];
    }
    lsum[threadIdx.x] = loss;
    __syncthreads();
    if (threadIdx.x == 0) {
        float l = 0.f;
        for (int i = 0; i < kTrainChunk; ++i) l += lsum[i];
        loss_partial[blockIdx.x] = l;
    }
}

// Fixed-order sum of per-block losses.
__global__ void k_sum_losses(const float *__restrict__ partial, uint32_t blocks, float *__restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        float l = 0.f;
        for (uint32_t b = 0; b < blocks; ++b) l += partial[b];
        *out = l;
    }
}

// Network output c for every sample.
__global__ void k_mlp_forward(const float *__restrict__ X, uint32_t count, const float *__restrict__ wglob,
                              float *__restrict__ out) {
    __shared__ float w[NPARAM];
    for (int e = threadIdx.x; e < NPARAM; e += blockDim.x) w[e] = wglob[e];
    __syncthreads();
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < count; s += gridDim.x * blockDim.x) {
        float x[IN];
#pragma unroll
        for (int i = 0; i < IN; ++i) x[i] = X[static_cast<size_t>(s) * IN + i];
        out[s] = mlp_eval(w, x);
    }
}

// Sum the per-block gradient partials (fixed order) and apply one Adam step.
__global__ void k_adam(float *__restrict__ w, float *__restrict__ m, float *__restrict__ v,
                       const float *__restrict__ grad_partial, uint32_t blocks, float scale, float lr, float b1,
                       float b2, float eps, uint32_t step, float *__restrict__ grad_out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= NPARAM) return;
    float gsum = 0.f;
    for (uint32_t b = 0; b < blocks; ++b) gsum += grad_partial[static_cast<size_t>(b) * NPARAM + e];
    const float g = gsum * scale;
    if (grad_out) grad_out[e] = g;
    if (lr == 0.f) return;  // gradient only
    m[e] = b1 * m[e] + (1.f - b1) * g;
    v[e] = b2 * v[e] + (1.f - b2) * g * g;
    const float mh = m[e] / (1.f - powf(b1, static_cast<float>(step)));
    const float vh = v[e] / (1.f - powf(b2, static_cast<float>(step)));
    w[e] -= lr * mh / (sqrtf(vh) + eps);
}

// Network inputs and denominators for training samples taken from features.
__global__ void k_mlp_inputs(const float *__restrict__ feat, const uint64_t *__restrict__ rows, const double *__restrict__ theta,
                             const uint32_t *__restrict__ which, uint32_t count, double scale, double eps,
                             float *__restrict__ X, float *__restrict__ den) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < count; s += gridDim.x * blockDim.x) {
        float x[IN];
        double d;
        mlp_inputs(feat + rows[s] * TCP_FEATURES, theta[which[s]], scale, eps, x, d);
#pragma unroll
        for (int i = 0; i < IN; ++i) X[static_cast<size_t>(s) * IN + i] = x[i];
        den[s] = static_cast<float>(d);
    }
}

// ---------------------- alignment objective of the training ---------------------
// A training set s covers the states [seg_begin[s], seg_begin[s + 1]).  With
// g = -exp(clamp(c)) / den per state its sums are A = sum g alpha, B = sum g^2 a,
// C = sum g gamma, D = max(B - |C|^2, 1e-300), and its loss is
// 1 - |A|^2 / (E_s D): one minus the squared cosine between the correction
// g o r, made orthogonal to the Ritz vector, and the missing direction.  The
// objective is the mean over the sets.
constexpr int kAlignThreads = 256;
constexpr int kAlignWords = 6;  // A (2), B, C (2), loss per set

__device__ __forceinline__ double align_g(float c, float den, float clamp) {
    const double cc = fmin(fmax(static_cast<double>(c), -static_cast<double>(clamp)), static_cast<double>(clamp));
    return -exp(cc) / static_cast<double>(den);
}

// One block per set; a fixed-order tree reduction, so the sums do not depend
// on scheduling.
__global__ void __launch_bounds__(kAlignThreads)
    k_align_sums(const float *__restrict__ c, const float *__restrict__ den, const double2 *__restrict__ alpha,
                 const double *__restrict__ a, const double2 *__restrict__ gamma, const double *__restrict__ E,
                 const uint64_t *__restrict__ seg_begin, float clamp, double *__restrict__ sums) {
    __shared__ double red[5][kAlignThreads];
    const uint32_t s = blockIdx.x, t = threadIdx.x;
    double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0, v4 = 0.0;
    for (uint64_t i = seg_begin[s] + t; i < seg_begin[s + 1]; i += kAlignThreads) {
        const double g = align_g(c[i], den[i], clamp);
        const double2 al = alpha[i], ga = gamma[i];
        v0 += g * al.x;
        v1 += g * al.y;
        v2 += g * g * a[i];
        v3 += g * ga.x;
        v4 += g * ga.y;
    }
    red[0][t] = v0;
    red[1][t] = v1;
    red[2][t] = v2;
    red[3][t] = v3;
    red[4][t] = v4;
    __syncthreads();
    for (uint32_t stride = kAlignThreads / 2; stride > 0; stride >>= 1) {
        if (t < stride) {
#pragma unroll
            for (int k = 0; k < 5; ++k) red[k][t] += red[k][t + stride];
        }
        __syncthreads();
    }
    if (t == 0) {
        double *q = sums + static_cast<size_t>(s) * kAlignWords;
#pragma unroll
        for (int k = 0; k < 5; ++k) q[k] = red[k][0];
        const double D = fmax(red[2][0] - (red[3][0] * red[3][0] + red[4][0] * red[4][0]), 1e-300);
        const double A2 = red[0][0] * red[0][0] + red[1][0] * red[1][0];
        q[5] = 1.0 - A2 / (E[s] * D);
    }
}

// dL/dc per state (zero where the clamp is active).
__global__ void k_align_dc(const float *__restrict__ c, const float *__restrict__ den, const double2 *__restrict__ alpha,
                           const double *__restrict__ a, const double2 *__restrict__ gamma, const double *__restrict__ E,
                           const int64_t *__restrict__ seg, uint64_t count, uint32_t nsets, float clamp,
                           const double *__restrict__ sums, float *__restrict__ dc) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const int64_t s = seg[i];
        const double *q = sums + static_cast<size_t>(s) * kAlignWords;
        const double D = fmax(q[2] - (q[3] * q[3] + q[4] * q[4]), 1e-300);
        const double A2 = q[0] * q[0] + q[1] * q[1];
        const double g = align_g(c[i], den[i], clamp);
        const double2 al = alpha[i], ga = gamma[i];
        const double dA2 = 2.0 * (q[0] * al.x + q[1] * al.y);
        const double dD = 2.0 * g * a[i] - 2.0 * (q[3] * ga.x + q[4] * ga.y);
        const double dLdg = -(dA2 * D - A2 * dD) / (E[s] * D * D) / static_cast<double>(nsets);
        const float ci = c[i];
        dc[i] = (ci > -clamp && ci < clamp) ? static_cast<float>(dLdg * g) : 0.f;
    }
}

// Mean of the per-set losses, summed in set order.
__global__ void k_align_loss(const double *__restrict__ sums, uint32_t nsets, double *__restrict__ loss) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double l = 0.0;
        for (uint32_t s = 0; s < nsets; ++s) l += sums[static_cast<size_t>(s) * kAlignWords + 5];
        *loss = l / static_cast<double>(nsets);
    }
}

int grid_for(uint64_t n, int threads) {
    return static_cast<int>(std::min<uint64_t>((n + threads - 1) / threads, 148ull * 16));
}

bool valid_dtype(int d) { return d == TCP_DTYPE_C128 || d == TCP_DTYPE_C64; }

template <int QJ>
void launch_gram_tiles(int grid, size_t smem, cudaStream_t s, const void *A, bool a64, uint32_t p, const void *B,
                       bool b64, uint32_t q, uint64_t n, uint32_t groups, bool pairs_of_rows, double2 *partial) {
#define TCP_GRAM_LAUNCH(A64, B64, RPL)                                                                            \
    do {                                                                                                        \
        cudaFuncSetAttribute(k_gram_tiles<QJ, A64, B64, RPL>, cudaFuncAttributeMaxDynamicSharedMemorySize,       \
                             kGramRedBytes);                                                                    \
        k_gram_tiles<QJ, A64, B64, RPL><<<grid, kGramThreads, smem, s>>>(A, p, B, q, n, groups, partial);       \
    } while (0)
    if (a64 && b64 && pairs_of_rows) {
        TCP_GRAM_LAUNCH(true, true, 2);
    } else if (a64 && b64) {
        TCP_GRAM_LAUNCH(true, true, 1);
    } else if (a64) {
        TCP_GRAM_LAUNCH(true, false, 1);
    } else if (b64) {
        TCP_GRAM_LAUNCH(false, true, 1);
    } else {
        TCP_GRAM_LAUNCH(false, false, 1);
    }
#undef TCP_GRAM_LAUNCH
}

// cuTensorMapEncodeTiled from the driver, looked up once.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void *ptr = nullptr;
        cudaDriverEntryPointQueryResult qres;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &qres) != cudaSuccess ||
            qres != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return static_cast<PFN_cuTensorMapEncodeTiled_v12000>(nullptr);
        }
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
    }();
    return fn;
}

// Tensor map of `vecs` vectors of length n (element size es) seen as a 2-D
// array of 8-byte units; box = `rows` rows of every vector.
bool vector_block_map(CUtensorMap *map, const void *base, uint32_t vecs, uint64_t n, size_t es, uint32_t rows) {
    PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
    if (!encode) return false;
    const cuuint64_t dims[2] = {n * (es / 8), vecs};
    const cuuint64_t strides[1] = {n * es};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(rows * (es / 8)), vecs};
    const cuuint32_t elem_strides[2] = {1, 1};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<void *>(base), dims, strides, box, elem_strides,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The TMA-fed Gram for two complex128 blocks: 16-byte aligned vectors, at
// most 16 warp tiles, n * 8-byte units below 2^31.  Returns false (nothing
// launched) when those conditions do not hold.  Complex64 blocks take the
// register-fed kernel, which measured faster for them (3.1 against 2.6 TB/s
// at n = 2^24 with 64 + 4 vectors; both are bound by FP64 work, 16 FMAs and
// 2 conversions per 8-byte value), while complex128 gains 5.2 -> 5.7 TB/s.
// (The kernel template also reads complex64 blocks with n even.)
bool launch_gram_tma(const void *A, bool a64, uint32_t p, const void *B, bool b64, uint32_t q, uint64_t n,
                     uint32_t qj, uint32_t ntiles, cudaStream_t s, double2 *partial, uint32_t *grid_used) {
    if (a64 || b64 || ntiles > static_cast<uint32_t>(kGramWarps)) return false;
    const size_t es = a64 ? sizeof(float2) : sizeof(double2);
    if ((n * es) % 16 != 0 || n * (es / 8) >= (1ull << 31) || reinterpret_cast<uintptr_t>(A) % 16 != 0 ||
        reinterpret_cast<uintptr_t>(B) % 16 != 0)
        return false;
    const uint32_t vecs = p + q;
    // rows per chunk: a multiple of 32, one stage <= kGramStageBytes, a box
    // edge <= 256 units
    uint32_t rows = static_cast<uint32_t>(kGramStageBytes / (vecs * es)) / 32u * 32u;
    rows = std::min<uint32_t>(rows, static_cast<uint32_t>(256 / (es / 8)));
    if (rows < 32) return false;
    CUtensorMap ta, tb;
    if (!vector_block_map(&ta, A, p, n, es, rows) || !vector_block_map(&tb, B, q, n, es, rows)) return false;
    const uint32_t groups = std::max<uint32_t>(1u, std::min<uint32_t>(kGramWarps / ntiles, rows / 32u));
    const uint64_t chunks = n / rows;
    const int grid = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(kGramGrid, chunks)));
    const size_t smem = static_cast<size_t>(kGramStages) * vecs * rows * es;
#define TCP_GRAM_TMA(QJ, C64)                                                                                   \
    do {                                                                                                      \
        cudaFuncSetAttribute(k_gram_tma<QJ, C64>, cudaFuncAttributeMaxDynamicSharedMemorySize,                 \
                             static_cast<int>(kGramStages * kGramStageBytes));                                \
        k_gram_tma<QJ, C64><<<grid, kGramThreads, smem, s>>>(ta, tb, A, p, B, q, n, rows, groups, partial);   \
    } while (0)
    if (qj == 1) {
        TCP_GRAM_TMA(1, false);
    } else if (qj == 2) {
        TCP_GRAM_TMA(2, false);
    } else {
        TCP_GRAM_TMA(4, false);
    }
#undef TCP_GRAM_TMA
    *grid_used = static_cast<uint32_t>(grid);
    return true;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" size_t tcp_gram_work_bytes(uint32_t p, uint32_t q) {
    return static_cast<size_t>(kGramBlocks) * p * q * sizeof(double2);
}

extern "C" int tcp_gram(const void *A, int a_dtype, uint32_t p, const void *B, int b_dtype, uint32_t q, uint64_t n,
                        void *d_G, void *d_work, void *stream) {
    if (!valid_dtype(a_dtype) || !valid_dtype(b_dtype)) return fail(TCP_ERR_INVALID_ARGUMENT, "unknown dtype");
    if (p == 0 || q == 0) return TCP_OK;
    if (p + q > kGramMaxVectors || p * q > kGramMaxPairs) {
        return fail(TCP_ERR_INVALID_ARGUMENT, "tcp_gram supports p + q <= 96 and p * q <= 512");
    }
    if (!A || !B || !d_G || !d_work) return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    auto *partial = static_cast<double2 *>(d_work);
    const uint32_t qj = q == 1 ? 1u : (q == 2 ? 2u : 4u);
    const uint32_t pi = qj == 4 ? 4u : 8u;  // tile shape of k_gram_tiles<qj>
    const uint32_t ntiles = ((p + pi - 1) / pi) * ((q + qj - 1) / qj);
    const bool a64 = a_dtype == TCP_DTYPE_C64, b64 = b_dtype == TCP_DTYPE_C64;
    uint32_t grid_used = 0;
    if (launch_gram_tma(A, a64, p, B, b64, q, n, qj, ntiles, s, partial, &grid_used)) {
        const uint32_t pairs = p * q;
        k_gram_reduce<<<(pairs + 127) / 128, 128, 0, s>>>(partial, grid_used, pairs, static_cast<double2 *>(d_G));
        cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? TCP_OK : cuda_fail(e, "gram kernel launch");
    }
    // Register-fed tiles (mixed storage types, odd complex64 lengths, more
    // than 16 tiles).  Row groups per CTA: slots = ntiles * groups =
    // lcm(ntiles, 16) keeps all 16 warps equally busy; if those partial sums
    // do not fit in shared memory, fall back to 16 / ntiles groups (or one).
    const uint32_t tp = pi * qj;
    uint32_t groups = kGramWarps / std::gcd(ntiles, static_cast<uint32_t>(kGramWarps));
    if (static_cast<size_t>(groups) * ntiles * tp * sizeof(double2) > static_cast<size_t>(kGramRedBytes))
        groups = ntiles >= static_cast<uint32_t>(kGramWarps) ? 1u : kGramWarps / ntiles;
    const size_t smem = groups > 1 ? static_cast<size_t>(groups) * ntiles * tp * sizeof(double2) : 0;
    const bool pairs_of_rows = a64 && b64 && n % 2 == 0 && reinterpret_cast<uintptr_t>(A) % 16 == 0 &&
                               reinterpret_cast<uintptr_t>(B) % 16 == 0;
    const uint64_t rows_per_chunk = pairs_of_rows ? 64 : 32;
    const uint64_t chunks = (n + rows_per_chunk - 1) / rows_per_chunk;
    const int grid = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(kGramGrid, (chunks + groups - 1) / groups)));
    if (qj == 1) {
        launch_gram_tiles<1>(grid, smem, s, A, a64, p, B, b64, q, n, groups, pairs_of_rows, partial);
    } else if (qj == 2) {
        launch_gram_tiles<2>(grid, smem, s, A, a64, p, B, b64, q, n, groups, pairs_of_rows, partial);
    } else {
        launch_gram_tiles<4>(grid, smem, s, A, a64, p, B, b64, q, n, groups, pairs_of_rows, partial);
    }
    const uint32_t pairs = p * q;
    k_gram_reduce<<<(pairs + 127) / 128, 128, 0, s>>>(partial, static_cast<uint32_t>(grid), pairs,
                                                      static_cast<double2 *>(d_G));
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "gram kernel launch");
}

extern "C" int tcp_block_combine(const void *A, int a_dtype, uint32_t p, const void *d_S, uint32_t k, uint64_t n,
                                 double alpha, double beta, void *out, int out_dtype, void *stream) {
    if (!valid_dtype(a_dtype) || !valid_dtype(out_dtype)) return fail(TCP_ERR_INVALID_ARGUMENT, "unknown dtype");
    if (k == 0) return TCP_OK;
    if (k > static_cast<uint32_t>(kCombineMaxK)) return fail(TCP_ERR_INVALID_ARGUMENT, "tcp_block_combine supports k <= 32");
    uint32_t njp = 1;
    while (njp * kCombineTile < k) njp <<= 1;
    const size_t smem = static_cast<size_t>(p) * njp * kCombineTile * sizeof(double2);
    if (smem > 96 * 1024) return fail(TCP_ERR_INVALID_ARGUMENT, "coefficient block too large");
    if (!A || !d_S || !out) return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    if (n == 0) return TCP_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint32_t rb = kCombineThreads / njp;
    const int grid = static_cast<int>(std::min<uint64_t>((n + rb - 1) / rb, 148ull * 8));
    const bool a64 = a_dtype == TCP_DTYPE_C64, o64 = out_dtype == TCP_DTYPE_C64;
    const auto *S = static_cast<const double2 *>(d_S);
    if (a64 && o64) {
        cudaFuncSetAttribute(k_combine_tiles<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
        k_combine_tiles<true, true><<<grid, kCombineThreads, smem, s>>>(A, p, S, k, njp, n, alpha, beta, out);
    } else if (a64) {
        cudaFuncSetAttribute(k_combine_tiles<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
        k_combine_tiles<true, false><<<grid, kCombineThreads, smem, s>>>(A, p, S, k, njp, n, alpha, beta, out);
    } else if (o64) {
        cudaFuncSetAttribute(k_combine_tiles<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
        k_combine_tiles<false, true><<<grid, kCombineThreads, smem, s>>>(A, p, S, k, njp, n, alpha, beta, out);
    } else {
        cudaFuncSetAttribute(k_combine_tiles<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
        k_combine_tiles<false, false><<<grid, kCombineThreads, smem, s>>>(A, p, S, k, njp, n, alpha, beta, out);
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "combine kernel launch");
}

extern "C" int tcp_precond_jacobi(const void *R, int r_dtype, uint64_t n, uint32_t k, const void *d_diag,
                                  const double *d_theta, double eps, void *T, int t_dtype, void *stream) {
    if (!valid_dtype(r_dtype) || !valid_dtype(t_dtype)) return fail(TCP_ERR_INVALID_ARGUMENT, "unknown dtype");
    if (!R || !d_diag || !d_theta || !T) return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    k_jacobi<<<grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        R, r_dtype == TCP_DTYPE_C64, n, k, static_cast<const double2 *>(d_diag), d_theta, eps, T, t_dtype == TCP_DTYPE_C64);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "jacobi kernel launch");
}

extern "C" int tcp_state_features(const tcp_mvp_plan *plan, float *d_features, uint64_t n, void *stream) {
    int st = tcp::check_plan(plan);
    if (st) return st;
    if (n != plan->dim) return tcp::length_error(plan->dim, n);
    if (!d_features) return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    const tcp::Schedule &h = plan->sched.host;
    uint32_t gzero = 0xffffffffu;
    for (size_t g = 0; g < h.g_mask.size(); ++g)
        if (h.g_mask[g] == 0) gzero = static_cast<uint32_t>(g);
    k_features<<<grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(plan->sched.dev, gzero, plan->nqubits, n,
                                                                              d_features);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "feature kernel launch");
}

extern "C" int tcp_precond_mlp(const void *R, int r_dtype, uint64_t n, uint32_t k, const float *d_features,
                               const void *d_diag, const double *d_theta, double scale, double eps, float clamp,
                               const float *d_params, void *T, int t_dtype, void *stream) {
    if (!valid_dtype(r_dtype) || !valid_dtype(t_dtype)) return fail(TCP_ERR_INVALID_ARGUMENT, "unknown dtype");
    if (!R || !d_features || !d_diag || !d_theta || !d_params || !T) return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    k_mlp_precond<<<grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        R, r_dtype == TCP_DTYPE_C64, n, k, d_features, static_cast<const double2 *>(d_diag), d_theta, scale, eps, clamp,
        d_params, T, t_dtype == TCP_DTYPE_C64);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "mlp preconditioner launch");
}

extern "C" int tcp_mlp_inputs(const float *d_features, const uint64_t *d_rows, const double *d_theta,
                              const uint32_t *d_which, uint32_t count, double scale, double eps, float *d_X,
                              float *d_den, void *stream) {
    if (!d_features || !d_rows || !d_theta || !d_which || !d_X || !d_den) return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    if (count == 0) return TCP_OK;
    k_mlp_inputs<<<grid_for(count, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(d_features, d_rows, d_theta, d_which,
                                                                                   count, scale, eps, d_X, d_den);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "mlp input kernel launch");
}

extern "C" int tcp_mlp_forward(const float *d_X, uint32_t count, const float *d_params, float *d_out, void *stream) {
    if (!d_X || !d_params || !d_out) return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    if (count == 0) return TCP_OK;
    k_mlp_forward<<<grid_for(count, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(d_X, count, d_params, d_out);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "mlp forward launch");
}

extern "C" int tcp_mlp_backward_step(const float *d_X, const float *d_dc, uint32_t count, float *d_params, float *d_m,
                                     float *d_v, float *d_work, float lr, uint32_t step, float *d_grad_out,
                                     void *stream) {
    if (!d_X || !d_dc || !d_params || !d_work) return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    if (lr != 0.f && (!d_m || !d_v || step == 0)) return fail(TCP_ERR_INVALID_ARGUMENT, "Adam state missing");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    float *grad_partial = d_work;
    float *loss_partial = d_work + static_cast<size_t>(TCP_MLP_TRAIN_BLOCKS) * TCP_MLP_PARAMS;
    k_mlp_train<<<TCP_MLP_TRAIN_BLOCKS, kTrainChunk, 0, s>>>(d_X, nullptr, nullptr, nullptr, nullptr, nullptr, d_dc,
                                                             count, d_params, grad_partial, loss_partial);
    k_adam<<<(TCP_MLP_PARAMS + 255) / 256, 256, 0, s>>>(d_params, d_m, d_v, grad_partial, TCP_MLP_TRAIN_BLOCKS, 1.f, lr,
                                                       0.9f, 0.999f, 1e-8f, step, d_grad_out);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "mlp backward launch");
}

extern "C" size_t tcp_mlp_train_work_bytes(void) {
    return static_cast<size_t>(TCP_MLP_TRAIN_BLOCKS) * (TCP_MLP_PARAMS + 1) * sizeof(float);
}

extern "C" int tcp_mlp_train_step(const float *d_X, const float *d_den, const float *d_a, const float *d_b,
                                  const float *d_e2, const float *d_wt, uint32_t count, float *d_params, float *d_m,
                                  float *d_v, float *d_work, float lr, uint32_t step, float *d_grad_out,
                                  float *d_loss_out, void *stream) {
    if (!d_X || !d_den || !d_a || !d_b || !d_e2 || !d_wt || !d_params || !d_work) {
        return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    }
    if (lr != 0.f && (!d_m || !d_v || step == 0)) return fail(TCP_ERR_INVALID_ARGUMENT, "Adam state missing");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    float *grad_partial = d_work;
    float *loss_partial = d_work + static_cast<size_t>(TCP_MLP_TRAIN_BLOCKS) * TCP_MLP_PARAMS;
    k_mlp_train<<<TCP_MLP_TRAIN_BLOCKS, kTrainChunk, 0, s>>>(d_X, d_den, d_a, d_b, d_e2, d_wt, nullptr, count,
                                                             d_params, grad_partial, loss_partial);
    k_adam<<<(TCP_MLP_PARAMS + 255) / 256, 256, 0, s>>>(d_params, d_m, d_v, grad_partial, TCP_MLP_TRAIN_BLOCKS, 1.f, lr,
                                                       0.9f, 0.999f, 1e-8f, step, d_grad_out);
    if (d_loss_out) k_sum_losses<<<1, 32, 0, s>>>(loss_partial, TCP_MLP_TRAIN_BLOCKS, d_loss_out);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "mlp training launch");
}

extern "C" size_t tcp_mlp_alignment_work_bytes(uint32_t nsets) {
    return static_cast<size_t>(nsets) * kAlignWords * sizeof(double);
}

extern "C" int tcp_mlp_alignment_grad(const float *d_c, const float *d_den, const void *d_alpha, const double *d_a,
                                      const void *d_gamma, const double *d_E, const int64_t *d_seg,
                                      const uint64_t *d_seg_begin, uint32_t nsets, uint64_t count, float clamp,
                                      double *d_work, float *d_dc, double *d_loss, void *stream) {
    if (!d_c || !d_den || !d_alpha || !d_a || !d_gamma || !d_E || !d_seg || !d_seg_begin || !d_work || !d_dc) {
        return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    }
    if (nsets == 0) return fail(TCP_ERR_INVALID_ARGUMENT, "the alignment objective needs at least one set");
    if (!(clamp > 0.f)) return fail(TCP_ERR_INVALID_ARGUMENT, "clamp must be positive");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_align_sums<<<nsets, kAlignThreads, 0, s>>>(d_c, d_den, static_cast<const double2 *>(d_alpha), d_a,
                                                 static_cast<const double2 *>(d_gamma), d_E, d_seg_begin, clamp, d_work);
    if (count > 0) {
        k_align_dc<<<grid_for(count, 256), 256, 0, s>>>(d_c, d_den, static_cast<const double2 *>(d_alpha), d_a,
                                                       static_cast<const double2 *>(d_gamma), d_E, d_seg, count, nsets,
                                                       clamp, d_work, d_dc);
    }
    if (d_loss) k_align_loss<<<1, 32, 0, s>>>(d_work, nsets, d_loss);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "alignment gradient launch");
}
