// libtcpmvp.so -- sm_100a kernels and the C ABI of the matrix-free Pauli MVP.
//
// Kernels (all hand-written for sm_100a):
//   k_tiled     tile-staged grouped MVP.  One CTA owns an output tile of
//               2^S consecutive rows and keeps its accumulators in registers;
//               for every outer pattern d ("step") the source tile
//               (tile ^ d) is copied into shared memory by the TMA bulk-copy
//               engine (cp.async.bulk + mbarrier, double-buffered), and every
//               x-mask group of that step is applied from shared memory:
//               D_m(c) = sum_{k in m} w_k (-1)^{popcount(z_k & c)} evaluated
//               at the source column c = r ^ m, then y[r] += D_m(c) x[c].
//               FP64 (complex128) and FP32-with-Kahan (complex64) variants.
//   k_rowwise   one thread per row, direct gathers; for states smaller than
//               one tile and for buffers the bulk-copy engine cannot address.
//   k_transitions / k_diagonal   eager transition count and H_ii extraction.
//
// Reference semantics (paths inside the reference project):
//   crates/tencir-pauli-core/src/hamiltonian.rs:204-270 (apply_into),
//   :121-139 (eager diagonal), :166-179 (transition_count).
#include <cuda_runtime.h>

#include <algorithm>
#include <condition_variable>
#include <cstdlib>
#include <thread>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "tcp_internal.h"

using tcp::fail;

#include "tcp_device.cuh"
#include "tcp_plan_impl.h"
#include "tcp_ring.cuh"

using namespace tcpdev;

namespace {

// --------------------------------- kernels ---------------------------------
// One term applied to the thread's E rows.  `rec` is the term record's first
// 16 bytes (zlo | (pattern | kind << 24) << 32, zt); `w` its weight with the
// per-step and per-group signs already folded in.  The remaining sign,
// parity(zlo & tid) ^ parity(zt & tile), is one POPC of an XOR (the parity of
// a XOR equals the XOR of the parities).
template <int JH, int LOGE, typename R>
__device__ __forceinline__ void apply_term(ulonglong2 rec, typename Cx<R>::T w, uint32_t tid, uint64_t tile,
                                           const typename Cx<R>::T (&xv)[1 << LOGE], Acc<R> (&acc)[1 << LOGE]) {
    constexpr int E = 1 << LOGE;
    constexpr uint32_t kPatMask = (1u << E) - 1u;
    const uint32_t lo = static_cast<uint32_t>(rec.x);
    const uint32_t hi = static_cast<uint32_t>(rec.x >> 32);
    const uint64_t zt_tile = rec.y & tile;
    const uint32_t base =
        __popc((lo & tid) ^ static_cast<uint32_t>(zt_tile) ^ static_cast<uint32_t>(zt_tile >> 32)) & 1u;
    const uint32_t pattern = hi & kPatMask;
    const uint32_t kind = hi >> 24;
    if (pattern == 0u) {
        const R wr = flip_by(w.x, base), wi = flip_by(w.y, base);
        if (kind == tcp::kKindReal) {
#pragma unroll
            for (int jj = 0; jj < E; ++jj) acc[jj ^ JH].add_real(wr, xv[jj]);
        } else if (kind == tcp::kKindImag) {
#pragma unroll
            for (int jj = 0; jj < E; ++jj) acc[jj ^ JH].add_imag(wi, xv[jj]);
        } else {
#pragma unroll
            for (int jj = 0; jj < E; ++jj) acc[jj ^ JH].add_complex(wr, wi, xv[jj]);
        }
    } else {
        const uint32_t pat = (pattern ^ (0u - base)) & kPatMask;  // sign bit of every source jj
        if (kind == tcp::kKindReal) {
#pragma unroll
            for (int jj = 0; jj < E; ++jj) acc[jj ^ JH].add_real(flip_if(w.x, pat, jj), xv[jj]);
        } else if (kind == tcp::kKindImag) {
#pragma unroll
            for (int jj = 0; jj < E; ++jj) acc[jj ^ JH].add_imag(flip_if(w.y, pat, jj), xv[jj]);
        } else {
#pragma unroll
            for (int jj = 0; jj < E; ++jj)
                acc[jj ^ JH].add_complex(flip_if(w.x, pat, jj), flip_if(w.y, pat, jj), xv[jj]);
        }
    }
}

// Terms of one x-mask group applied to the thread's E rows.  JH is a
// compile-time row permutation between the loaded values and the rows; the
// tiled kernel loads its values in row order already (JH = 0).
// Term records come from the step block in shared memory; a term whose z mask
// has no bit among the thread's row bits (pattern 0) has one sign for all E
// rows, otherwise the sign of source jj is bit jj of the pattern.
template <int JH, int LOGE, typename R>
__device__ __forceinline__ void apply_group(const unsigned char *__restrict__ trm, uint32_t tb, uint32_t te,
                                            uint32_t tid, uint64_t tile, const typename Cx<R>::T (&xv)[1 << LOGE],
                                            Acc<R> (&acc)[1 << LOGE]) {
    for (uint32_t t = tb; t < te; ++t) {
        const unsigned char *r0 = trm + t * tcp::kTermRecBytes;
        apply_term<JH, LOGE, R>(*reinterpret_cast<const ulonglong2 *>(r0), record_weight<R>(r0), tid, tile, xv, acc);
    }
}

// Source values of one group for the thread, in row order: row j of the
// thread (tile row tid + j * T) reads source tile row (tid ^ m_lo) +
// (j ^ jh) * T, where m_lo and jh are the group's inner-mask bits at and
// above the thread index.
template <int LOGE, typename C>
__device__ __forceinline__ void load_group(const C *__restrict__ xs, uint32_t tid, uint32_t m, C (&xv)[1 << LOGE]) {
    const C *src = xs + (tid ^ (m & (kThreads - 1)));
    const uint32_t jh = m >> kLogThreads;
#pragma unroll
    for (int j = 0; j < (1 << LOGE); ++j) xv[j] = src[(static_cast<uint32_t>(j) ^ jh) << kLogThreads];
}

template <typename R> __device__ __forceinline__ const unsigned char *step_blocks(const DevSchedule &s);
template <> __device__ __forceinline__ const unsigned char *step_blocks<double>(const DevSchedule &s) {
    return s.blocks128;
}
template <> __device__ __forceinline__ const unsigned char *step_blocks<float>(const DevSchedule &s) {
    return s.blocks64;
}

// Issue the bulk copies of one step (source tile + step block) on one mbarrier.
template <typename C, uint32_t S>
__device__ __forceinline__ void issue_step(const uint4 info, uint64_t tile, const C *__restrict__ x,
                                           const unsigned char *__restrict__ blocks, C *tile_dst,
                                           unsigned char *blk_dst, uint64_t *bar) {
    constexpr uint32_t BYTES = (1u << S) * sizeof(C);
    const uint64_t d = static_cast<uint64_t>(info.x) | (static_cast<uint64_t>(info.y) << 32);
    const uint32_t blk_bytes = (info.w >> 16) * 16u;
    mbar_arrive_expect_tx(bar, BYTES + blk_bytes);
    bulk_copy_g2s(tile_dst, x + ((tile ^ d) << S), BYTES, bar);
    bulk_copy_g2s(blk_dst, blocks + static_cast<size_t>(info.z) * 16u, blk_bytes, bar);
}

// Tile-staged grouped MVP (see file header).  Grid: one CTA per output tile;
// thread t owns rows t + j * kThreads of the tile.  Shared memory: two source
// tiles and two step blocks (double buffering), refilled by the TMA engine.
// PASSES = false runs every step and overwrites y.  PASSES = true runs pass
// `pass` (0..kPassChunks-1): only the steps whose source tiles lie in part
// `pass` of the state (see DevSchedule::pass_begin), adding to y when
// `accumulate`.
template <int LOGE, typename R, bool PASSES>
__global__ void __launch_bounds__(kThreads, 1)
    k_tiled(DevSchedule s, const typename Cx<R>::T *__restrict__ x, typename Cx<R>::T *__restrict__ y,
            int *__restrict__ err, uint64_t tile0, uint32_t pass, uint32_t accumulate) {
    using C = typename Cx<R>::T;
    static_assert(LOGE == 3, "the group dispatch below covers 8 rows per thread");
    constexpr int E = 1 << LOGE;
    constexpr int S = kLogThreads + LOGE;
    constexpr uint32_t TILE = 1u << S;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    C *tiles = reinterpret_cast<C *>(smem_raw);
    unsigned char *blks = smem_raw + 2 * TILE * sizeof(C);
    __shared__ __align__(8) uint64_t bars[2];

    const uint32_t tid = threadIdx.x;
    const uint64_t tile = tile0 + blockIdx.x;
    uint32_t step0 = 0, nsteps = s.nsteps;
    if constexpr (PASSES) {
        uint32_t b0, b1;
        pass_range(s.pass_begin, s.pass_shift, tile, pass, b0, b1);
        step0 = b0;
        nsteps = b1 - b0;
    }
    const uint4 *steps = s.step_info + step0;
    const unsigned char *blocks = step_blocks<R>(s);

    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0 && nsteps > 0) issue_step<C, S>(__ldg(&steps[0]), tile, x, blocks, tiles, blks, &bars[0]);

    Acc<R> acc[E];
    for (uint32_t st = 0; st < nsteps; ++st) {
        const uint32_t b = st & 1u;
        const uint4 info = __ldg(&steps[st]);
        const bool ok = mbar_wait_bounded(&bars[b], (st >> 1) & 1u);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicOr(err, kErrTimeout);
            return;
        }
        // Every thread has finished step st-1, so the other buffers are free.
        if (tid == 0 && st + 1 < nsteps) {
            fence_proxy_async_smem();
            issue_step<C, S>(__ldg(&steps[st + 1]), tile, x, blocks, tiles + (b ^ 1u) * TILE,
                             blks + (b ^ 1u) * tcp::kBlockBytesMax, &bars[b ^ 1u]);
        }
        const C *xs = tiles + b * TILE;
        const unsigned char *blk = blks + b * tcp::kBlockBytesMax;
        const uint32_t ng = info.w & 0xffffu;
        const uint4 *grp = reinterpret_cast<const uint4 *>(blk);
        const unsigned char *trm = blk + ng * tcp::kGroupRecBytes;
        for (uint32_t g = 0; g < ng; ++g) {
            const uint4 gr = grp[g];
            C xv[E];
            load_group<LOGE>(xs, tid, gr.x, xv);
            apply_group<0, LOGE, R>(trm, gr.y, gr.z, tid, tile, xv, acc);
            // FP32: fold the running group sum into the compensated row sum
            // every kCompensateGroups groups and at the end of the step.
            if (((g + 1) % kCompensateGroups) == 0u || g + 1 == ng) {
#pragma unroll
                for (int j = 0; j < E; ++j) acc[j].compensate();
            }
        }
    }
    C *yt = y + (tile << S);
    if (accumulate) {
#pragma unroll
        for (int j = 0; j < E; ++j) {
            C &out = yt[tid + (j << kLogThreads)];
            const C v = acc[j].value();
            out.x += v.x;
            out.y += v.y;
        }
    } else {
#pragma unroll
        for (int j = 0; j < E; ++j) yt[tid + (j << kLogThreads)] = acc[j].value();
    }
}

// ------------------------------- ring kernel --------------------------------
// k_ring: the tiled MVP with a ring of source tiles.
//  * Sixteen warps own the output tile's 4096 rows (thread t: rows
//    t + j * 512, j = 0..7) and keep their sums in registers.  Per step they
//    wait for its stage ("full" mbarrier), walk its cosets -- one row-ordered
//    load of 8 source values per coset -- and apply every group of the coset
//    through a compile-time register permutation a (row j reads loaded value
//    j ^ a).  Then each warp releases the stage with one arrive ("empty").
//  * Thread 0 is also the producer: whenever a stage is released by every
//    warp it has the TMA bulk-copy engine refill it with a later step's
//    source tile (tile ^ d) and block.  It only tests the empty barriers
//    (never waits on them), at each step and while its own warp waits for
//    data, so no warp is set aside for issuing copies and no CTA-wide barrier
//    runs after set-up: warps drift apart by up to the ring depth.
//  * Every wait is bounded (2 s) and also ends when another thread raised the
//    CTA's abort word; the kernel then records kErrTimeout, and thread 0
//    waits (bounded) for the last fill of every stage before the block exits,
//    so no copy is left writing into a finished block's memory.
#ifdef TCP_DEBUG_BOUNDS
// A block stays inside its `bytes`: header, coset records, group words and
// the records they count; thread-bit masks below 512, permutations below 8.
__device__ __forceinline__ bool ring_block_in_bounds(uint4 hdr, const uint4 *cos, const uint32_t *gw, uint32_t bytes) {
    if (bytes > tcp::kRingBlockBytes || 16u + 16u * hdr.x + 4u * hdr.y > 16u * hdr.z || 16u * hdr.z > bytes) return false;
    uint32_t groups = 0, records = 0;
    for (uint32_t c = 0; c < hdr.x; ++c) {
        if (cos[c].x >= 512u || cos[c].y != 0u) return false;
        groups += cos[c].z;
    }
    if (groups != hdr.y) return false;
    for (uint32_t g = 0; g < groups; ++g) records += gw[g] >> 4;
    return 16u * hdr.z + 16u * records <= bytes;
}
#endif

// Issue the fill of ring step `i` (source tile and block) into its stage.
template <typename R>
__device__ __forceinline__ void ring_fill(const DevSchedule &s, const typename Cx<R>::T *__restrict__ x,
                                          uint64_t tile, const uint4 *__restrict__ info, uint32_t i,
                                          unsigned char *smem, uint64_t *full) {
    constexpr uint32_t K = RingDepth<R>::K;
    constexpr uint32_t TILE_BYTES = ring_tile_bytes<R>();
    const uint32_t st = i % K;
    const uint4 in = __ldg(&info[i]);
    const uint64_t d = static_cast<uint64_t>(in.x) | (static_cast<uint64_t>(in.y) << 32);
    const uint32_t blk_bytes = in.w * 16u;
    unsigned char *dst = smem + st * ring_stage_bytes<R>();
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&full[st], TILE_BYTES + blk_bytes);
    bulk_copy_g2s(dst, x + ((tile ^ d) << kTileBitsC128), TILE_BYTES, &full[st]);
    bulk_copy_g2s(dst + TILE_BYTES, ring_blocks<R>(s) + static_cast<size_t>(in.z) * 16u, blk_bytes, &full[st]);
}

template <typename R, bool PASSES, bool RHS_BLOCK = false>
__global__ void __launch_bounds__(RingShape<R>::kThreadsPerCta, 1)
    k_ring(DevSchedule s, const typename Cx<R>::T *__restrict__ x, typename Cx<R>::T *__restrict__ y,
           int *__restrict__ err, uint64_t tile0, uint32_t pass, uint32_t accumulate, uint64_t rhs_stride) {
    using C = typename Cx<R>::T;
    constexpr uint32_t K = RingDepth<R>::K;
    constexpr uint32_t TILE_BYTES = ring_tile_bytes<R>();
    constexpr uint32_t STAGE = ring_stage_bytes<R>();
    constexpr bool kProducerWarp = RingShape<R>::kProducerWarp;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[K];
    __shared__ __align__(8) uint64_t empty[K];
    __shared__ uint32_t released[K];
    __shared__ uint32_t issued_end;
    __shared__ int abort_word;

    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31u;
    const uint64_t tile = tile0 + blockIdx.x;
    if constexpr (RHS_BLOCK) {
        // blockIdx.y selects the right-hand side of an RHS-major block (a
        // separate instantiation, so the single-vector kernel keeps its
        // registers)
        x += blockIdx.y * rhs_stride;
        y += blockIdx.y * rhs_stride;
    }
    uint32_t step0 = 0, nsteps = s.ring_steps;
    if constexpr (PASSES) {
        uint32_t b0, b1;
        pass_range(s.ring_pass_begin, s.ring_pass_shift, tile, pass, b0, b1);
        step0 = b0;
        nsteps = b1 - b0;
    }
    const uint4 *info = s.ring_info + step0;
    if (tid == 0) {
#pragma unroll
        for (uint32_t k = 0; k < K; ++k) {
            mbar_init(&full[k], 1);
            mbar_init(&empty[k], kRingWarps);
            released[k] = 0;
        }
        abort_word = 0;
        fence_mbar_init();
        if constexpr (!kProducerWarp) {
            const uint32_t first = nsteps < K ? nsteps : K;
            for (uint32_t i = 0; i < first; ++i) ring_fill<R>(s, x, tile, info, i, smem_raw, full);
            issued_end = first;
        }
    }
    __syncthreads();
    volatile int *abort_flag = &abort_word;

    if constexpr (kProducerWarp) {
        if (tid >= kRingWarps * 32u) {
            // ---------------- producer warp (lane 0 issues) ----------------
            if (tid != kRingWarps * 32u) return;
            uint32_t issued = 0;
            for (uint32_t st = 0; st < nsteps; ++st) {
                if (st >= K && !mbar_wait_or_abort(&empty[st % K], ((st / K) - 1u) & 1u, abort_flag)) {
                    atomicOr(err, kErrTimeout);
                    *abort_flag = 1;
                    break;
                }
                ring_fill<R>(s, x, tile, info, st, smem_raw, full);
                issued = st + 1;
            }
            // the last fill issued into each stage has landed before this returns
            for (uint32_t i = issued > K ? issued - K : 0u; i < issued; ++i)
                mbar_wait_bounded(&full[i % K], (i / K) & 1u);
            return;
        }
    }

    // ---------------- row warps ----------------
    const uint32_t tile32 = static_cast<uint32_t>(tile);
    RingAcc<R> acc[8];
    uint32_t stage = 0, phase = 0, since = 0;
    for (uint32_t st = 0; st < nsteps; ++st) {
        const bool landed = mbar_wait_or_abort(&full[stage], phase, abort_flag);
        if (__any_sync(0xffffffffu, !landed)) {
            if (lane == 0u) {
                atomicOr(err, kErrTimeout);
                *abort_flag = 1;
                if constexpr (!kProducerWarp) {
                    // every fill issued so far has landed (bounded) before
                    // the block may exit
                    const uint32_t end = *reinterpret_cast<volatile uint32_t *>(&issued_end);
                    for (uint32_t i = end > K ? end - K : 0u; i < end; ++i)
                        mbar_wait_bounded(&full[i % K], (i / K) & 1u);
                }
            }
            return;
        }
        const C *xs = reinterpret_cast<const C *>(smem_raw + stage * STAGE);
        const unsigned char *blk = smem_raw + stage * STAGE + TILE_BYTES;
        uint4 hdr = *reinterpret_cast<const uint4 *>(blk);
        const uint4 *cos = reinterpret_cast<const uint4 *>(blk + 16);
        const uint32_t *gw = reinterpret_cast<const uint32_t *>(blk + 16u + hdr.x * 16u);
        const uint4 *trm = reinterpret_cast<const uint4 *>(blk + hdr.z * 16u);
#ifdef TCP_DEBUG_BOUNDS
        // debug builds check every block against its stage before walking it
        // and skip (recording kErrBounds) a block that would read outside it
        if (!ring_block_in_bounds(hdr, cos, gw, __ldg(&info[st]).w * 16u)) {
            if (lane == 0u) atomicOr(err, kErrBounds);
            hdr.x = 0u;
        }
#endif
        uint32_t g = 0;
        for (uint32_t c = 0; c < hdr.x; ++c) {
            const uint4 cr = cos[c];
            C xv[8];
            const C *src = xs + (tid ^ cr.x);
#pragma unroll
            for (int j = 0; j < 8; ++j) xv[j] = src[static_cast<uint32_t>(j) << kLogThreads];
            for (uint32_t k = 0; k < cr.z; ++k, ++g) {
                const uint32_t word = gw[g];
                const uint32_t nt = word >> 4;
                switch (word & 7u) {
                case 0: ring_group<0, R>(trm, nt, tid, tile32, xv, acc); break;
                case 1: ring_group<1, R>(trm, nt, tid, tile32, xv, acc); break;
                case 2: ring_group<2, R>(trm, nt, tid, tile32, xv, acc); break;
                case 3: ring_group<3, R>(trm, nt, tid, tile32, xv, acc); break;
                case 4: ring_group<4, R>(trm, nt, tid, tile32, xv, acc); break;
                case 5: ring_group<5, R>(trm, nt, tid, tile32, xv, acc); break;
                case 6: ring_group<6, R>(trm, nt, tid, tile32, xv, acc); break;
                default: ring_group<7, R>(trm, nt, tid, tile32, xv, acc); break;
                }
                trm += nt;
                // FP32: fold the running partial sums into the compensated
                // row sum every kRingCompensateGroups groups (counted across
                // steps)
                if constexpr (sizeof(R) == 4) {
                    if (++since == kRingCompensateGroups) {
                        since = 0;
#pragma unroll
                        for (int j = 0; j < 8; ++j) acc[j].compensate();
                    }
                }
            }
        }
        __syncwarp();
        if (lane == 0u) {
            if constexpr (kProducerWarp) {
                mbar_arrive(&empty[stage]);
            } else {
                // The warp that releases the stage last refills it with step
                // st + K: its reads, and every other warp's, are ordered
                // before the counter update (fence), and the refill after it.
                __threadfence_block();
                if (atomicAdd(&released[stage], 1u) == kRingWarps - 1u) {
                    released[stage] = 0u;
                    __threadfence_block();
                    if (st + K < nsteps) {
                        ring_fill<R>(s, x, tile, info, st + K, smem_raw, full);
                        atomicMax(&issued_end, st + K + 1u);
                    }
                }
            }
        }
        if (++stage == K) {
            stage = 0;
            phase ^= 1u;
        }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j].compensate();
    C *yt = y + (tile << kTileBitsC128);
    if (accumulate) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            C &out = yt[tid + (j << kLogThreads)];
            const C v = acc[j].value();
            out.x += v.x;
            out.y += v.y;
        }
    } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) yt[tid + (j << kLogThreads)] = acc[j].value();
    }
}

// One thread per row; gathers straight from global memory.
template <typename R>
__global__ void k_rowwise(DevSchedule s, const typename Cx<R>::T *__restrict__ x,
                          typename Cx<R>::T *__restrict__ y, uint64_t dim, uint32_t accumulate) {
    using C = typename Cx<R>::T;
    for (uint64_t r = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; r < dim;
         r += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        Acc<R> acc;
        for (uint32_t g = 0; g < s.ngroups; ++g) {
            const uint64_t c = r ^ s.g_mask[g];
            const C v = x[c];
            R dre = R(0), dimv = R(0);
            for (uint32_t t = s.g_tbeg[g]; t < s.g_tbeg[g + 1]; ++t) {
                const C w = weight_of<R>(s, t);
                const bool neg = __popcll(s.t_z[t] & c) & 1;
                dre = dre + (neg ? -w.x : w.x);
                dimv = dimv + (neg ? -w.y : w.y);
            }
            acc.add_product(dre, dimv, v);
        }
        if (accumulate) {
            const C v = acc.value();
            y[r].x += v.x;
            y[r].y += v.y;
        } else {
            y[r] = acc.value();
        }
    }
}

// Eager transition count: nonzero D_m[c] over all groups m and columns c, with
// D summed in canonical term order exactly as hamiltonian.rs:125-133.
__global__ void k_transitions(DevSchedule s, uint32_t ngroups, uint64_t dim, unsigned long long *count) {
    unsigned long long local = 0;
    const uint64_t total = static_cast<uint64_t>(ngroups) * dim;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t g = static_cast<uint32_t>(i / dim);
        const uint64_t c = i % dim;
        double re = 0.0, im = 0.0;
        for (uint32_t t = s.g_tbeg[g]; t < s.g_tbeg[g + 1]; ++t) {
            const double2 w = s.t_w[t];
            const bool neg = __popcll(s.t_z[t] & c) & 1;
            re = re + (neg ? -w.x : w.x);
            im = im + (neg ? -w.y : w.y);
        }
        local += (re != 0.0 || im != 0.0);
    }
    for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(count, local);
}

// H_ii: the x_mask == 0 group's diagonal (zero when the operator has none).
__global__ void k_diagonal(DevSchedule s, uint32_t gzero, uint64_t dim, double2 *__restrict__ out) {
    for (uint64_t c = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; c < dim;
         c += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        double re = 0.0, im = 0.0;
        if (gzero != 0xffffffffu) {
            for (uint32_t t = s.g_tbeg[gzero]; t < s.g_tbeg[gzero + 1]; ++t) {
                const double2 w = s.t_w[t];
                const bool neg = __popcll(s.t_z[t] & c) & 1;
                re = re + (neg ? -w.x : w.x);
                im = im + (neg ? -w.y : w.y);
            }
        }
        out[c] = make_double2(re, im);
    }
}

}  // namespace

// --------------------------------- host side --------------------------------
namespace tcp {

int cuda_fail(cudaError_t e, const char *what) {
    return fail(TCP_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

cudaError_t dev_malloc(void **p, size_t bytes) {
    if (injected_alloc_failure()) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return cudaMalloc(p, bytes);
}


int check_plan(const tcp_mvp_plan *plan) {
    if (plan == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "plan is null");
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev != plan->device) {
        return fail(TCP_ERR_WRONG_DEVICE, "plan lives on device " + std::to_string(plan->device) +
                                              " but the current device is " + std::to_string(dev));
    }
    return TCP_OK;
}

int length_error(uint64_t expected, uint64_t actual) {
    return fail_fields(TCP_ERR_INVALID_STRUCTURE_LENGTH,
                       "expected structure length " + std::to_string(expected) + ", got " + std::to_string(actual),
                       expected, actual);
}

bool overlaps(const void *a, const void *b, size_t bytes) {
    auto pa = reinterpret_cast<uintptr_t>(a), pb = reinterpret_cast<uintptr_t>(b);
    return pa < pb + bytes && pb < pa + bytes;
}
}  // namespace tcp

using tcp::check_plan;
using tcp::cuda_fail;
using tcp::dev_malloc;
using tcp::length_error;
using tcp::overlaps;

namespace {

int g_num_sms = 0;
// Host apply at n = 28 (65,536 tiles): 4 input parts and 8 output chunks
// measured 280 ms; 8 parts and 16 chunks measured 312 ms (more passes over
// y and more pass start-up than the shorter exposed copies save).
constexpr uint64_t kHostEqualChunks = 8;                  // output-tile chunks of a large host apply,
constexpr uint64_t kHostChunks = kHostEqualChunks + 2;    // the last one split into 1/2, 1/4, 1/4

// First output tile of chunk c (c = kHostChunks: the end): equal chunks, the
// last of them split in a half and two quarters, so that the copy still to
// do once the last kernel has finished is a quarter of an equal chunk.
uint64_t chunk_start(uint64_t c, uint64_t tiles) {
    const uint64_t per = tiles / kHostEqualChunks, last = (kHostEqualChunks - 1) * per;
    if (c + 3 <= kHostChunks) return c * per;
    if (c + 2 == kHostChunks) return last + per / 2;
    if (c + 1 == kHostChunks) return last + 3 * per / 4;
    return tiles;
}
constexpr uint64_t kHostChunkTiles = 8192;  // tiles from which the host apply is chunked

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Step ranges of the source-chunk passes (see DevSchedule::pass_begin): the
// top kPassBits bits v of each step's outer pattern d, which is
// non-decreasing in step order because steps are sorted by d.
void set_passes(const std::vector<uint32_t> &step_info, uint32_t tile_bits, uint32_t nqubits, uint32_t *pass_begin,
                uint32_t *pass_shift) {
    const uint32_t nsteps = static_cast<uint32_t>(step_info.size() / 4);
    *pass_shift = kNoPasses;
    for (uint32_t v = 0; v <= kPassChunks; ++v) pass_begin[v] = v == 0 ? 0u : nsteps;
    if (tile_bits == 0 || nqubits < tile_bits + kPassBits) return;
    const uint32_t shift = nqubits - tile_bits - kPassBits;
    uint32_t prev = 0;
    for (uint32_t st = 0; st < nsteps; ++st) {
        const uint64_t d = static_cast<uint64_t>(step_info[4 * st]) | (static_cast<uint64_t>(step_info[4 * st + 1]) << 32);
        const uint32_t v = static_cast<uint32_t>(d >> shift);
        if (v >= kPassChunks || v < prev) return;  // not a sorted schedule: no passes
        for (uint32_t w = prev + 1; w <= v; ++w) pass_begin[w] = st;
        prev = v;
    }
    for (uint32_t w = prev + 1; w <= kPassChunks; ++w) pass_begin[w] = nsteps;
    *pass_shift = shift;
}

// Lay both schedules out in one device allocation.
int upload(tcp_mvp_plan *p) {
    tcp::Range range("plan upload");
    struct Piece {
        const void *src;
        size_t bytes;
        const void **dst;
    };
    std::vector<Piece> pieces;
    auto add = [&](const void *src, size_t bytes, const void **dst) { pieces.push_back({src, bytes, dst}); };
    {
        tcp::DeviceSchedule *ds = &p->sched;
        tcp::Schedule &h = ds->host;
        add(h.step_info.data(), h.step_info.size() * 4, reinterpret_cast<const void **>(&ds->dev.step_info));
        add(h.blocks_c128.data(), h.blocks_c128.size(), reinterpret_cast<const void **>(&ds->dev.blocks128));
        add(h.blocks_c64.data(), h.blocks_c64.size(), reinterpret_cast<const void **>(&ds->dev.blocks64));
        add(h.g_mask.data(), h.g_mask.size() * 8, reinterpret_cast<const void **>(&ds->dev.g_mask));
        add(h.g_tbeg.data(), h.g_tbeg.size() * 4, reinterpret_cast<const void **>(&ds->dev.g_tbeg));
        add(h.t_z.data(), h.t_z.size() * 8, reinterpret_cast<const void **>(&ds->dev.t_z));
        add(h.t_w.data(), h.t_w.size() * 8, reinterpret_cast<const void **>(&ds->dev.t_w));
        add(h.t_wf.data(), h.t_wf.size() * 4, reinterpret_cast<const void **>(&ds->dev.t_wf));
        ds->dev.nsteps = static_cast<uint32_t>(h.step_info.size() / 4);
        ds->dev.tile_bits = h.tile_bits;
        set_passes(h.step_info, h.tile_bits, p->nqubits, ds->dev.pass_begin, &ds->dev.pass_shift);
        tcp::RingSchedule &r = ds->ring;
        add(r.step_info.data(), r.step_info.size() * 4, reinterpret_cast<const void **>(&ds->dev.ring_info));
        add(r.blocks_c128.data(), r.blocks_c128.size(), reinterpret_cast<const void **>(&ds->dev.ring128));
        add(r.blocks_c64.data(), r.blocks_c64.size(), reinterpret_cast<const void **>(&ds->dev.ring64));
        ds->dev.ring_steps = static_cast<uint32_t>(r.step_info.size() / 4);
        set_passes(r.step_info, r.tile_bits, p->nqubits, ds->dev.ring_pass_begin, &ds->dev.ring_pass_shift);
        ds->dev.ngroups = static_cast<uint32_t>(h.g_mask.size());
    }
    size_t total = 256;  // error word first
    for (auto &pc : pieces) total = align_up(total, 256) + std::max<size_t>(pc.bytes, 16);
    void *block = nullptr;
    cudaError_t e = dev_malloc(&block, total);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(TCP_ERR_ALLOCATION, std::string("device allocation of the plan failed: ") + cudaGetErrorString(e));
    }
    std::vector<unsigned char> staging(total, 0);
    size_t off = 256;
    for (auto &pc : pieces) {
        off = align_up(off, 256);
        if (pc.bytes) std::memcpy(staging.data() + off, pc.src, pc.bytes);
        *pc.dst = static_cast<unsigned char *>(block) + off;
        off += std::max<size_t>(pc.bytes, 16);
    }
    e = cudaMemcpy(block, staging.data(), total, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(block);
        return cuda_fail(e, "plan upload");
    }
    p->dev_block = block;
    p->dev_bytes = total;
    p->d_err = static_cast<int *>(block);
    return TCP_OK;
}




template <int LOGE, typename R> constexpr size_t tiled_smem_bytes() {
    return 2 * (size_t(1) << (kLogThreads + LOGE)) * sizeof(typename Cx<R>::T) + 2 * size_t(tcp::kBlockBytesMax);
}

template <int LOGE, typename R> int set_smem_attr() {
    constexpr size_t bytes = tiled_smem_bytes<LOGE, R>();
    cudaError_t e = cudaFuncSetAttribute(k_tiled<LOGE, R, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(bytes));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_tiled<LOGE, R, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(bytes));
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "cudaFuncSetAttribute");
}

template <typename R> int set_ring_smem_attr() {
    constexpr size_t bytes = ring_smem_bytes<R>();
    cudaError_t e = cudaFuncSetAttribute(k_ring<R, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(bytes));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_ring<R, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_ring<R, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(bytes));
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "cudaFuncSetAttribute");
}

// The ring kernel serves every plan with a ring schedule whose input the TMA
// engine can address (16-byte aligned).
bool ring_ok(const tcp_mvp_plan *p, const void *x) {
    return p->sched.ring.tile_bits == kTileBitsC128 && p->nqubits >= kTileBitsC128 &&
           (reinterpret_cast<uintptr_t>(x) % 16) == 0;
}

// Number of output tiles of the tiled kernels (0 when the plan uses the row
// kernel for these buffers).
template <typename R>
uint64_t tiled_tiles(const tcp_mvp_plan *p, const void *x) {
    constexpr int LOGE = sizeof(R) == 8 ? kLogRowsC128 : kLogRowsC64;
    const uint32_t S = kLogThreads + LOGE;
    const bool aligned = (reinterpret_cast<uintptr_t>(x) % 16) == 0;
    if (ring_ok(p, x)) return p->dim >> kTileBitsC128;
    return (p->nqubits >= S && p->sched.host.tile_bits == S && aligned) ? (p->dim >> S) : 0;
}

// Whether the host path can split the state into kPassChunks parts for the
// kernel that serves these buffers.
bool has_passes(const tcp_mvp_plan *p, const void *x) {
    return (ring_ok(p, x) ? p->sched.dev.ring_pass_shift : p->sched.dev.pass_shift) != kNoPasses;
}

// Per-device, once: the shared-memory opt-in of the tiled kernels.
template <typename R> int ensure_smem_attrs(int device) {
    static std::mutex attr_mutex;
    static bool attr_done[64] = {};
    std::lock_guard<std::mutex> lock(attr_mutex);
    if (device < 0 || device >= 64) return fail(TCP_ERR_WRONG_DEVICE, "device ordinal out of range");
    if (!attr_done[device]) {
        constexpr int LOGE = sizeof(R) == 8 ? kLogRowsC128 : kLogRowsC64;
        int st = set_smem_attr<LOGE, R>();
        if (st == TCP_OK) st = set_ring_smem_attr<R>();
        if (st != TCP_OK) return st;
        attr_done[device] = true;
    }
    return TCP_OK;
}

// Apply on `stream`; the tiled kernels write output tiles [tile0, tile0 +
// ntiles) (ntiles = 0: all of them).  pass >= 0 runs one source-part pass of
// the host path, adding to y when `accumulate`.
template <typename R>
int launch_one(const tcp_mvp_plan *p, const void *x, void *y, cudaStream_t stream, uint64_t tile0 = 0,
               uint64_t ntiles = 0, int pass = -1, bool accumulate = false) {
    using C = typename Cx<R>::T;
    constexpr bool is64 = sizeof(R) == 8;
    constexpr int LOGE = is64 ? kLogRowsC128 : kLogRowsC64;
    const tcp::DeviceSchedule &ds = p->sched;
    const uint32_t S = kLogThreads + LOGE;
    const bool aligned = (reinterpret_cast<uintptr_t>(x) % 16) == 0;
    if (ring_ok(p, x)) {
        int st = ensure_smem_attrs<R>(p->device);
        if (st != TCP_OK) return st;
        const uint64_t tiles = ntiles ? ntiles : (p->dim >> kTileBitsC128) - tile0;
        const size_t smem = ring_smem_bytes<R>();
        if (pass >= 0) {
            k_ring<R, true><<<static_cast<unsigned>(tiles), RingShape<R>::kThreadsPerCta, smem, stream>>>(
                ds.dev, static_cast<const C *>(x), static_cast<C *>(y), p->d_err, tile0, static_cast<uint32_t>(pass),
                accumulate ? 1u : 0u, 0ull);
        } else {
            k_ring<R, false><<<static_cast<unsigned>(tiles), RingShape<R>::kThreadsPerCta, smem, stream>>>(
                ds.dev, static_cast<const C *>(x), static_cast<C *>(y), p->d_err, tile0, 0u, accumulate ? 1u : 0u, 0ull);
        }
    } else if (p->nqubits >= S && ds.host.tile_bits == S && aligned) {
        int st = ensure_smem_attrs<R>(p->device);
        if (st != TCP_OK) return st;
        const uint64_t tiles = ntiles ? ntiles : (p->dim >> S) - tile0;
        const size_t smem = tiled_smem_bytes<LOGE, R>();
        if (pass >= 0) {
            k_tiled<LOGE, R, true><<<static_cast<unsigned>(tiles), kThreads, smem, stream>>>(
                ds.dev, static_cast<const C *>(x), static_cast<C *>(y), p->d_err, tile0, static_cast<uint32_t>(pass),
                accumulate ? 1u : 0u);
        } else {
            k_tiled<LOGE, R, false><<<static_cast<unsigned>(tiles), kThreads, smem, stream>>>(
                ds.dev, static_cast<const C *>(x), static_cast<C *>(y), p->d_err, tile0, 0u, accumulate ? 1u : 0u);
        }
    } else {
        const int threads = 256;
        uint64_t blocks = (p->dim + threads - 1) / threads;
        blocks = std::min<uint64_t>(blocks, 1u << 20);
        k_rowwise<R><<<static_cast<unsigned>(blocks), threads, 0, stream>>>(
            ds.dev, static_cast<const C *>(x), static_cast<C *>(y), p->dim, accumulate ? 1u : 0u);
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "MVP kernel launch");
}

}  // namespace

namespace tcp {
// Whether `p` can run the ring kernel, with its shared-memory opt-in for the
// dtype set up (outside any stream capture).
int ring_prepare(const tcp_mvp_plan *p, bool c64) {
    if (p->sched.ring.tile_bits != kTileBitsC128 || p->nqubits < kTileBitsC128)
        return fail(TCP_ERR_INVALID_ARGUMENT, "the ring configuration needs a ring schedule (at least " +
                                                  std::to_string(kTileBitsC128) + " qubits) for every batch member");
    return c64 ? ensure_smem_attrs<float>(p->device) : ensure_smem_attrs<double>(p->device);
}

// One ring-kernel launch over every output tile of `p` and `nrhs`
// right-hand sides stored RHS-major (vector v at offset v * dim); a timed-out
// wait is recorded in `err`.  Fails with TCP_ERR_INVALID_ARGUMENT when the
// plan has no ring schedule or the buffers are not 16-byte aligned.
int launch_ring_rhs(const tcp_mvp_plan *p, const void *x, void *y, uint32_t nrhs, bool c64, int *err,
                    cudaStream_t stream) {
    if (!ring_ok(p, x) || (reinterpret_cast<uintptr_t>(y) % 16) != 0)
        return fail(TCP_ERR_INVALID_ARGUMENT, "the ring kernel needs a ring schedule and 16-byte aligned buffers");
    if (nrhs == 0 || nrhs > 65535u) return fail(TCP_ERR_INVALID_ARGUMENT, "RHS count out of range for one launch");
    const dim3 grid(static_cast<unsigned>(p->dim >> kTileBitsC128), nrhs);
    if (c64) {
        int st = ensure_smem_attrs<float>(p->device);
        if (st != TCP_OK) return st;
        k_ring<float, false, true><<<grid, RingShape<float>::kThreadsPerCta, ring_smem_bytes<float>(), stream>>>(
            p->sched.dev, static_cast<const float2 *>(x), static_cast<float2 *>(y), err, 0ull, 0u, 0u, p->dim);
    } else {
        int st = ensure_smem_attrs<double>(p->device);
        if (st != TCP_OK) return st;
        k_ring<double, false, true><<<grid, RingShape<double>::kThreadsPerCta, ring_smem_bytes<double>(), stream>>>(
            p->sched.dev, static_cast<const double2 *>(x), static_cast<double2 *>(y), err, 0ull, 0u, 0u, p->dim);
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "ring kernel launch");
}
}  // namespace tcp

namespace {

int read_device_status(const tcp_mvp_plan *p) {
    int h = 0;
    cudaError_t e = cudaMemcpy(&h, p->d_err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "reading device status");
    if (h != 0) {
        int zero = 0;
        cudaMemcpy(p->d_err, &zero, sizeof(int), cudaMemcpyHostToDevice);
        if (h & kErrTimeout) return fail(TCP_ERR_DEVICE_TIMEOUT, "a bounded device-side wait expired");
        if (h & kErrBounds) return fail(TCP_ERR_INVALID_ARGUMENT, "a plan block failed its bounds check (TCP_DEBUG_BOUNDS)");
    }
    return TCP_OK;
}

// Host threads for the copies between a caller's ordinary (pageable) buffer
// and the page-locked staging slots.  One copy at a time, split over the
// workers and the calling thread; the pool lives until the process exits.
class CopyPool {
  public:
    static CopyPool &get() {
        static CopyPool *pool = new CopyPool(std::max(1u, std::min(8u, std::thread::hardware_concurrency() / 2)));
        return *pool;
    }
    void copy(void *dst, const void *src, size_t bytes) {
        std::lock_guard<std::mutex> call(call_mutex_);
        {
            std::lock_guard<std::mutex> lock(mutex_);
            dst_ = static_cast<unsigned char *>(dst);
            src_ = static_cast<const unsigned char *>(src);
            bytes_ = bytes;
            pending_ = workers_;
            ++generation_;
        }
        start_.notify_all();
        piece(workers_);
        std::unique_lock<std::mutex> lock(mutex_);
        finished_.wait(lock, [&] { return pending_ == 0; });
    }

  private:
    explicit CopyPool(unsigned workers) : workers_(workers) {
        for (unsigned w = 0; w < workers; ++w) std::thread([this, w] { run(w); }).detach();
    }
    void piece(unsigned index) {
        const size_t parts = workers_ + 1;
        const size_t per = ((bytes_ / parts) + 4095) & ~size_t(4095);
        const size_t off = per * index;
        if (off < bytes_) std::memcpy(dst_ + off, src_ + off, std::min(per, bytes_ - off));
    }
    void run(unsigned index) {
        uint64_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lock(mutex_);
                start_.wait(lock, [&] { return generation_ != seen; });
                seen = generation_;
            }
            piece(index);
            std::lock_guard<std::mutex> lock(mutex_);
            if (--pending_ == 0) finished_.notify_all();
        }
    }
    unsigned workers_;
    std::mutex call_mutex_, mutex_;
    std::condition_variable start_, finished_;
    unsigned char *dst_ = nullptr;
    const unsigned char *src_ = nullptr;
    size_t bytes_ = 0;
    unsigned pending_ = 0;
    uint64_t generation_ = 0;
};

// Page-locked host memory (cudaHostAlloc or cudaHostRegister) moves by DMA
// without staging.
bool page_locked(const void *p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Copies of one host apply.  Page-locked buffers go straight to the DMA
// engine.  Ordinary buffers of at least two slots go through the staging
// ring: the host threads fill a free slot while the DMA engine drains the
// previous ones (input), or empty a slot whose DMA has landed while later
// slots are in flight (output), so both directions stay asynchronous to the
// kernels.
struct HostCopies {
    tcp::Staging *stage = nullptr;
    bool stage_in = false, stage_out = false;
    struct Out {
        unsigned char *dst;
        size_t len;
        int slot;
    };
    std::vector<Out> inflight;  // output slots in flight, oldest first

    unsigned char *slot_ptr(int slot) const { return stage->host + static_cast<size_t>(slot) * tcp::kStageSlotBytes; }
    int next_slot() {
        const int slot = static_cast<int>(stage->uses % tcp::kStageSlots);
        ++stage->uses;
        return slot;
    }
    int to_device(void *dst, const void *src, size_t len, cudaStream_t s) {
        tcp::Range range(stage_in ? "staged H2D" : "H2D");
        if (!stage_in) {
            cudaError_t e = cudaMemcpyAsync(dst, src, len, cudaMemcpyHostToDevice, s);
            return e == cudaSuccess ? TCP_OK : cuda_fail(e, "H2D copy");
        }
        for (size_t off = 0; off < len; off += tcp::kStageSlotBytes) {
            const size_t n = std::min(tcp::kStageSlotBytes, len - off);
            const int slot = next_slot();
            cudaError_t e = cudaEventSynchronize(stage->ev[slot]);  // its previous DMA has finished
            if (e != cudaSuccess) return cuda_fail(e, "staging slot");
            CopyPool::get().copy(slot_ptr(slot), static_cast<const unsigned char *>(src) + off, n);
            e = cudaMemcpyAsync(static_cast<unsigned char *>(dst) + off, slot_ptr(slot), n, cudaMemcpyHostToDevice, s);
            if (e == cudaSuccess) e = cudaEventRecord(stage->ev[slot], s);
            if (e != cudaSuccess) return cuda_fail(e, "staged H2D copy");
        }
        return TCP_OK;
    }
    int drain_one() {
        const Out o = inflight.front();
        inflight.erase(inflight.begin());
        cudaError_t e = cudaEventSynchronize(stage->ev[o.slot]);
        if (e != cudaSuccess) return cuda_fail(e, "staged D2H copy");
        CopyPool::get().copy(o.dst, slot_ptr(o.slot), o.len);
        return TCP_OK;
    }
    int to_host(void *dst, const void *src, size_t len, cudaStream_t s) {
        tcp::Range range(stage_out ? "staged D2H" : "D2H");
        if (!stage_out) {
            cudaError_t e = cudaMemcpyAsync(dst, src, len, cudaMemcpyDeviceToHost, s);
            return e == cudaSuccess ? TCP_OK : cuda_fail(e, "D2H copy");
        }
        for (size_t off = 0; off < len; off += tcp::kStageSlotBytes) {
            const size_t n = std::min(tcp::kStageSlotBytes, len - off);
            if (inflight.size() == static_cast<size_t>(tcp::kStageSlots)) {
                int st = drain_one();
                if (st) return st;
            }
            const int slot = next_slot();
            cudaError_t e = cudaEventSynchronize(stage->ev[slot]);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(slot_ptr(slot), static_cast<const unsigned char *>(src) + off, n,
                                    cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaEventRecord(stage->ev[slot], s);
            if (e != cudaSuccess) return cuda_fail(e, "staged D2H copy");
            inflight.push_back({static_cast<unsigned char *>(dst) + off, n, slot});
        }
        return TCP_OK;
    }
    int finish() {
        while (!inflight.empty()) {
            int st = drain_one();
            if (st) return st;
        }
        return TCP_OK;
    }
};

int ensure_staging(tcp::Workspace &ws) {
    if (ws.stage) return TCP_OK;
    auto *stage = new tcp::Staging();
    cudaError_t e = cudaHostAlloc(reinterpret_cast<void **>(&stage->host), tcp::kStageSlots * tcp::kStageSlotBytes,
                                  cudaHostAllocPortable);
    for (int k = 0; k < tcp::kStageSlots && e == cudaSuccess; ++k)
        e = cudaEventCreateWithFlags(&stage->ev[k], cudaEventDisableTiming);
    if (e == cudaSuccess) {
        // every slot starts free: its event has completed
        for (int k = 0; k < tcp::kStageSlots && e == cudaSuccess; ++k) e = cudaEventRecord(stage->ev[k], nullptr);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        for (auto &ev : stage->ev)
            if (ev) cudaEventDestroy(ev);
        if (stage->host) cudaFreeHost(stage->host);
        delete stage;
        return fail(TCP_ERR_ALLOCATION, std::string("page-locked staging ring: ") + cudaGetErrorString(e));
    }
    ws.stage = stage;
    return TCP_OK;
}

void release_staging(tcp::Staging *stage) {
    if (!stage) return;
    for (auto &ev : stage->ev)
        if (ev) cudaEventDestroy(ev);
    if (stage->host) cudaFreeHost(stage->host);
    delete stage;
}

template <typename R>
int apply_host(const tcp_mvp_plan *plan, const R *state, uint64_t state_len, R *result, uint64_t result_len) {
    tcp::Range range(sizeof(R) == 8 ? "tcp_mvp_apply_into_host" : "tcp_mvp_apply_into_host_c64");
    int st = check_plan(plan);
    if (st) return st;
    if (state_len != plan->dim) return length_error(plan->dim, state_len);
    if (result_len != plan->dim) return length_error(plan->dim, result_len);
    if (state == nullptr || result == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    const size_t bytes = plan->dim * 2 * sizeof(R);
    if (overlaps(state, result, bytes)) return fail(TCP_ERR_INVALID_ARGUMENT, "input and output must not overlap");
    tcp::Workspace ws;
    {
        std::lock_guard<std::mutex> lock(plan->ws_mutex);
        for (size_t i = 0; i < plan->ws_free.size(); ++i) {
            if (plan->ws_free[i].bytes >= bytes) {
                ws = plan->ws_free[i];
                plan->ws_free.erase(plan->ws_free.begin() + static_cast<long>(i));
                break;
            }
        }
    }
    if (ws.x == nullptr) {
        cudaError_t e1 = dev_malloc(&ws.x, bytes);
        cudaError_t e2 = e1 == cudaSuccess ? dev_malloc(&ws.y, bytes) : e1;
        if (e1 != cudaSuccess || e2 != cudaSuccess) {
            cudaGetLastError();
            if (ws.x) cudaFree(ws.x);
            return fail(TCP_ERR_ALLOCATION, "device allocation of the apply workspace failed");
        }
        ws.bytes = bytes;
        std::lock_guard<std::mutex> lock(plan->ws_mutex);
        plan->ws_all.push_back(ws);
    }
    HostCopies copies;
    int status = TCP_OK;
    const bool large = bytes >= 2 * tcp::kStageSlotBytes;
    copies.stage_in = large && !page_locked(state);
    copies.stage_out = large && !page_locked(result);
    if (copies.stage_in || copies.stage_out) {
        if (ensure_staging(ws) == TCP_OK) {
            std::lock_guard<std::mutex> lock(plan->ws_mutex);
            for (auto &w : plan->ws_all)
                if (w.x == ws.x) w.stage = ws.stage;
            copies.stage = ws.stage;
        } else {
            // no page-locked memory to stage through: plain (synchronous) copies
            copies.stage_in = copies.stage_out = false;
        }
    }
    cudaStream_t stream = nullptr;
    cudaError_t e = status ? cudaSuccess : cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) status = cuda_fail(e, "cudaStreamCreate");
    // Large tiled applies overlap both copies with the kernel.
    //  * Input: the state goes in as kParts parts on its own stream (an
    //    eighth, an eighth, a quarter, a half).  Pass k waits for part k only
    //    and runs the steps whose source tiles lie in it (the kernels'
    //    `pass`), adding to y after the first, so the copy of parts 1..
    //    overlaps the earlier passes.
    //  * Output: the first kFirstChunked passes run over every output tile;
    //    the last one, half of the source, runs per chunk of consecutive
    //    output tiles (chunk_start), and a third stream copies each finished
    //    chunk of y to the host while the next chunk computes, so the output
    //    copies overlap half of the kernel time.  The last chunks are
    //    smaller, so little copying is left once the last kernel has
    //    finished.
    // Every launch is queued right after the copy it waits for; ordinary
    // (pageable) buffers move through the staging ring (HostCopies).  Smaller
    // applies copy, launch once and copy back on one stream.
    const uint64_t tiles = tiled_tiles<R>(plan, ws.x);
    const uint64_t chunks = tiles >= kHostChunkTiles ? kHostChunks : 1;
    const bool passes = chunks > 1 && has_passes(plan, ws.x);
    // Source parts in eighths of the state's tiles: the input goes in as
    // eighth 0, eighth 1, the second quarter and the second half; pass k
    // reads exactly part k (kHostPass: base part | log2(parts) << 4), so the
    // first kernel waits for one eighth of the state only.  The last pass,
    // half of the source, runs per output chunk.
    static_assert(kPassChunks == 8, "host passes are laid out in eighths");
    constexpr int kParts = 4;
    constexpr int kHostPass[kParts] = {0, 1, 2 | (1 << 4), 4 | (2 << 4)};
    constexpr size_t kPartBegin[kParts + 1] = {0, 1, 2, 4, 8};  // eighths
    constexpr int kFirstChunked = kParts - 1;  // passes run per output chunk from here on
    cudaStream_t copy_stream = nullptr, in_stream = nullptr;
    cudaEvent_t done[kHostChunks] = {};
    cudaEvent_t landed[kParts] = {};
    if (!status && chunks > 1) {
        e = cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking);
        for (uint64_t c = 0; c < chunks && e == cudaSuccess; ++c) e = cudaEventCreateWithFlags(&done[c], cudaEventDisableTiming);
        if (passes && e == cudaSuccess) e = cudaStreamCreateWithFlags(&in_stream, cudaStreamNonBlocking);
        for (int k = 0; passes && k < kParts && e == cudaSuccess; ++k)
            e = cudaEventCreateWithFlags(&landed[k], cudaEventDisableTiming);
        if (e != cudaSuccess) status = cuda_fail(e, "creating the copy streams");
    }
    if (!status && chunks > 1) {
        if (passes) {
            const size_t eighth = bytes / kPassChunks;
            for (int k = 0; k < kParts && !status; ++k) {
                const size_t off = kPartBegin[k] * eighth, len = (kPartBegin[k + 1] - kPartBegin[k]) * eighth;
                status = copies.to_device(static_cast<unsigned char *>(ws.x) + off,
                                          reinterpret_cast<const unsigned char *>(state) + off, len, in_stream);
                if (!status) {
                    e = cudaEventRecord(landed[k], in_stream);
                    if (e == cudaSuccess) e = cudaStreamWaitEvent(stream, landed[k], 0);
                    if (e != cudaSuccess) status = cuda_fail(e, "waiting for an input part");
                }
                if (!status && k < kFirstChunked)
                    status = launch_one<R>(plan, ws.x, ws.y, stream, 0, 0, kHostPass[k], k > 0);
            }
        } else {
            status = copies.to_device(ws.x, state, bytes, stream);
        }
        auto start = [&](uint64_t c) { return chunks == 1 ? (c ? tiles : 0) : chunk_start(c, tiles); };
        for (uint64_t c = 0; c < chunks && !status; ++c) {
            const uint64_t t0 = start(c), nt = start(c + 1) - t0;
            if (passes) {
                for (int k = kFirstChunked; k < kParts && !status; ++k)
                    status = launch_one<R>(plan, ws.x, ws.y, stream, t0, nt, kHostPass[k], k > 0);
            } else {
                status = launch_one<R>(plan, ws.x, ws.y, stream, t0, nt);
            }
            if (!status) {
                e = cudaEventRecord(done[c], stream);
                if (e != cudaSuccess) status = cuda_fail(e, "chunk event");
            }
        }
        const size_t row_bytes = 2 * sizeof(R);
        const uint64_t rows_per_tile = plan->dim / tiles;
        for (uint64_t c = 0; c < chunks && !status; ++c) {
            const uint64_t t0 = start(c), nt = start(c + 1) - t0;
            const size_t off = t0 * rows_per_tile * row_bytes, len = nt * rows_per_tile * row_bytes;
            e = cudaStreamWaitEvent(copy_stream, done[c], 0);
            if (e != cudaSuccess) status = cuda_fail(e, "waiting for an output chunk");
            if (!status)
                status = copies.to_host(reinterpret_cast<unsigned char *>(result) + off,
                                        static_cast<const unsigned char *>(ws.y) + off, len, copy_stream);
        }
    } else if (!status) {
        status = copies.to_device(ws.x, state, bytes, stream);
        if (!status) status = launch_one<R>(plan, ws.x, ws.y, stream);
        if (!status) status = copies.to_host(result, ws.y, bytes, stream);
    }
    if (!status) status = copies.finish();
    for (cudaStream_t side : {in_stream, copy_stream}) {
        if (!side) continue;
        e = cudaStreamSynchronize(side);
        if (!status && e != cudaSuccess) status = cuda_fail(e, "copy stream synchronize");
        cudaStreamDestroy(side);
    }
    for (auto &ev : done)
        if (ev) cudaEventDestroy(ev);
    for (auto &ev : landed)
        if (ev) cudaEventDestroy(ev);
    if (stream) {
        e = cudaStreamSynchronize(stream);
        if (!status && e != cudaSuccess) status = cuda_fail(e, "stream synchronize");
        cudaStreamDestroy(stream);
    }
    if (ws.stage) {
        // staging events may still name copies that an error path left
        // queued; the streams are synchronised above, so every slot is free
        ws.stage->uses = 0;
    }
    if (!status) status = read_device_status(plan);
    {
        std::lock_guard<std::mutex> lock(plan->ws_mutex);
        plan->ws_free.push_back(ws);
    }
    return status;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" int tcp_mvp_plan_create(uint32_t nqubits, uint64_t term_count, uint32_t word_count,
                                   const uint64_t *x_words, const uint64_t *z_words, const double *coefficients,
                                   int storage, uint64_t max_bytes, tcp_mvp_plan **out_plan) {
    tcp::Range range("tcp_mvp_plan_create");
    if (out_plan == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "out_plan is null");
    *out_plan = nullptr;
    if (storage != TCP_STORAGE_LAZY && storage != TCP_STORAGE_EAGER) {
        return fail(TCP_ERR_INVALID_SECTOR, "invalid sector: storage must be either 'eager' or 'lazy'");
    }
    if (term_count > 0 && (x_words == nullptr || z_words == nullptr || coefficients == nullptr)) {
        return fail(TCP_ERR_INVALID_ARGUMENT, "null term arrays");
    }
    if (term_count > 0xffffffffull) return fail(TCP_ERR_OVERFLOW, "integer overflow while counting plan terms");
    std::unique_ptr<tcp_mvp_plan> p(new tcp_mvp_plan());
    int st = tcp::compile_terms(nqubits, term_count, word_count, x_words, z_words, coefficients, p->terms);
    if (st) return st;
    p->nqubits = nqubits;
    p->word_count = word_count;
    p->dim = 1ull << nqubits;
    p->storage = storage;
    p->group_count = tcp::distinct_x_masks(p->terms);
    if (storage == TCP_STORAGE_EAGER) {
        // from_operator_reusable budget (hamiltonian.rs:84-119): G*dim*16
        // diagonal bytes (+ 2 * T * 32 term bytes + G * 32 group headers).
        unsigned __int128 diag = static_cast<unsigned __int128>(p->group_count) * p->dim * 16u;
        unsigned __int128 term_bytes = static_cast<unsigned __int128>(term_count) * 32u;
        if (diag >> 64) return fail(TCP_ERR_OVERFLOW, "integer overflow while estimating reusable MVP plan memory");
        if (term_bytes > max_bytes) {
            return tcp::fail_fields(TCP_ERR_MEMORY_LIMIT,
                                    "requested " + std::to_string(static_cast<uint64_t>(term_bytes)) +
                                        " bytes exceeds memory limit " + std::to_string(max_bytes),
                                    tcp::clamp_u64(term_bytes), max_bytes);
        }
        unsigned __int128 construction = diag + 2 * term_bytes + static_cast<unsigned __int128>(p->group_count) * 32u;
        if (construction > max_bytes) {
            std::string req = construction >> 64 ? std::string("more than 2^64")
                                                  : std::to_string(static_cast<uint64_t>(construction));
            return tcp::fail_fields(TCP_ERR_MEMORY_LIMIT,
                                    "requested " + req + " bytes exceeds memory limit " + std::to_string(max_bytes),
                                    tcp::clamp_u64(construction), max_bytes);
        }
    }
    cudaError_t e = cudaGetDevice(&p->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (g_num_sms == 0) cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, p->device);
    {
        tcp::Range range("tile schedules");
        p->sched.host = tcp::build_schedule(p->terms, nqubits, kTileBitsC128, kLogThreads);
        p->sched.ring = tcp::build_ring_schedule(p->terms, nqubits, kTileBitsC128, kLogThreads);
    }
    st = upload(p.get());
    if (st) return st;
    if (storage == TCP_STORAGE_EAGER) {
        uint64_t count = 0;
        st = tcp_mvp_transition_count(p.get(), &count);
        if (st) {
            cudaFree(p->dev_block);
            return st;
        }
        p->transitions = static_cast<int64_t>(count);
    }
    *out_plan = p.release();
    return TCP_OK;
}

extern "C" int tcp_mvp_plan_destroy(tcp_mvp_plan *plan) {
    if (plan == nullptr) return TCP_OK;
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != plan->device) cudaSetDevice(plan->device);
    for (auto &w : plan->ws_all) {
        cudaFree(w.x);
        cudaFree(w.y);
        release_staging(w.stage);
    }
    if (plan->dev_block) cudaFree(plan->dev_block);
    if (prev >= 0 && prev != plan->device) cudaSetDevice(prev);
    delete plan;
    return TCP_OK;
}

extern "C" int tcp_mvp_plan_info(const tcp_mvp_plan *plan, tcp_mvp_plan_info_t *info) {
    if (plan == nullptr || info == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "null argument");
    info->nqubits = plan->nqubits;
    info->word_count = plan->word_count;
    info->dimension = plan->dim;
    info->term_count = plan->terms.size();
    info->group_count = plan->group_count;
    info->storage = plan->storage;
    info->device = plan->device;
    info->transition_count = plan->transitions;
    info->device_bytes = plan->dev_bytes;
    info->tile_bits = plan->sched.host.tile_bits;
    info->log_threads = plan->sched.host.log_threads;
    info->steps = plan->sched.host.step_info.size() / 4;
    info->outer_patterns = plan->sched.host.distinct_outer;
    info->ring_steps = plan->sched.ring.step_info.size() / 4;
    info->cosets = plan->sched.ring.cosets;
    return TCP_OK;
}

extern "C" int tcp_mvp_apply_into_host(const tcp_mvp_plan *plan, const double *state, uint64_t state_len,
                                       double *result, uint64_t result_len, uint64_t max_bytes) {
    (void)max_bytes;  // advisory, ignored by the reference apply (hamiltonian.rs:223)
    return apply_host<double>(plan, state, state_len, result, result_len);
}

extern "C" int tcp_mvp_apply_into_host_c64(const tcp_mvp_plan *plan, const float *state, uint64_t state_len,
                                           float *result, uint64_t result_len) {
    return apply_host<float>(plan, state, state_len, result, result_len);
}

namespace {
int apply_device(const tcp_mvp_plan *plan, const void *d_state, void *d_result, uint64_t len, uint32_t nrhs,
                 int dtype, void *stream, bool accumulate) {
    tcp::Range range(accumulate ? "tcp_mvp_apply_add_device" : "tcp_mvp_apply_into_device");
    int st = check_plan(plan);
    if (st) return st;
    if (len != plan->dim) return length_error(plan->dim, len);
    if (dtype != TCP_DTYPE_C128 && dtype != TCP_DTYPE_C64) return fail(TCP_ERR_INVALID_ARGUMENT, "unknown dtype");
    if (nrhs == 0) return TCP_OK;
    if (d_state == nullptr || d_result == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    const size_t elem = dtype == TCP_DTYPE_C128 ? 16 : 8;
    const size_t bytes = static_cast<size_t>(len) * elem * nrhs;
    if (overlaps(d_state, d_result, bytes)) return fail(TCP_ERR_INVALID_ARGUMENT, "input and output must not overlap");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    for (uint32_t v = 0; v < nrhs; ++v) {
        const void *x = static_cast<const unsigned char *>(d_state) + static_cast<size_t>(v) * len * elem;
        void *y = static_cast<unsigned char *>(d_result) + static_cast<size_t>(v) * len * elem;
        st = dtype == TCP_DTYPE_C128 ? launch_one<double>(plan, x, y, s, 0, 0, -1, accumulate)
                                     : launch_one<float>(plan, x, y, s, 0, 0, -1, accumulate);
        if (st) return st;
    }
    return TCP_OK;
}
}  // namespace

extern "C" int tcp_mvp_apply_into_device(const tcp_mvp_plan *plan, const void *d_state, void *d_result,
                                         uint64_t len, uint32_t nrhs, int dtype, void *stream) {
    return apply_device(plan, d_state, d_result, len, nrhs, dtype, stream, false);
}

extern "C" int tcp_mvp_apply_add_device(const tcp_mvp_plan *plan, const void *d_state, void *d_result, uint64_t len,
                                        uint32_t nrhs, int dtype, void *stream) {
    return apply_device(plan, d_state, d_result, len, nrhs, dtype, stream, true);
}

extern "C" int tcp_mvp_plan_device_status(const tcp_mvp_plan *plan) {
    int st = check_plan(plan);
    if (st) return st;
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceSynchronize");
    return read_device_status(plan);
}

extern "C" int tcp_mvp_transition_count(const tcp_mvp_plan *plan, uint64_t *out_count) {
    int st = check_plan(plan);
    if (st) return st;
    if (out_count == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "out_count is null");
    unsigned long long *d_count = nullptr;
    cudaError_t e = dev_malloc(reinterpret_cast<void **>(&d_count), sizeof(unsigned long long));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(TCP_ERR_ALLOCATION, "device allocation of the transition counter failed");
    }
    cudaMemset(d_count, 0, sizeof(unsigned long long));
    const uint32_t ngroups = static_cast<uint32_t>(plan->sched.host.g_mask.size());
    const uint64_t total = static_cast<uint64_t>(ngroups) * plan->dim;
    if (total > 0) {
        const int threads = 256;
        uint64_t blocks = std::min<uint64_t>((total + threads - 1) / threads, 148ull * 64);
        k_transitions<<<static_cast<unsigned>(blocks), threads>>>(plan->sched.dev, ngroups, plan->dim, d_count);
    }
    unsigned long long h = 0;
    e = cudaMemcpy(&h, d_count, sizeof h, cudaMemcpyDeviceToHost);
    cudaFree(d_count);
    if (e != cudaSuccess) return cuda_fail(e, "transition count");
    *out_count = h;
    return TCP_OK;
}

extern "C" int tcp_mvp_diagonal_device(const tcp_mvp_plan *plan, void *d_diag, uint64_t len, void *stream) {
    int st = check_plan(plan);
    if (st) return st;
    if (len != plan->dim) return length_error(plan->dim, len);
    if (d_diag == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    const tcp::Schedule &h = plan->sched.host;
    uint32_t gzero = 0xffffffffu;
    for (size_t g = 0; g < h.g_mask.size(); ++g) {
        if (h.g_mask[g] == 0) {
            gzero = static_cast<uint32_t>(g);
            break;
        }
    }
    const int threads = 256;
    uint64_t blocks = std::min<uint64_t>((plan->dim + threads - 1) / threads, 1u << 20);
    k_diagonal<<<static_cast<unsigned>(blocks), threads, 0, static_cast<cudaStream_t>(stream)>>>(
        plan->sched.dev, gzero, plan->dim, static_cast<double2 *>(d_diag));
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "diagonal kernel launch");
}

// ---------------------------------------------------------------------------
// Self-test of the bounded device waits: one CTA arms an mbarrier for bytes
// that no copy will ever deliver and waits on it with a short limit; the wait
// gives up, the kernel records a timeout in the plan's status word and exits.
// No copy is in flight, so nothing touches the abandoned barrier afterwards.
// ---------------------------------------------------------------------------
namespace {
__global__ void k_wait_selftest(unsigned long long limit_ns, int *err) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) mbar_arrive_expect_tx(&bar, 16);  // 16 bytes that never arrive
    __syncthreads();
    const bool ok = mbar_wait_bounded(&bar, 0, limit_ns);
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) atomicOr(err, kErrTimeout);
    }
}
}  // namespace

extern "C" int tcp_selftest_bounded_wait(const tcp_mvp_plan *plan, uint64_t limit_ns) {
    int st = check_plan(plan);
    if (st) return st;
    if (limit_ns > 100000000ull) return fail(TCP_ERR_INVALID_ARGUMENT, "self-test wait limit above 100 ms");
    k_wait_selftest<<<1, 32>>>(limit_ns, plan->d_err);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "self-test kernel launch");
    return tcp_mvp_plan_device_status(plan);
}

// ---------------------------------------------------------------------------
// Allocation-free host apply (tcp_mvp_apply_into_host_noalloc).
//
// For callers that may not allocate device memory while applying.  The state
// and the result are staged through one static device array that belongs to
// the library image: a 256-byte status block (cleared at the start of every
// call) followed by two vectors of 2^TCP_NOALLOC_MAX_QUBITS complex128.  Every
// GPU that loads the library holds it (32 MiB + 256 B) until the process exits.
// All calls share it, so calls that overlap on the GPU race; it keeps the last
// call's contents.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kNoallocStatusBytes = 256;
constexpr size_t kNoallocMaxDim = size_t(1) << TCP_NOALLOC_MAX_QUBITS;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocStatusBytes + 2 * kNoallocMaxDim * sizeof(double2)];

std::mutex g_noalloc_mutex;
unsigned char *g_noalloc_ptr[64] = {};
bool g_noalloc_attr[64] = {};

// Set-up, once per device, with that device current: the host-side name of a
// __device__ array is only a stand-in, so its device address is looked up.
int noalloc_scratch(int device, unsigned char **out) {
    if (device < 0 || device >= 64) return fail(TCP_ERR_WRONG_DEVICE, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (g_noalloc_ptr[device] == nullptr) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress of the static scratch");
        g_noalloc_ptr[device] = static_cast<unsigned char *>(p);
    }
    if (!g_noalloc_attr[device]) {
        int st = ensure_smem_attrs<double>(device);
        if (st) return st;
        g_noalloc_attr[device] = true;
    }
    *out = g_noalloc_ptr[device];
    return TCP_OK;
}

}  // namespace

extern "C" int tcp_mvp_apply_into_host_noalloc(const tcp_mvp_plan *plan, const double *state, uint64_t state_len,
                                               double *result, uint64_t result_len, void *stream) {
    int st = check_plan(plan);
    if (st) return st;
    if (state_len != plan->dim) return length_error(plan->dim, state_len);
    if (result_len != plan->dim) return length_error(plan->dim, result_len);
    if (state == nullptr || result == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    if (plan->nqubits > TCP_NOALLOC_MAX_QUBITS) {
        return tcp::fail_fields(TCP_ERR_MEMORY_LIMIT,
                                "tcp_mvp_apply_into_host_noalloc handles at most " +
                                    std::to_string(TCP_NOALLOC_MAX_QUBITS) + " qubits (static scratch of 2^" +
                                    std::to_string(TCP_NOALLOC_MAX_QUBITS) + " amplitudes per vector); this plan has " +
                                    std::to_string(plan->nqubits),
                                plan->dim * 2 * sizeof(double2), 2 * kNoallocMaxDim * sizeof(double2));
    }
    const size_t bytes = plan->dim * sizeof(double2);
    if (overlaps(state, result, bytes)) return fail(TCP_ERR_INVALID_ARGUMENT, "input and output must not overlap");
    unsigned char *base = nullptr;
    st = noalloc_scratch(plan->device, &base);
    if (st) return st;
    int *d_status = reinterpret_cast<int *>(base);
    double2 *dx = reinterpret_cast<double2 *>(base + kNoallocStatusBytes);
    double2 *dy = dx + kNoallocMaxDim;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    cudaError_t e = cudaMemsetAsync(d_status, 0, kNoallocStatusBytes, s);  // must start at zero
    if (e != cudaSuccess) return cuda_fail(e, "clearing the static scratch status");
    e = cudaMemcpyAsync(dx, state, bytes, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_fail(e, "H2D copy into the static scratch");
    const tcp::DeviceSchedule &ds = plan->sched;
    const uint32_t S = kTileBitsC128;
    if (ring_ok(plan, dx)) {
        k_ring<double, false><<<static_cast<unsigned>(plan->dim >> S), RingShape<double>::kThreadsPerCta, ring_smem_bytes<double>(), s>>>(
            ds.dev, dx, dy, d_status, 0, 0u, 0u, 0ull);
    } else if (plan->nqubits >= S && ds.host.tile_bits == S) {
        const size_t smem = tiled_smem_bytes<kLogRowsC128, double>();
        k_tiled<kLogRowsC128, double, false><<<static_cast<unsigned>(plan->dim >> S), kThreads, smem, s>>>(
            ds.dev, dx, dy, d_status, 0, 0u, 0u);
    } else {
        const int threads = 256;
        const uint64_t blocks = (plan->dim + threads - 1) / threads;
        k_rowwise<double><<<static_cast<unsigned>(blocks), threads, 0, s>>>(ds.dev, dx, dy, plan->dim, 0u);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "MVP kernel launch");
    e = cudaMemcpyAsync(result, dy, bytes, cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return cuda_fail(e, "D2H copy from the static scratch");
    int h_status = 0;
    e = cudaMemcpyAsync(&h_status, d_status, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return cuda_fail(e, "reading the static scratch status");
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "stream synchronize");
    if (h_status & kErrTimeout) {
        // the kernel gave up before writing every output tile: no stale rows
        // of an earlier call reach the caller
        std::memset(result, 0, bytes);
        return fail(TCP_ERR_DEVICE_TIMEOUT, "a bounded device-side wait expired");
    }
    return TCP_OK;
}
