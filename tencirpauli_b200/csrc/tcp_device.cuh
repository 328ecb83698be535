// Device-side building blocks shared by the MVP kernels of libtcpmvp.so:
// launch constants, the device view of a plan's schedule, PTX wrappers for
// the TMA bulk-copy engine and mbarriers (with bounded waits), complex types,
// sign helpers and the row accumulators.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "tcp_internal.h"

namespace tcpdev {

constexpr int kLogThreads = 9;               // 512 threads per CTA
constexpr int kThreads = 1 << kLogThreads;
constexpr int kLogRowsC128 = 3;              // 8 rows per thread  -> 4096-row tile
constexpr int kLogRowsC64 = 3;               // 8 rows per thread  -> 4096-row tile
constexpr uint32_t kTileBitsC128 = kLogThreads + kLogRowsC128;
constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // 2 s bound on any device wait
constexpr uint32_t kCompensateGroups = 4;   // FP32: groups per Kahan fold

constexpr uint32_t kPassBits = 3;            // host path: the state goes in by eighths of its tiles
constexpr uint32_t kPassChunks = 1u << kPassBits;
constexpr uint32_t kNoPasses = 0xffffffffu;

// Error bits written by kernels into the plan's device status word.
constexpr int kErrTimeout = 1;
constexpr int kErrBounds = 2;  // TCP_DEBUG_BOUNDS builds: a block failed its bounds check

struct DevSchedule {
    // step view (tiled kernels); see tcp::Schedule
    const uint4 *step_info;          // d lo, d hi, block offset / 16, ngroups | (bytes / 16) << 16
    const unsigned char *blocks128;  // step blocks with FP64 weights
    const unsigned char *blocks64;   // step blocks with FP32 weights
    uint32_t nsteps;
    uint32_t tile_bits;
    // Source-part passes of the host path: steps [pass_begin[v],
    // pass_begin[v + 1]) have outer patterns d whose top kPassBits bits equal
    // v (steps are sorted by d), so an output tile t reads source tiles t ^ d
    // in part v ^ (t >> pass_shift) of the kPassChunks equal parts of the
    // state (pass_range).  pass_shift = kNoPasses when the state has fewer
    // than kPassChunks tiles.
    uint32_t pass_begin[kPassChunks + 1];
    uint32_t pass_shift;
    // ring view (k_ring; see tcp::RingSchedule): ring_steps = 0 when the
    // plan has no ring schedule.  Pass ranges as above, over the ring steps.
    const uint4 *ring_info;          // d lo, d hi, block offset / 16, block bytes / 16
    const unsigned char *ring128;    // blocks with FP64 weights
    const unsigned char *ring64;     // blocks with FP32 weights
    uint32_t ring_steps;
    uint32_t ring_pass_begin[kPassChunks + 1];
    uint32_t ring_pass_shift;
    // group view (row kernel, transition count, diagonal): unfolded weights
    const uint64_t *g_mask;
    const uint32_t *g_tbeg;
    const uint64_t *t_z;
    const double2 *t_w;
    const float2 *t_wf;
    uint32_t ngroups;
};

// Step range [b0, b1) of host-path pass `pass` = p | log2(span) << 4 for
// output tile `tile`: the pass reads the source parts of the aligned block
// of `span` parts that contains part p, i.e. the steps whose top pattern bits
// lie in the aligned block containing p ^ (tile >> shift), one contiguous
// range since steps are sorted by d.  Constant indices only: a computed index
// into the kernel's parameter struct would copy it to the stack.
__device__ __forceinline__ void pass_range(const uint32_t (&begin)[kPassChunks + 1], uint32_t shift, uint64_t tile,
                                           uint32_t pass, uint32_t &b0, uint32_t &b1) {
    const uint32_t span = 1u << (pass >> 4);
    const uint32_t v = (pass ^ static_cast<uint32_t>(tile >> shift)) & (kPassChunks - 1u) & ~(span - 1u);
    b0 = begin[0];
    b1 = begin[kPassChunks];
#pragma unroll
    for (uint32_t w = 1; w < kPassChunks; ++w) {
        if (v == w) b0 = begin[w];
    }
#pragma unroll
    for (uint32_t w = 1; w < kPassChunks; ++w) {
        if (v + span == w) b1 = begin[w];
    }
}

// ------------------------------- PTX helpers -------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// 1-D bulk copy global -> shared through the TMA engine; completes tx bytes
// on the mbarrier.  Both addresses 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// Plain arrive (count 1) on an mbarrier.
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// Non-blocking test of an mbarrier phase.
__device__ __forceinline__ uint32_t mbar_test_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok;
}
__device__ __forceinline__ uint32_t mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok;
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait on an mbarrier phase: returns false after `limit_ns`.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity,
                                                  unsigned long long limit_ns = kWaitLimitNs) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long start = global_ns();
    for (uint32_t spin = 1;; ++spin) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((spin & 255u) == 0u && global_ns() - start > limit_ns) return false;
    }
}

// Bounded wait that also gives up as soon as another thread of the CTA has
// raised `abort_flag` (a shared-memory word); returns false on either.
__device__ __forceinline__ bool mbar_wait_or_abort(uint64_t *bar, uint32_t parity, const volatile int *abort_flag,
                                                   unsigned long long limit_ns = kWaitLimitNs) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long start = global_ns();
    for (uint32_t spin = 1;; ++spin) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((spin & 63u) == 0u && (*abort_flag || global_ns() - start > limit_ns)) return false;
    }
}

// ------------------------------ complex types ------------------------------
template <typename R> struct Cx;
template <> struct Cx<double> { using T = double2; };
template <> struct Cx<float> { using T = float2; };

template <typename R> __device__ __forceinline__ typename Cx<R>::T weight_of(const DevSchedule &s, uint32_t t);
template <> __device__ __forceinline__ double2 weight_of<double>(const DevSchedule &s, uint32_t t) {
    return __ldg(&s.t_w[t]);
}
template <> __device__ __forceinline__ float2 weight_of<float>(const DevSchedule &s, uint32_t t) {
    return __ldg(&s.t_wf[t]);
}
// Weight of a term record in a shared-memory step block (offset 16 bytes).
template <typename R> __device__ __forceinline__ typename Cx<R>::T record_weight(const unsigned char *rec);
template <> __device__ __forceinline__ double2 record_weight<double>(const unsigned char *rec) {
    return *reinterpret_cast<const double2 *>(rec + 16);
}
template <> __device__ __forceinline__ float2 record_weight<float>(const unsigned char *rec) {
    return *reinterpret_cast<const float2 *>(rec + 16);
}

// Flip the sign of w when bit `bit` of `pattern` is set (an integer op on the
// sign bit; `bit` is a compile-time constant after unrolling).
__device__ __forceinline__ double flip_if(double w, uint32_t pattern, int bit) {
    const int hi = __double2hiint(w) ^ static_cast<int>((pattern << (31 - bit)) & 0x80000000u);
    return __hiloint2double(hi, __double2loint(w));
}
__device__ __forceinline__ float flip_if(float w, uint32_t pattern, int bit) {
    return __int_as_float(__float_as_int(w) ^ static_cast<int>((pattern << (31 - bit)) & 0x80000000u));
}
// Flip the sign of w when `odd` (0 or 1) is set.
__device__ __forceinline__ double flip_by(double w, uint32_t odd) {
    return __hiloint2double(__double2hiint(w) ^ static_cast<int>(odd << 31), __double2loint(w));
}
__device__ __forceinline__ float flip_by(float w, uint32_t odd) {
    return __int_as_float(__float_as_int(w) ^ static_cast<int>(odd << 31));
}

// Accumulator of one output row.  FP64: terms are added straight into the
// row sum.  FP32: terms are summed into a running partial sum, which is folded
// into the row sum with Kahan compensation (one compensation term per
// component) after every kCompensateGroups x-mask groups and at the end of
// every step, so the long sum across x-mask groups is compensated.
template <typename R> struct Acc;
template <> struct Acc<double> {
    double re = 0.0, im = 0.0;
    __device__ __forceinline__ void compensate() {}
    __device__ __forceinline__ void add_real(double w, double2 v) {
        re = fma(w, v.x, re);
        im = fma(w, v.y, im);
    }
    __device__ __forceinline__ void add_imag(double w, double2 v) {
        re = fma(-w, v.y, re);
        im = fma(w, v.x, im);
    }
    __device__ __forceinline__ void add_complex(double wr, double wi, double2 v) {
        re = fma(wr, v.x, re);
        re = fma(-wi, v.y, re);
        im = fma(wr, v.y, im);
        im = fma(wi, v.x, im);
    }
    // group view: D = sum of signed weights, then y += D x
    __device__ __forceinline__ void add_product(double dre, double dim, double2 v) { add_complex(dre, dim, v); }
    __device__ __forceinline__ double2 value() const { return make_double2(re, im); }
};
template <> struct Acc<float> {
    float re = 0.f, im = 0.f, cre = 0.f, cim = 0.f;  // Kahan sums
    float pre = 0.f, pim = 0.f;                      // current group's contribution
    __device__ __forceinline__ static void kahan(float &sum, float &comp, float term) {
        const float yv = __fsub_rn(term, comp);
        const float tv = __fadd_rn(sum, yv);
        comp = __fsub_rn(__fsub_rn(tv, sum), yv);
        sum = tv;
    }
    // Fold the running partial sum into the Kahan-compensated row sum.
    __device__ __forceinline__ void compensate() {
        kahan(re, cre, pre);
        kahan(im, cim, pim);
        pre = pim = 0.f;
    }
    __device__ __forceinline__ void add_real(float w, float2 v) {
        pre = __fmaf_rn(w, v.x, pre);
        pim = __fmaf_rn(w, v.y, pim);
    }
    __device__ __forceinline__ void add_imag(float w, float2 v) {
        pre = __fmaf_rn(-w, v.y, pre);
        pim = __fmaf_rn(w, v.x, pim);
    }
    __device__ __forceinline__ void add_complex(float wr, float wi, float2 v) {
        pre = __fmaf_rn(wr, v.x, pre);
        pre = __fmaf_rn(-wi, v.y, pre);
        pim = __fmaf_rn(wr, v.y, pim);
        pim = __fmaf_rn(wi, v.x, pim);
    }
    __device__ __forceinline__ void add_product(float dre, float dim, float2 v) {
        add_complex(dre, dim, v);
        compensate();
    }
    __device__ __forceinline__ float2 value() const { return make_float2(re, im); }
};

// Row accumulator of the ring kernel.  FP64: the plain Acc.  FP32: (re, im)
// pairs packed in 64-bit registers and updated with the paired FP32
// instructions of sm_100 (fma/add/sub .rn.f32x2: each lane rounds exactly as
// the scalar instruction), so one instruction serves both components.  Two
// running partial sums -- p for real weights (w x) and q for imaginary
// weights (w x, whose contribution is i q) -- take the same instruction form;
// compensate() folds p + i q into the Kahan-compensated row sum.
template <typename R> struct RingAcc;
template <> struct RingAcc<double> : Acc<double> {};

__device__ __forceinline__ uint64_t pack2(float lo, float hi) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ float2 unpack2(uint64_t v) {
    float lo, hi;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
    return make_float2(lo, hi);
}
__device__ __forceinline__ uint64_t fma2(uint64_t a, uint64_t b, uint64_t c) {
    uint64_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ uint64_t add2(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t sub2(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

template <> struct RingAcc<float> {
    uint64_t s = 0, c = 0;  // Kahan sum and compensation, (re, im)
    uint64_t p = 0, q = 0;  // running partial sums of real / imaginary weights
    __device__ __forceinline__ void add_real(float w, float2 v) { p = fma2(pack2(w, w), pack2(v.x, v.y), p); }
    __device__ __forceinline__ void add_imag(float w, float2 v) { q = fma2(pack2(w, w), pack2(v.x, v.y), q); }
    __device__ __forceinline__ void compensate() {
        const float2 qq = unpack2(q);
        const uint64_t term = add2(p, pack2(-qq.y, qq.x));  // p + i q
        const uint64_t yv = sub2(term, c);
        const uint64_t tv = add2(s, yv);
        c = sub2(sub2(tv, s), yv);
        s = tv;
        p = q = 0;
    }
    __device__ __forceinline__ float2 value() const { return unpack2(s); }
};

}  // namespace tcpdev
