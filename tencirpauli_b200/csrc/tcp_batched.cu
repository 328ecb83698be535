// libtcpmvp.so -- batched MVP: many Hamiltonians of uneven qubit and term
// counts, each applied to a block of right-hand sides, replayed from one CUDA
// graph, with the configuration picked by an autotuner (on-disk cache): one
// persistent launch of k_batched (tile shape and RHS block), or the ring
// configuration described below.
//
// k_batched<LOGT, RB, R>: persistent CTAs of 2^LOGT threads take work items
// (Hamiltonian h, output tile of 2^LOGT rows, block of RB right-hand sides)
// from an atomic counter; items are ordered largest Hamiltonian first.  Each
// thread owns one row of the tile and RB accumulators.  For every step (outer
// pattern d) of h the TMA engine copies the RB source tiles (tile ^ d) and the
// step's block of group/term records into shared memory (double-buffered,
// bounded mbarrier waits); the next item's first step is prefetched during the
// current item's last step.  Per term, the sign and weight are evaluated once
// and applied to all RB right-hand sides.
//
// The ring configuration (tile_rows_log2 = 12, rhs_block = 1) instead runs
// the single-operator ring kernel once per member, its grid covering every
// output tile and every right-hand side (blockIdx.y), members largest first,
// all captured in the same CUDA graph.  It needs a ring schedule for every
// member (n >= 12).
//
// State layout: the RHS block of Hamiltonian h is RHS-major, vector v at
// offset v * 2^n (complex128 or complex64), as for tcp_mvp_apply_into_device.
#include <cuda_runtime.h>

#include <algorithm>
#include <utility>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "tcp_device.cuh"
#include "tcp_plan_impl.h"

using namespace tcpdev;
using tcp::cuda_fail;
using tcp::dev_malloc;
using tcp::fail;

namespace {

// Device descriptor of one batch member (one Hamiltonian and its RHS block).
struct BatchHam {
    const uint4 *step_info;
    const unsigned char *blocks;  // step blocks with weights of the batch dtype
    const void *x;                // RHS-major [nrhs][dim]
    void *y;
    uint64_t dim;
    uint32_t nsteps;
    uint32_t nqubits;
};

struct BatchItem {
    uint32_t ham;
    uint32_t rhs0;
    uint64_t tile;
};

template <typename C, uint32_t LOGT, int RB>
__device__ __forceinline__ void issue_batch_step(const BatchHam &h, const BatchItem &it, uint32_t st, C *tile_dst,
                                                 unsigned char *blk_dst, uint64_t *bar) {
    constexpr uint32_t TR = 1u << LOGT;
    const uint4 info = __ldg(&h.step_info[st]);
    const uint64_t d = static_cast<uint64_t>(info.x) | (static_cast<uint64_t>(info.y) << 32);
    const uint32_t blk_bytes = (info.w >> 16) * 16u;
    mbar_arrive_expect_tx(bar, RB * TR * static_cast<uint32_t>(sizeof(C)) + blk_bytes);
    const C *x = static_cast<const C *>(h.x);
    const uint64_t src_row = (it.tile ^ d) << LOGT;
#pragma unroll
    for (int r = 0; r < RB; ++r) {
        bulk_copy_g2s(tile_dst + r * TR, x + (it.rhs0 + r) * h.dim + src_row, TR * sizeof(C), bar);
    }
    bulk_copy_g2s(blk_dst, h.blocks + static_cast<size_t>(info.z) * 16u, blk_bytes, bar);
}

template <int LOGT, int RB, typename R>
__global__ void __launch_bounds__(1 << LOGT, 1)
    k_batched(const BatchHam *__restrict__ hams, const BatchItem *__restrict__ items, uint32_t nitems,
              unsigned int *__restrict__ counter, int *__restrict__ err) {
    using C = typename Cx<R>::T;
    constexpr uint32_t TR = 1u << LOGT;
    constexpr uint32_t TILE_ELEMS = RB * TR;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    C *tiles = reinterpret_cast<C *>(smem_raw);                   // [2][RB][TR]
    unsigned char *blks = smem_raw + 2 * TILE_ELEMS * sizeof(C);  // [2][kBlockBytesMax]
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ uint32_t s_next;
    const uint32_t tid = threadIdx.x;

    uint32_t cur;
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
        cur = atomicAdd(counter, 1u);
        s_next = cur < nitems ? atomicAdd(counter, 1u) : nitems;
        if (cur < nitems) {
            const BatchItem it = items[cur];
            issue_batch_step<C, LOGT, RB>(hams[it.ham], it, 0, tiles, blks, &bars[0]);
        }
    }
    __shared__ uint32_t s_cur;
    if (tid == 0) s_cur = cur;
    __syncthreads();
    cur = s_cur;
    uint32_t nxt = s_next;
    if (cur >= nitems) return;

    uint32_t k = 0;  // steps consumed by this CTA: buffer k & 1, phase (k >> 1) & 1
    Acc<R> acc[RB];
    while (true) {
        const BatchItem it = items[cur];
        const BatchHam h = hams[it.ham];
        for (uint32_t st = 0; st < h.nsteps; ++st, ++k) {
            const uint32_t b = k & 1u;
            const uint4 info = __ldg(&h.step_info[st]);
            const bool ok = mbar_wait_bounded(&bars[b], (k >> 1) & 1u);
            if (__syncthreads_or(!ok)) {
                if (tid == 0) atomicOr(err, kErrTimeout);
                return;
            }
            // Every thread has finished the previous step: the other buffers are free.
            if (tid == 0) {
                if (st + 1 < h.nsteps) {
                    fence_proxy_async_smem();
                    issue_batch_step<C, LOGT, RB>(h, it, st + 1, tiles + (b ^ 1u) * TILE_ELEMS,
                                                  blks + (b ^ 1u) * tcp::kBlockBytesMax, &bars[b ^ 1u]);
                } else if (nxt < nitems) {
                    fence_proxy_async_smem();
                    const BatchItem nit = items[nxt];
                    issue_batch_step<C, LOGT, RB>(hams[nit.ham], nit, 0, tiles + (b ^ 1u) * TILE_ELEMS,
                                                  blks + (b ^ 1u) * tcp::kBlockBytesMax, &bars[b ^ 1u]);
                }
            }
            const C *xs = tiles + b * TILE_ELEMS;
            const unsigned char *blk = blks + b * tcp::kBlockBytesMax;
            const uint32_t ng = info.w & 0xffffu;
            const uint4 *grp = reinterpret_cast<const uint4 *>(blk);
            const unsigned char *trm = blk + ng * tcp::kGroupRecBytes;
            for (uint32_t g = 0; g < ng; ++g) {
                const uint4 gr = grp[g];
                const uint32_t tl = tid ^ gr.x;  // every inner-mask bit is a thread bit
                C xv[RB];
#pragma unroll
                for (int r = 0; r < RB; ++r) xv[r] = xs[r * TR + tl];
                for (uint32_t t = gr.y; t < gr.z; ++t) {
                    const unsigned char *rp = trm + t * tcp::kTermRecBytes;
                    const ulonglong2 rec = *reinterpret_cast<const ulonglong2 *>(rp);
                    const C w = record_weight<R>(rp);
                    const uint64_t zt_tile = rec.y & it.tile;
                    const uint32_t base = __popc((static_cast<uint32_t>(rec.x) & tid) ^
                                                 static_cast<uint32_t>(zt_tile) ^
                                                 static_cast<uint32_t>(zt_tile >> 32)) &
                                          1u;
                    const uint32_t kind = static_cast<uint32_t>(rec.x >> 56);
                    const R wr = flip_by(w.x, base), wi = flip_by(w.y, base);
                    if (kind == tcp::kKindReal) {
#pragma unroll
                        for (int r = 0; r < RB; ++r) acc[r].add_real(wr, xv[r]);
                    } else if (kind == tcp::kKindImag) {
#pragma unroll
                        for (int r = 0; r < RB; ++r) acc[r].add_imag(wi, xv[r]);
                    } else {
#pragma unroll
                        for (int r = 0; r < RB; ++r) acc[r].add_complex(wr, wi, xv[r]);
                    }
                }
                if (((g + 1) % kCompensateGroups) == 0u || g + 1 == ng) {
#pragma unroll
                    for (int r = 0; r < RB; ++r) acc[r].compensate();
                }
            }
        }
        C *y = static_cast<C *>(h.y);
        const uint64_t row = (it.tile << LOGT) + tid;
#pragma unroll
        for (int r = 0; r < RB; ++r) {
            y[(it.rhs0 + r) * h.dim + row] = acc[r].value();
            acc[r] = Acc<R>();
        }
        // Advance: fetch the item after `nxt` (its first step is issued during
        // the last step of `nxt`).
        __syncthreads();
        if (tid == 0) s_next = nxt < nitems ? atomicAdd(counter, 1u) : nitems;
        __syncthreads();
        cur = nxt;
        nxt = s_next;
        if (cur >= nitems) break;
    }
}

// ------------------------------- variants ----------------------------------
struct Variant {
    uint32_t logt;
    uint32_t rb;
    bool c64;
    const void *fn;  // null for the ring configuration
    size_t smem;
};

constexpr uint32_t kRingLogt = 12;  // the ring configuration: (12, 1)

Variant ring_variant(bool c64) { return Variant{kRingLogt, 1, c64, nullptr, 0}; }

template <int LOGT, int RB, typename R> Variant make_variant() {
    Variant v;
    v.logt = LOGT;
    v.rb = RB;
    v.c64 = sizeof(R) == 4;
    v.fn = reinterpret_cast<const void *>(&k_batched<LOGT, RB, R>);
    v.smem = 2 * size_t(RB) * (size_t(1) << LOGT) * sizeof(typename Cx<R>::T) + 2 * size_t(tcp::kBlockBytesMax);
    return v;
}

const std::vector<Variant> &variants() {
    static const std::vector<Variant> all = {
        make_variant<8, 1, float>(),  make_variant<8, 2, float>(),  make_variant<8, 4, float>(),
        make_variant<8, 8, float>(),  make_variant<9, 1, float>(),  make_variant<9, 2, float>(),
        make_variant<9, 4, float>(),  make_variant<9, 8, float>(),  make_variant<10, 1, float>(),
        make_variant<10, 2, float>(), make_variant<10, 4, float>(), make_variant<8, 1, double>(),
        make_variant<8, 2, double>(), make_variant<8, 4, double>(), make_variant<8, 8, double>(),
        make_variant<9, 1, double>(), make_variant<9, 2, double>(), make_variant<9, 4, double>(),
        make_variant<9, 8, double>(), make_variant<10, 1, double>(), make_variant<10, 2, double>(),
        make_variant<10, 4, double>(), ring_variant(true), ring_variant(false),
    };
    return all;
}

const Variant *find_variant(uint32_t logt, uint32_t rb, bool c64) {
    for (const Variant &v : variants())
        if (v.logt == logt && v.rb == rb && v.c64 == c64) return &v;
    return nullptr;
}

uint64_t fnv1a(const std::string &s) {
    uint64_t h = 1469598103934665603ull;
    for (unsigned char c : s) {
        h ^= c;
        h *= 1099511628211ull;
    }
    return h;
}

}  // namespace

// One batch: its members, the current configuration, device tables, graph.
struct tcp_mvp_batch {
    std::vector<const tcp_mvp_plan *> plans;
    uint32_t nrhs = 1;
    bool c64 = false;
    int device = 0;
    uint32_t logt = 0;
    uint32_t rb = 0;
    // per configuration
    std::vector<tcp::Schedule> schedules;
    void *d_sched = nullptr;  // step infos and blocks of every member
    std::vector<BatchHam> hams_host;
    BatchHam *d_hams = nullptr;
    BatchItem *d_items = nullptr;
    uint32_t nitems = 0;
    std::vector<uint32_t> empty_members;  // members without terms: y is zeroed
    unsigned int *d_counter = nullptr;
    int *d_err = nullptr;
    int grid = 0;
    bool ring = false;                 // ring configuration: one launch per member
    std::vector<uint32_t> ring_order;  // members with terms, largest first
    // graph
    cudaStream_t capture_stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    std::vector<const void *> bound_x;
    std::vector<void *> bound_y;
    std::mutex mutex;
};

namespace {

void release_config(tcp_mvp_batch *b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    if (b->d_sched) cudaFree(b->d_sched);
    if (b->d_hams) cudaFree(b->d_hams);
    if (b->d_items) cudaFree(b->d_items);
    b->d_sched = nullptr;
    b->d_hams = nullptr;
    b->d_items = nullptr;
    b->schedules.clear();
    b->hams_host.clear();
    b->ring = false;
    b->ring_order.clear();
    b->bound_x.clear();
    b->bound_y.clear();
}

// The ring configuration: no batch schedules or work list; every member's own
// ring schedule serves its launch.
int configure_ring(tcp_mvp_batch *b) {
    if (b->nrhs > 65535u) return fail(TCP_ERR_INVALID_ARGUMENT, "the ring configuration takes at most 65535 right-hand sides");
    for (const tcp_mvp_plan *p : b->plans) {
        int st = tcp::ring_prepare(p, b->c64);
        if (st) return st;
    }
    release_config(b);
    b->logt = kRingLogt;
    b->rb = 1;
    b->ring = true;
    b->hams_host.assign(b->plans.size(), BatchHam{});
    b->empty_members.clear();
    std::vector<std::pair<double, uint32_t>> order;
    uint64_t ctas = 0;
    for (size_t h = 0; h < b->plans.size(); ++h) {
        const tcp_mvp_plan *p = b->plans[h];
        b->hams_host[h].dim = p->dim;
        b->hams_host[h].nqubits = p->nqubits;
        if (p->sched.dev.ring_steps == 0) {
            b->empty_members.push_back(static_cast<uint32_t>(h));
            continue;
        }
        order.push_back({static_cast<double>(p->terms.size()) * static_cast<double>(p->dim), static_cast<uint32_t>(h)});
        ctas += (p->dim >> kRingLogt) * b->nrhs;
    }
    std::stable_sort(order.begin(), order.end(), [](const auto &a, const auto &c) { return a.first > c.first; });
    for (const auto &o : order) b->ring_order.push_back(o.second);
    b->nitems = static_cast<uint32_t>(std::min<uint64_t>(ctas, 0xffffffffull));
    b->grid = static_cast<int>(b->ring_order.size());
    return TCP_OK;
}

// Build schedules, the work list and the device tables for (logt, rb).
int configure(tcp_mvp_batch *b, uint32_t logt, uint32_t rb) {
    const Variant *v = find_variant(logt, rb, b->c64);
    if (v == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "no batched kernel variant for this tile / RHS block");
    if (b->nrhs % rb != 0) return fail(TCP_ERR_INVALID_ARGUMENT, "the RHS block must divide the RHS count");
    if (v->fn == nullptr) return configure_ring(b);
    for (const tcp_mvp_plan *p : b->plans) {
        if (p->nqubits < logt) {
            return fail(TCP_ERR_INVALID_ARGUMENT, "every batch member needs at least " + std::to_string(logt) +
                                                      " qubits for this tile shape");
        }
    }
    release_config(b);
    b->logt = logt;
    b->rb = rb;
    // schedules and one device allocation for all of them
    size_t total = 0;
    std::vector<size_t> off_info, off_blk;
    for (const tcp_mvp_plan *p : b->plans) {
        b->schedules.push_back(tcp::build_schedule(p->terms, p->nqubits, logt, logt));
        const tcp::Schedule &s = b->schedules.back();
        const std::vector<uint8_t> &blk = b->c64 ? s.blocks_c64 : s.blocks_c128;
        off_info.push_back(total);
        total += (s.step_info.size() * 4 + 255) / 256 * 256;
        off_blk.push_back(total);
        total += (blk.size() + 255) / 256 * 256;
    }
    total = std::max<size_t>(total, 256);
    cudaError_t e = dev_malloc(&b->d_sched, total);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(TCP_ERR_ALLOCATION, "device allocation of the batch schedules failed");
    }
    std::vector<unsigned char> staging(total, 0);
    b->hams_host.resize(b->plans.size());
    b->empty_members.clear();
    struct Cost {
        double cost;
        uint32_t ham;
    };
    std::vector<Cost> order;
    for (size_t h = 0; h < b->plans.size(); ++h) {
        const tcp::Schedule &s = b->schedules[h];
        const std::vector<uint8_t> &blk = b->c64 ? s.blocks_c64 : s.blocks_c128;
        std::memcpy(staging.data() + off_info[h], s.step_info.data(), s.step_info.size() * 4);
        std::memcpy(staging.data() + off_blk[h], blk.data(), blk.size());
        BatchHam &bh = b->hams_host[h];
        bh.step_info = reinterpret_cast<const uint4 *>(static_cast<unsigned char *>(b->d_sched) + off_info[h]);
        bh.blocks = static_cast<unsigned char *>(b->d_sched) + off_blk[h];
        bh.x = nullptr;
        bh.y = nullptr;
        bh.dim = b->plans[h]->dim;
        bh.nsteps = static_cast<uint32_t>(s.step_info.size() / 4);
        bh.nqubits = b->plans[h]->nqubits;
        if (bh.nsteps == 0) {
            b->empty_members.push_back(static_cast<uint32_t>(h));
        } else {
            order.push_back({static_cast<double>(b->plans[h]->terms.size() + bh.nsteps) * static_cast<double>(bh.dim),
                             static_cast<uint32_t>(h)});
        }
    }
    e = cudaMemcpy(b->d_sched, staging.data(), total, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "batch schedule upload");
    // work list: largest Hamiltonian first, tiles in order, RHS blocks inside
    std::stable_sort(order.begin(), order.end(), [](const Cost &a, const Cost &c) { return a.cost > c.cost; });
    std::vector<BatchItem> items;
    for (const Cost &c : order) {
        const uint64_t tiles = b->plans[c.ham]->dim >> logt;
        for (uint64_t t = 0; t < tiles; ++t)
            for (uint32_t r0 = 0; r0 < b->nrhs; r0 += rb) items.push_back(BatchItem{c.ham, r0, t});
    }
    if (items.size() >= 0xffffffffull) return fail(TCP_ERR_OVERFLOW, "integer overflow while counting batch items");
    b->nitems = static_cast<uint32_t>(items.size());
    e = dev_malloc(reinterpret_cast<void **>(&b->d_hams), sizeof(BatchHam) * std::max<size_t>(1, b->hams_host.size()));
    if (e == cudaSuccess)
        e = dev_malloc(reinterpret_cast<void **>(&b->d_items), sizeof(BatchItem) * std::max<size_t>(1, items.size()));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(TCP_ERR_ALLOCATION, "device allocation of the batch work list failed");
    }
    if (!items.empty()) {
        e = cudaMemcpy(b->d_items, items.data(), sizeof(BatchItem) * items.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_fail(e, "batch work list upload");
    }
    e = cudaFuncSetAttribute(v->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(v->smem));
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute (batched kernel)");
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, v->fn, 1 << logt, v->smem);
    if (e != cudaSuccess) return cuda_fail(e, "occupancy query (batched kernel)");
    if (per_sm < 1) return fail(TCP_ERR_INVALID_ARGUMENT, "batched kernel variant does not fit on an SM");
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    b->grid = std::max(1, std::min<int>(sms * per_sm, static_cast<int>(std::max<uint32_t>(1, b->nitems))));
    return TCP_OK;
}

int bind_buffers(tcp_mvp_batch *b, const void *const *d_x, void *const *d_y, cudaStream_t stream, bool *changed) {
    *changed = false;
    if (b->bound_x.size() != b->plans.size()) {
        b->bound_x.assign(b->plans.size(), nullptr);
        b->bound_y.assign(b->plans.size(), nullptr);
        *changed = true;
    }
    for (size_t h = 0; h < b->plans.size(); ++h) {
        if (d_x[h] == nullptr || d_y[h] == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "null batch buffer");
        if (reinterpret_cast<uintptr_t>(d_x[h]) % 16 != 0) return fail(TCP_ERR_INVALID_ARGUMENT, "batch input not 16-byte aligned");
        const size_t bytes = b->plans[h]->dim * b->nrhs * (b->c64 ? 8 : 16);
        if (tcp::overlaps(d_x[h], d_y[h], bytes)) return fail(TCP_ERR_INVALID_ARGUMENT, "input and output must not overlap");
        if (b->bound_x[h] != d_x[h] || b->bound_y[h] != d_y[h]) *changed = true;
        b->bound_x[h] = d_x[h];
        b->bound_y[h] = d_y[h];
        b->hams_host[h].x = d_x[h];
        b->hams_host[h].y = d_y[h];
    }
    if (*changed && !b->hams_host.empty() && !b->ring) {
        cudaError_t e = cudaMemcpyAsync(b->d_hams, b->hams_host.data(), sizeof(BatchHam) * b->hams_host.size(),
                                        cudaMemcpyHostToDevice, stream);
        if (e != cudaSuccess) return cuda_fail(e, "batch descriptor upload");
    }
    return TCP_OK;
}

// Record the batch's launch sequence on `s` (used under stream capture).
int record_launch(tcp_mvp_batch *b, cudaStream_t s) {
    if (b->ring) {
        for (uint32_t h : b->empty_members) {
            cudaError_t e = cudaMemsetAsync(b->hams_host[h].y, 0, b->plans[h]->dim * b->nrhs * (b->c64 ? 8 : 16), s);
            if (e != cudaSuccess) return cuda_fail(e, "zeroing an empty member");
        }
        for (uint32_t h : b->ring_order) {
            int st = tcp::launch_ring_rhs(b->plans[h], b->hams_host[h].x, b->hams_host[h].y, b->nrhs, b->c64, b->d_err, s);
            if (st) return st;
        }
        return TCP_OK;
    }
    const Variant *v = find_variant(b->logt, b->rb, b->c64);
    cudaError_t e = cudaMemsetAsync(b->d_counter, 0, sizeof(unsigned int), s);
    if (e != cudaSuccess) return cuda_fail(e, "batch counter reset");
    for (uint32_t h : b->empty_members) {
        e = cudaMemsetAsync(b->hams_host[h].y, 0, b->plans[h]->dim * b->nrhs * (b->c64 ? 8 : 16), s);
        if (e != cudaSuccess) return cuda_fail(e, "zeroing an empty member");
    }
    if (b->nitems == 0) return TCP_OK;
    void *args[] = {&b->d_hams, &b->d_items, &b->nitems, &b->d_counter, &b->d_err};
    e = cudaLaunchKernel(v->fn, dim3(b->grid), dim3(1u << b->logt), args, v->smem, s);
    if (e != cudaSuccess) return cuda_fail(e, "batched kernel launch");
    return TCP_OK;
}

int build_graph(tcp_mvp_batch *b) {
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(b->capture_stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamBeginCapture");
    int st = record_launch(b, b->capture_stream);
    e = cudaStreamEndCapture(b->capture_stream, &g);
    if (st) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
    return TCP_OK;
}

int apply_locked(tcp_mvp_batch *b, const void *const *d_x, void *const *d_y, cudaStream_t stream) {
    bool changed = false;
    int st = bind_buffers(b, d_x, d_y, stream, &changed);
    if (st) return st;
    // The persistent kernel's graph only captures pointers to device tables,
    // except the memsets of empty members' outputs; the ring configuration's
    // launches take the buffers themselves.  Rebuild the graph when the
    // configuration or the captured buffers change.
    if (b->graph == nullptr || (changed && (b->ring || !b->empty_members.empty()))) {
        st = build_graph(b);
        if (st) return st;
    }
    cudaError_t e = cudaGraphLaunch(b->graph, stream);
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "cudaGraphLaunch");
}

int check_batch(tcp_mvp_batch *b) {
    if (b == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "batch is null");
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev != b->device) return fail(TCP_ERR_WRONG_DEVICE, "batch used on another device");
    return TCP_OK;
}

std::string cache_key(const tcp_mvp_batch *b) {
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, b->device);
    std::ostringstream k;
    k << prop.name << "|" << (b->c64 ? "c64" : "c128") << "|" << b->nrhs;
    for (const tcp_mvp_plan *p : b->plans) k << "|" << p->nqubits << ":" << p->terms.size() << ":" << p->group_count;
    char buf[32];
    std::snprintf(buf, sizeof buf, "%016llx", static_cast<unsigned long long>(fnv1a(k.str())));
    return buf;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" int tcp_mvp_batch_create(uint32_t count, const tcp_mvp_plan *const *plans, uint32_t nrhs, int dtype,
                                    tcp_mvp_batch **out_batch) {
    if (out_batch == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "out_batch is null");
    *out_batch = nullptr;
    if (count == 0 || plans == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "a batch needs at least one plan");
    if (nrhs == 0) return fail(TCP_ERR_INVALID_ARGUMENT, "a batch needs at least one right-hand side");
    if (dtype != TCP_DTYPE_C128 && dtype != TCP_DTYPE_C64) return fail(TCP_ERR_INVALID_ARGUMENT, "unknown dtype");
    std::unique_ptr<tcp_mvp_batch> b(new tcp_mvp_batch());
    b->nrhs = nrhs;
    b->c64 = dtype == TCP_DTYPE_C64;
    cudaError_t e = cudaGetDevice(&b->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    for (uint32_t i = 0; i < count; ++i) {
        int st = tcp::check_plan(plans[i]);
        if (st) return st;
        b->plans.push_back(plans[i]);
    }
    e = dev_malloc(reinterpret_cast<void **>(&b->d_counter), 256);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(TCP_ERR_ALLOCATION, "device allocation of the batch counter failed");
    }
    b->d_err = reinterpret_cast<int *>(reinterpret_cast<unsigned char *>(b->d_counter) + 128);
    cudaMemset(b->d_counter, 0, 256);
    e = cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        cudaFree(b->d_counter);
        return cuda_fail(e, "cudaStreamCreate");
    }
    // persistent-kernel default: 512-row tiles, the largest RHS block dividing nrhs
    uint32_t rb = 8;
    while (rb > 1 && nrhs % rb != 0) rb >>= 1;
    uint32_t logt = 9;
    for (const tcp_mvp_plan *p : b->plans) logt = std::min(logt, p->nqubits);
    if (logt < 8) {
        cudaStreamDestroy(b->capture_stream);
        cudaFree(b->d_counter);
        return fail(TCP_ERR_INVALID_ARGUMENT, "batched plans need at least 8 qubits");
    }
    // the ring configuration when every member can run it (measured faster
    // on the 64-lattice set), else the persistent kernel
    bool ring = b->nrhs <= 65535u;
    for (const tcp_mvp_plan *p : b->plans) ring = ring && p->nqubits >= kRingLogt;
    int st = ring ? configure(b.get(), kRingLogt, 1) : TCP_ERR_INVALID_ARGUMENT;
    if (st) st = configure(b.get(), logt, rb);
    if (st) {
        release_config(b.get());
        cudaStreamDestroy(b->capture_stream);
        cudaFree(b->d_counter);
        return st;
    }
    *out_batch = b.release();
    return TCP_OK;
}

extern "C" int tcp_mvp_batch_destroy(tcp_mvp_batch *b) {
    if (b == nullptr) return TCP_OK;
    release_config(b);
    if (b->capture_stream) cudaStreamDestroy(b->capture_stream);
    if (b->d_counter) cudaFree(b->d_counter);
    delete b;
    return TCP_OK;
}

extern "C" int tcp_mvp_batch_configure(tcp_mvp_batch *b, uint32_t tile_rows_log2, uint32_t rhs_block) {
    int st = check_batch(b);
    if (st) return st;
    std::lock_guard<std::mutex> lock(b->mutex);
    return configure(b, tile_rows_log2, rhs_block);
}

extern "C" int tcp_mvp_batch_apply(tcp_mvp_batch *b, const void *const *d_x, void *const *d_y, void *stream) {
    tcp::Range range("tcp_mvp_batch_apply");
    int st = check_batch(b);
    if (st) return st;
    if (d_x == nullptr || d_y == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer table");
    std::lock_guard<std::mutex> lock(b->mutex);
    return apply_locked(b, d_x, d_y, static_cast<cudaStream_t>(stream));
}

extern "C" int tcp_mvp_batch_info(const tcp_mvp_batch *b, uint32_t *tile_rows_log2, uint32_t *rhs_block,
                                  uint64_t *items, uint32_t *grid) {
    if (b == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "batch is null");
    if (tile_rows_log2) *tile_rows_log2 = b->logt;
    if (rhs_block) *rhs_block = b->rb;
    if (items) *items = b->nitems;
    if (grid) *grid = static_cast<uint32_t>(b->grid);
    return TCP_OK;
}

extern "C" int tcp_mvp_batch_device_status(tcp_mvp_batch *b) {
    int st = check_batch(b);
    if (st) return st;
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceSynchronize");
    int h = 0;
    e = cudaMemcpy(&h, b->d_err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "reading the batch status");
    if (h) {
        cudaMemset(b->d_err, 0, sizeof(int));
        return fail(TCP_ERR_DEVICE_TIMEOUT, "a bounded device-side wait expired in the batched kernel");
    }
    return TCP_OK;
}

extern "C" int tcp_mvp_batch_autotune(tcp_mvp_batch *b, const void *const *d_x, void *const *d_y,
                                      const char *cache_path, uint32_t repeats, void *stream) {
    int st = check_batch(b);
    if (st) return st;
    if (d_x == nullptr || d_y == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer table");
    std::lock_guard<std::mutex> lock(b->mutex);
    const std::string key = cache_key(b);
    if (cache_path != nullptr && *cache_path) {
        std::ifstream in(cache_path);
        std::string k;
        uint32_t logt = 0, rb = 0;
        while (in >> k >> logt >> rb) {
            if (k == key) return configure(b, logt, rb);
        }
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best_ms = 1e30f;
    uint32_t best_logt = b->logt, best_rb = b->rb;
    repeats = std::max<uint32_t>(repeats, 1);
    for (const Variant &v : variants()) {
        if (v.c64 != b->c64 || b->nrhs % v.rb != 0) continue;
        if (configure(b, v.logt, v.rb) != TCP_OK) continue;
        if (apply_locked(b, d_x, d_y, s) != TCP_OK) continue;  // warm-up (and graph build)
        cudaEventRecord(e0, s);
        bool ok = true;
        for (uint32_t r = 0; r < repeats && ok; ++r) ok = apply_locked(b, d_x, d_y, s) == TCP_OK;
        cudaEventRecord(e1, s);
        if (cudaEventSynchronize(e1) != cudaSuccess || !ok) {
            cudaGetLastError();
            continue;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_ms) {
            best_ms = ms;
            best_logt = v.logt;
            best_rb = v.rb;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    st = configure(b, best_logt, best_rb);
    if (st) return st;
    if (cache_path != nullptr && *cache_path) {
        std::ofstream outf(cache_path, std::ios::app);
        outf << key << " " << best_logt << " " << best_rb << "\n";
    }
    return TCP_OK;
}
