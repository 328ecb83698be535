// Dense / COO / CSR materialisation of a full-space plan (include/tcp_matrix.h).
//
// Reference (paths inside the TenCirPauli project):
//   crates/tencir-pauli-core/src/hamiltonian.rs:311-478  dense_matrix, coo_matrix, csr_matrix
//   crates/tencir-pauli-core/src/hamiltonian.rs:584-770  sparse_entries, fill_sparse_row, sort_sparse_row
//
// The plan's group view holds the x-mask groups in ascending mask order with
// their terms in canonical order, so a group value summed term by term from 0
// is the reference's value bit for bit (additions only, no fused products).
// Sparse rows: count nonzero groups per row, exclusive scan, fill in group
// order, then a CUB segmented sort orders the columns of every row.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <string>

#include "../../include/tcp_matrix.h"
#include "tcp_internal.h"
#include "tcp_plan_impl.h"

using tcp::fail;

namespace {

constexpr int kMxThreads = 256;

__device__ __forceinline__ double2 group_value_at(const tcpdev::DevSchedule &s, uint32_t g, uint64_t column) {
    double re = 0.0, im = 0.0;
    for (uint32_t t = s.g_tbeg[g]; t < s.g_tbeg[g + 1]; ++t) {
        const double2 w = s.t_w[t];
        if (__popcll(s.t_z[t] & column) & 1) {
            re = re - w.x;
            im = im - w.y;
        } else {
            re = re + w.x;
            im = im + w.y;
        }
    }
    return make_double2(re, im);
}

// Dense: every (row, group) pair writes its value at (row, row ^ mask).
__global__ void k_mx_dense(tcpdev::DevSchedule s, uint32_t ngroups, uint64_t dim, double2 *__restrict__ out) {
    const uint64_t total = static_cast<uint64_t>(ngroups) * dim;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t row = i / ngroups;
        const uint32_t g = static_cast<uint32_t>(i % ngroups);
        const uint64_t column = row ^ s.g_mask[g];
        out[row * dim + column] = group_value_at(s, g, column);
    }
}

__global__ void k_mx_count(tcpdev::DevSchedule s, uint32_t ngroups, uint64_t dim, uint64_t *__restrict__ counts) {
    for (uint64_t row = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; row < dim;
         row += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint64_t c = 0;
        for (uint32_t g = 0; g < ngroups; ++g) {
            const double2 v = group_value_at(s, g, row ^ s.g_mask[g]);
            c += (v.x != 0.0 || v.y != 0.0);
        }
        counts[row] = c;
    }
}

__global__ void k_mx_fill(tcpdev::DevSchedule s, uint32_t ngroups, uint64_t dim, const uint64_t *__restrict__ indptr,
                          uint64_t *__restrict__ cols, double2 *__restrict__ vals) {
    for (uint64_t row = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; row < dim;
         row += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint64_t pos = indptr[row];
        for (uint32_t g = 0; g < ngroups; ++g) {
            const uint64_t column = row ^ s.g_mask[g];
            const double2 v = group_value_at(s, g, column);
            if (v.x == 0.0 && v.y == 0.0) continue;
            cols[pos] = column;
            vals[pos] = v;
            ++pos;
        }
    }
}

int grid_of(uint64_t work) {
    return static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>((work + kMxThreads - 1) / kMxThreads, 148ull * 32)));
}

std::string bytes_text(unsigned __int128 v) {
    return v >> 64 ? std::string("more than 2^64") : std::to_string(static_cast<uint64_t>(v));
}

int memory_limit(unsigned __int128 requested, uint64_t limit) {
    return tcp::fail_fields(TCP_ERR_MEMORY_LIMIT,
                            "requested " + bytes_text(requested) + " bytes exceeds memory limit " + std::to_string(limit),
                            tcp::clamp_u64(requested), limit);
}

// The reference's budget for a sparse target (hamiltonian.rs:358-445):
// upper_bound = groups * dimension candidate entries.
int sparse_budget(const tcp_mvp_plan *p, int target, uint64_t max_bytes) {
    const unsigned __int128 dim = p->dim;
    const unsigned __int128 G = p->sched.host.g_mask.size();
    const unsigned __int128 upper = G * dim;
    bool direct = true;  // every group holds exactly one term
    const auto &tb = p->sched.host.g_tbeg;
    for (size_t g = 0; g + 1 < tb.size(); ++g) direct = direct && (tb[g + 1] - tb[g] == 1);
    const unsigned __int128 candidate = 24;  // SparseEntry: u64 column + complex128 value
    unsigned __int128 need = 0;
    if (target == TCP_MATRIX_COO) {
        need = direct ? upper * 32 : upper * (candidate + 32) + dim * 8;
    } else {
        const unsigned __int128 output = (dim + 1) * 8 + upper * 24;
        need = direct ? output : upper * candidate + output + dim * 8;
    }
    return need > max_bytes ? memory_limit(need, max_bytes) : TCP_OK;
}

int count_rows(const tcp_mvp_plan *p, uint64_t *d_counts) {
    const uint32_t G = static_cast<uint32_t>(p->sched.host.g_mask.size());
    if (G) k_mx_count<<<grid_of(p->dim), kMxThreads>>>(p->sched.dev, G, p->dim, d_counts);
    else cudaMemset(d_counts, 0, 8 * p->dim);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TCP_OK : tcp::cuda_fail(e, "counting sparse entries");
}

}  // namespace

extern "C" int tcp_mvp_dense(const tcp_mvp_plan *plan, double *out, uint64_t capacity, uint64_t max_bytes) {
    int st = tcp::check_plan(plan);
    if (st) return st;
    const unsigned __int128 entries = static_cast<unsigned __int128>(plan->dim) * plan->dim;
    if (entries * 16 > max_bytes) return memory_limit(entries * 16, max_bytes);
    if (entries > capacity) return fail(TCP_ERR_INVALID_ARGUMENT, "dense output buffer is too small");
    if (out == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "null output");
    const size_t bytes = static_cast<size_t>(entries) * 16;
    double2 *d = nullptr;
    cudaError_t e = tcp::dev_malloc(reinterpret_cast<void **>(&d), bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(TCP_ERR_ALLOCATION, "device allocation of the dense matrix failed");
    }
    e = cudaMemset(d, 0, bytes);
    const uint32_t G = static_cast<uint32_t>(plan->sched.host.g_mask.size());
    const uint64_t work = static_cast<uint64_t>(G) * plan->dim;
    if (e == cudaSuccess && work) {
        k_mx_dense<<<grid_of(work), kMxThreads>>>(plan->sched.dev, G, plan->dim, d);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, d, bytes, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? TCP_OK : tcp::cuda_fail(e, "building the dense matrix");
}

extern "C" int tcp_mvp_sparse_count(const tcp_mvp_plan *plan, int target, uint64_t max_bytes, uint64_t *out_nnz) {
    int st = tcp::check_plan(plan);
    if (st) return st;
    if (out_nnz == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "null output");
    if (target != TCP_MATRIX_COO && target != TCP_MATRIX_CSR) return fail(TCP_ERR_INVALID_ARGUMENT, "unknown target");
    st = sparse_budget(plan, target, max_bytes);
    if (st) return st;
    uint64_t total = 0;
    if (plan->sched.host.g_mask.empty()) {
        *out_nnz = 0;
        return TCP_OK;
    }
    // the transition count is the same quantity, counted without row storage
    st = tcp_mvp_transition_count(plan, &total);
    if (!st) *out_nnz = total;
    return st;
}

extern "C" int tcp_mvp_csr(const tcp_mvp_plan *plan, int target, uint64_t max_bytes, uint64_t *indptr,
                           uint64_t *columns, double *values, uint64_t capacity, uint64_t *out_nnz) {
    int st = tcp::check_plan(plan);
    if (st) return st;
    if (indptr == nullptr || out_nnz == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "null output");
    if (target != TCP_MATRIX_COO && target != TCP_MATRIX_CSR) return fail(TCP_ERR_INVALID_ARGUMENT, "unknown target");
    st = sparse_budget(plan, target, max_bytes);
    if (st) return st;
    const uint64_t D = plan->dim;
    if (D >= (1ull << 31)) return fail(TCP_ERR_OVERFLOW, "integer overflow while sizing the sparse rows (at most 2^31 - 1 rows)");
    uint64_t *d_counts = nullptr, *d_indptr = nullptr, *d_cols = nullptr;
    double2 *d_vals = nullptr;
    void *tmp = nullptr;
    cudaError_t e = tcp::dev_malloc(reinterpret_cast<void **>(&d_counts), 8 * (D + 1));
    if (e == cudaSuccess) e = tcp::dev_malloc(reinterpret_cast<void **>(&d_indptr), 8 * (D + 1));
    if (e != cudaSuccess) {
        cudaGetLastError();
        cudaFree(d_counts);
        return fail(TCP_ERR_ALLOCATION, "device allocation of the sparse row counts failed");
    }
    cudaMemset(d_counts, 0, 8 * (D + 1));
    st = count_rows(plan, d_counts);
    size_t scan_bytes = 0, sort_bytes = 0;
    uint64_t nnz = 0;
    if (!st) {
        cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, d_counts, d_indptr, static_cast<int>(D + 1));
        e = cudaMalloc(&tmp, std::max<size_t>(scan_bytes, 16));
        if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp, scan_bytes, d_counts, d_indptr, static_cast<int>(D + 1));
        if (e == cudaSuccess) e = cudaMemcpy(&nnz, d_indptr + D, 8, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) st = tcp::cuda_fail(e, "scanning sparse row counts");
    }
    if (!st) {
        *out_nnz = nnz;
        if (nnz >= (1ull << 31)) st = fail(TCP_ERR_OVERFLOW, "integer overflow while sizing the sparse entries (at most 2^31 - 1)");
        else if (nnz > capacity) st = fail(TCP_ERR_INVALID_ARGUMENT, "sparse output needs " + std::to_string(nnz) + " entries, capacity is " + std::to_string(capacity));
        else if (nnz && (columns == nullptr || values == nullptr)) st = fail(TCP_ERR_INVALID_ARGUMENT, "null output");
    }
    if (!st && nnz) {
        e = tcp::dev_malloc(reinterpret_cast<void **>(&d_cols), 16 * nnz);
        if (e == cudaSuccess) e = tcp::dev_malloc(reinterpret_cast<void **>(&d_vals), 32 * nnz);
        if (e != cudaSuccess) {
            cudaGetLastError();
            st = fail(TCP_ERR_ALLOCATION, "device allocation of the sparse arrays failed");
        }
    }
    if (!st && nnz) {
        const uint32_t G = static_cast<uint32_t>(plan->sched.host.g_mask.size());
        k_mx_fill<<<grid_of(D), kMxThreads>>>(plan->sched.dev, G, D, d_indptr, d_cols, d_vals);
        e = cudaGetLastError();
        uint64_t *cols_out = d_cols + nnz;
        double2 *vals_out = d_vals + nnz;
        if (e == cudaSuccess) {
            cub::DeviceSegmentedSort::SortPairs(nullptr, sort_bytes, d_cols, cols_out, d_vals, vals_out,
                                                static_cast<int>(nnz), static_cast<int>(D), d_indptr, d_indptr + 1);
            cudaFree(tmp);
            tmp = nullptr;
            e = cudaMalloc(&tmp, std::max<size_t>(sort_bytes, 16));
        }
        if (e == cudaSuccess)
            e = cub::DeviceSegmentedSort::SortPairs(tmp, sort_bytes, d_cols, cols_out, d_vals, vals_out,
                                                    static_cast<int>(nnz), static_cast<int>(D), d_indptr, d_indptr + 1);
        if (e == cudaSuccess) e = cudaMemcpy(columns, cols_out, 8 * nnz, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(values, vals_out, 16 * nnz, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) st = tcp::cuda_fail(e, "building the sparse arrays");
    }
    if (!st) {
        e = cudaMemcpy(indptr, d_indptr, 8 * (D + 1), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) st = tcp::cuda_fail(e, "copying the row pointers");
    }
    cudaFree(tmp);
    cudaFree(d_cols);
    cudaFree(d_vals);
    cudaFree(d_counts);
    cudaFree(d_indptr);
    return st;
}
