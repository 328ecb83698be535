// Fixed-Hamming-weight (U(1)) sector MVP of libtcpmvp.so: host plan builder,
// combinatorial ranking, device kernels and the C ABI of include/tcp_sector.h.
//
// Reference (paths inside the TenCirPauli project):
//   crates/tencir-pauli-core/src/sector.rs   U1Sector, U1LazyMvpPlan, U1RestrictedOperator
//   crates/tencir-pauli-core/src/operator.rs:396-444  number-charge selection rule
//
// Layout on the device.  A plan holds
//   basis[i]   the i-th sector state as a TensorCircuit integer (uint32 when
//              n <= 32, else uint64), generated on the device by unranking
//              one index per thread and stepping to the next state of equal
//              weight (Gosper's rule);
//   rank tables T[c][a][v] (8-bit chunks c of the state, a = ones above the
//              chunk, v = chunk value): the number of sector states that agree
//              with s above chunk c and have a smaller chunk c.  The rank of a
//              state is the sum over its chunks, so one rank costs one table
//              load and one popcount per chunk.  With k > n - k the tables
//              rank the n - k holes instead and rank = D - 1 - rank(~s);
//   groups     distinct x masks in first-appearance order of the canonical
//              terms (compile_terms, sector.rs:926-1021) with their terms'
//              z masks and weighted coefficients c * i^{#Y}.
// The apply kernel is destination-major: thread i owns output row i, walks
// the groups, keeps those whose source b_i ^ m has weight k, sums the group's
// signed weights at that source (in canonical term order, from 0, as
// aggregate_source does), skips exact zeros, ranks the source and gathers it.
// When the tables, groups and terms fit they are staged in shared memory.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/tcp_sector.h"
#include "tcp_internal.h"

using tcp::fail;

namespace {

constexpr int kU1Threads = 256;
constexpr size_t kU1SmemMax = 160 * 1024;

inline uint32_t word_count_of(uint32_t n) { return n / 64 + (n % 64 != 0); }

int cuda_fail(cudaError_t e, const char *what) {
    return fail(TCP_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// ------------------------------ combinatorics ------------------------------
// Exact binomial with a 128-bit running product (choose_u64, sector.rs:1342-1362).
bool choose_u64(uint64_t n, uint64_t k, uint64_t &out) {
    if (k > n) {
        out = 0;
        return true;
    }
    k = std::min(k, n - k);
    unsigned __int128 v = 1;
    for (uint64_t i = 1; i <= k; ++i) {
        v = v * (n - k + i) / i;
        if (v > static_cast<unsigned __int128>(~0ull)) return false;
    }
    out = static_cast<uint64_t>(v);
    return true;
}

int sector_dimension(uint32_t n, uint32_t k, uint64_t &dim) {
    if (k > n) return fail(TCP_ERR_INVALID_SECTOR, "invalid sector: particle_number must be between 0 and nqubits");
    if (!choose_u64(n, k, dim)) return fail(TCP_ERR_OVERFLOW, "integer overflow while representing U1 sector dimension as u64");
    return TCP_OK;
}

std::string leak_message(uint64_t source, uint32_t expected, uint32_t actual) {
    return "U(1) sector leakage from restricted source index " + std::to_string(source) +
           ": expected particle number " + std::to_string(expected) + ", got destination weight " +
           std::to_string(actual);
}

// Rank of a sector state given by its set qubits: the number of weight-k
// states below it in TensorCircuit integer order.  Qubit q is integer bit
// n-1-q, so the states are ordered by their lowest-numbered differing qubit.
// Walking qubits upward, every set qubit q counts the states that agree on
// the qubits before q, have q clear, and place the remaining ones after q.
int rank_packed(uint32_t n, uint32_t k, const uint64_t *words, uint32_t wc, uint64_t &rank) {
    uint32_t expected = word_count_of(n);
    if (wc != expected) {
        return tcp::fail_fields(TCP_ERR_INVALID_WORD_LENGTH,
                                "expected " + std::to_string(expected) + " packed words, got " + std::to_string(wc),
                                expected, wc);
    }
    if (n % 64 && wc && (words[wc - 1] >> (n % 64))) {
        return fail(TCP_ERR_INVALID_INDEX, "invalid sector index: packed basis word has nonzero padding bits");
    }
    uint64_t weight = 0;
    for (uint32_t w = 0; w < wc; ++w) weight += __builtin_popcountll(words[w]);
    if (weight != k) return fail(TCP_ERR_INVALID_INDEX, "invalid sector index: packed basis word has the wrong Hamming weight");
    uint64_t r = 0;
    uint32_t left = k;
    for (uint32_t q = 0; q < n && left; ++q) {
        if (!((words[q / 64] >> (q % 64)) & 1)) continue;
        uint64_t c = 0;
        choose_u64(n - q - 1, left, c);  // states with q clear: all `left` ones after q
        r += c;
        --left;
    }
    rank = r;
    return TCP_OK;
}

int unrank_packed(uint32_t n, uint32_t k, uint64_t dim, uint64_t index, uint64_t *words, uint32_t wc) {
    if (index >= dim) return fail(TCP_ERR_INVALID_INDEX, "invalid sector index: restricted basis index is out of range");
    uint32_t expected = word_count_of(n);
    if (wc != expected) {
        return tcp::fail_fields(TCP_ERR_INVALID_WORD_LENGTH,
                                "expected " + std::to_string(expected) + " packed words, got " + std::to_string(wc),
                                expected, wc);
    }
    std::fill(words, words + wc, 0ull);
    uint64_t r = index;
    uint32_t left = k;
    for (uint32_t q = 0; q < n && left; ++q) {
        uint64_t zero_count = 0;
        choose_u64(n - q - 1, left, zero_count);
        if (r >= zero_count) {
            r -= zero_count;
            words[q / 64] |= 1ull << (q % 64);
            --left;
        }
    }
    return TCP_OK;
}

// ----------------------------- compiled terms ------------------------------
struct U1Terms {
    std::vector<uint64_t> gx;   // group x masks (integer bit space, bit n-1-q)
    std::vector<uint32_t> gt;   // group g owns terms [gt[g], gt[g+1])
    std::vector<uint64_t> tz;   // term z masks
    std::vector<double> tw;     // weighted coefficients (re, im)
    uint64_t x_support = 0;     // sum of popcount(x) over groups
    uint64_t z_support = 0;     // sum of popcount(z) over terms
    int32_t gzero = -1;         // index of the x == 0 group
};

// compile_terms (sector.rs:926-1021): groups by x mask in first appearance
// order, terms in canonical order within a group, weighted coefficient
// c * i^{#Y} with the textbook complex product (:1034-1049).  Masks are kept
// in integer bit space (qubit q is bit n-1-q) as W 64-bit words, least
// significant word first (W = 1 for n <= 64).
int compile_u1(uint32_t n, uint64_t count, uint32_t wc, const uint64_t *xw, const uint64_t *zw, const double *coef,
               uint32_t W, U1Terms &out) {
    uint32_t expected = word_count_of(n);
    if (wc != expected) {
        return tcp::fail_fields(TCP_ERR_INVALID_WORD_LENGTH,
                                "expected " + std::to_string(expected) + " packed words, got " + std::to_string(wc),
                                expected, wc);
    }
    std::map<std::vector<uint64_t>, uint32_t> lookup;
    std::vector<uint32_t> group_of(count);
    std::vector<uint64_t> xm(count * W), zm(count * W);
    std::vector<double> w(2 * count);
    std::vector<uint32_t> counts;
    std::vector<uint64_t> key(W);
    for (uint64_t t = 0; t < count; ++t) {
        double re = coef[2 * t], im = coef[2 * t + 1];
        if (!std::isfinite(re) || !std::isfinite(im)) {
            return tcp::fail_fields(TCP_ERR_NON_FINITE_COEFFICIENT,
                                    "coefficient at index " + std::to_string(t) + " is not finite", t, 0);
        }
        uint32_t ny = 0;
        for (uint32_t q = 0; q < n; ++q) {
            const bool x = (xw[t * wc + q / 64] >> (q % 64)) & 1, z = (zw[t * wc + q / 64] >> (q % 64)) & 1;
            const uint32_t e = n - 1 - q;
            if (x) xm[t * W + e / 64] |= 1ull << (e % 64);
            if (z) zm[t * W + e / 64] |= 1ull << (e % 64);
            ny += x && z;
        }
        ny %= 4;
        double pr = ny == 0 ? 1.0 : (ny == 2 ? -1.0 : 0.0);
        double pi = ny == 1 ? 1.0 : (ny == 3 ? -1.0 : 0.0);
        w[2 * t] = re * pr - im * pi;
        w[2 * t + 1] = re * pi + im * pr;
        key.assign(xm.begin() + t * W, xm.begin() + (t + 1) * W);
        auto it = lookup.find(key);
        uint32_t g;
        if (it == lookup.end()) {
            g = static_cast<uint32_t>(counts.size());
            lookup.emplace(key, g);
            bool zero = true;
            for (uint64_t v : key) {
                out.gx.push_back(v);
                out.x_support += __builtin_popcountll(v);
                zero = zero && v == 0;
            }
            counts.push_back(0);
            if (zero) out.gzero = static_cast<int32_t>(g);
        } else {
            g = it->second;
        }
        group_of[t] = g;
        ++counts[g];
    }
    const size_t G = counts.size();
    out.gt.assign(G + 1, 0);
    for (size_t g = 0; g < G; ++g) out.gt[g + 1] = out.gt[g] + counts[g];
    std::vector<uint32_t> next(out.gt.begin(), out.gt.end() - 1);
    out.tz.assign(count * W, 0);
    out.tw.assign(2 * count, 0.0);
    for (uint64_t t = 0; t < count; ++t) {
        uint32_t slot = next[group_of[t]]++;
        for (uint32_t i = 0; i < W; ++i) {
            out.tz[slot * W + i] = zm[t * W + i];
            out.z_support += __builtin_popcountll(zm[t * W + i]);
        }
        out.tw[2 * slot] = w[2 * t];
        out.tw[2 * slot + 1] = w[2 * t + 1];
    }
    return TCP_OK;
}

// ------------------------------ device view --------------------------------
struct U1Dev {
    const void *basis;       // BT[dim]
    const void *tab;         // IT[nchunk * (kp + 1) * 256]
    const uint64_t *gx;      // [G]
    const uint32_t *gt;      // [G + 1]
    const uint64_t *tz;      // [T]
    const double2 *tw;       // [T]
    const float2 *twf;       // [T]
    const uint64_t *choose;  // [65 * 65] C(p, j)
    uint64_t dim;
    uint64_t mask;           // low n bits
    uint32_t n, k, kp, comp, nchunk, ngroups, nterms, pad;
};

// The apply kernel's view: only the groups that can map a sector state to a
// sector state (x != 0 with an even number of flips), masks in the state word
// type ST (uint32 for n <= 32, else uint64), and the diagonal of the x == 0
// group evaluated once per plan.
//
// Constant groups.  On a source s = b ^ x inside the sector exactly half of
// the flipped qubits are set, so a term whose z mask meets x in nothing or in
// all of x has the fixed sign (-1)^{|x|/2 * [z & x == x]} there, and the rest
// of its z mask (z_out = z & ~x) reads the same bits in s as in the row b.
// When every term of a group has such a z & x and one common z_out (XX + YY
// exchange; Jordan-Wigner hopping with one Z string), the group's value is
// (-1)^{popcount(z_out & b)} * C with C summed once at plan build, in the
// canonical term order from 0 as the reference sums it -- negating a sum term
// by term negates it exactly, so the value is bit-identical.  A constant group
// with C == 0 never contributes and is dropped.  The groups are laid out in
// three segments -- constant without z_out (A), constant with z_out (B),
// general (C, the term loop) -- each padded to a multiple of kU1Unroll with
// groups that are never live (x = 0, half = 1).
//
// Fast ranks (n <= 32): rank(s) = H[top] + M[popcount(top)][mid] + L[low]
// (three levels) or H[s >> L] + L[s & (2^L - 1)] (two levels, no middle):
// H counts the sector states with a smaller top part, M those with the same
// top part and a smaller middle part, L ranks the low bits among words of
// their own weight.
constexpr int kU1Unroll = 4;

// Wide plans (64 < n <= 256): states are W 64-bit words in integer bit
// space, least significant word first; ranks use the 8-bit-chunk tables
// (read from global memory) and the basis is unranked index by index.  Wide
// sectors fit in memory only for small k or n - k, so these kernels keep the
// plain group loop.
struct U1WDev {
    const uint64_t *basis;   // [dim * W]
    const uint64_t *gx;      // [G * W]
    const uint32_t *gt;      // [G + 1]
    const uint64_t *tz;      // [T * W]
    const double2 *tw;       // [T]
    const float2 *twf;       // [T]
    const uint64_t *choose;  // [256 * 257] C(e, j), saturated
    const void *tab;         // IT[nchunk * (kp + 1) * 256]
    uint64_t dim, tail;      // tail: valid bits of the top word
    uint32_t n, k, kp, comp, nchunk, ngroups, nterms, pad;
};

template <typename ST> struct GRec;
template <> struct GRec<uint32_t> {
    uint32_t x, half;
};
template <> struct GRec<uint64_t> {
    uint64_t x;
    uint32_t half, pad;
};

struct U1Apply {
    const uint32_t *ftab;  // fast rank tables (rk 2 or 3), else null
    uint32_t rk, rL, rM, lmask, mmask, h_off, m_off, l_off;
    size_t ftab_bytes;
    const void *grec;      // GRec<ST>[na + nb + nc]: x mask and popcount(x) / 2
    const double2 *ac;     // [na + nb]: C of the constant groups
    const float2 *acf;     // [na + nb]: C rounded to FP32
    const void *azo;       // ST[nb]: z_out of segment B
    const uint32_t *at;    // [nc + 1]: term offsets of segment C
    const void *az;        // ST[ta]: term z masks
    const double2 *aw;     // [ta]
    const float2 *awf;     // [ta]
    const double2 *diag;   // [dim] or null when there is no x == 0 group
    uint32_t na, nb, nc, ta;
};

template <typename R> struct Cplx;
template <> struct Cplx<double> { using T = double2; };
template <> struct Cplx<float> { using T = float2; };

template <typename ST> __device__ __forceinline__ uint32_t popc_t(ST v);
template <> __device__ __forceinline__ uint32_t popc_t<uint32_t>(uint32_t v) { return static_cast<uint32_t>(__popc(v)); }
template <> __device__ __forceinline__ uint32_t popc_t<uint64_t>(uint64_t v) { return static_cast<uint32_t>(__popcll(v)); }

// Rank of a sector state: one table load per 8-bit chunk, top chunk first,
// `a` counting the ones above the chunk.  IT is wide enough for the dimension.
template <typename ST, typename IT>
__device__ __forceinline__ uint64_t rank_t(ST s, const IT *__restrict__ tab, const U1Dev &p) {
    const ST a_state = p.comp ? static_cast<ST>(~s & static_cast<ST>(p.mask)) : s;
    IT r = 0;
    uint32_t a = 0;
    const uint32_t row = (p.kp + 1) * 256u;
#pragma unroll
    for (int c = static_cast<int>(sizeof(ST)) - 1; c >= 0; --c) {
        if (c < static_cast<int>(p.nchunk)) {
            const uint32_t v = static_cast<uint32_t>(a_state >> (8 * c)) & 255u;
            r += tab[static_cast<uint32_t>(c) * row + a * 256u + v];
            a += __popc(v);
        }
    }
    return p.comp ? (p.dim - 1 - static_cast<uint64_t>(r)) : static_cast<uint64_t>(r);
}

template <typename IT>
__device__ __forceinline__ uint64_t rank_state(uint64_t s, const IT *__restrict__ tab, const U1Dev &p) {
    return rank_t<uint64_t, IT>(s, tab, p);
}

// Stage the rank tables, groups and terms in shared memory (16-byte aligned
// pieces, copied with 16-byte vector loads).
__host__ __device__ inline size_t al16(size_t v) { return (v + 15) & ~size_t(15); }

struct U1ApplySmem {
    size_t tab, grec, ac, azo, at, az, aw, total;
};

__host__ __device__ inline U1ApplySmem u1_apply_layout(size_t tab_bytes, uint32_t na, uint32_t nb, uint32_t nc,
                                                       uint32_t T, size_t sbytes, size_t wbytes) {
    const size_t rec = 2 * sbytes;  // GRec<ST>
    U1ApplySmem s;
    s.tab = 0;
    s.grec = al16(tab_bytes);
    s.ac = s.grec + al16(rec * (na + nb + nc));
    s.azo = s.ac + al16(wbytes * (na + nb));
    s.at = s.azo + al16(sbytes * nb);
    s.az = s.at + al16(4ull * (nc + 1));
    s.aw = s.az + al16(sbytes * T);
    s.total = s.aw + al16(wbytes * T);
    return s;
}

__device__ __forceinline__ void copy16(unsigned char *dst, const void *src, size_t bytes) {
    const uint4 *s = static_cast<const uint4 *>(src);
    uint4 *d = reinterpret_cast<uint4 *>(dst);
    const size_t n16 = bytes / 16;
    for (size_t i = threadIdx.x; i < n16; i += blockDim.x) d[i] = __ldg(s + i);
    const size_t rem = bytes - n16 * 16;
    if (threadIdx.x < rem) dst[n16 * 16 + threadIdx.x] = static_cast<const unsigned char *>(src)[n16 * 16 + threadIdx.x];
}


template <typename R> struct ApplyW;
template <> struct ApplyW<double> {
    static __device__ __forceinline__ const double2 *terms(const U1Apply &a) { return a.aw; }
    static __device__ __forceinline__ const double2 *consts(const U1Apply &a) { return a.ac; }
};
template <> struct ApplyW<float> {
    static __device__ __forceinline__ const float2 *terms(const U1Apply &a) { return a.awf; }
    static __device__ __forceinline__ const float2 *consts(const U1Apply &a) { return a.acf; }
};

// Rank of a sector state for rank kind RK (2, 3: fast tables; 0: 8-bit chunks).
template <int RK, typename ST, typename IT>
__device__ __forceinline__ uint64_t rank_any(ST s, const IT *__restrict__ tab, const U1Dev &p, const U1Apply &a) {
    if constexpr (RK == 2) {
        const uint32_t v = static_cast<uint32_t>(s);
        return static_cast<uint64_t>(tab[a.h_off + (v >> a.rL)] + tab[a.l_off + (v & a.lmask)]);
    } else if constexpr (RK == 3) {
        const uint32_t v = static_cast<uint32_t>(s);
        const uint32_t top = v >> (a.rM + a.rL);
        const uint32_t mid = (v >> a.rL) & a.mmask;
        return static_cast<uint64_t>(tab[a.h_off + top] + tab[a.m_off + (static_cast<uint32_t>(__popc(top)) << a.rM) + mid] +
                                     tab[a.l_off + (v & a.lmask)]);
    } else {
        return rank_t<ST, IT>(s, tab, p);
    }
}

template <typename R, typename C>
__device__ __forceinline__ void cmac(R &ar, R &ai, R &cr, R &ci, R vr, R vi, const C &xv) {
    const R pr = vr * xv.x - vi * xv.y;
    const R pi = vr * xv.y + vi * xv.x;
    if (sizeof(R) == 8) {
        ar += pr;
        ai += pi;
    } else {  // Kahan-compensated FP32 sum
        const R yr = pr - cr, yi = pi - ci;
        const R tr = ar + yr, ti = ai + yi;
        cr = (tr - ar) - yr;
        ci = (ti - ai) - yi;
        ar = tr;
        ai = ti;
    }
}

// y = H_sector x.  One output row per thread, grid-stride over rows.  Row i
// starts from diag[i] * x[i]; then the three group segments.  A group is live
// for row b when its source b ^ x lies in the sector (popcount(b & x) ==
// |x| / 2).  Each block of kU1Unroll groups is tested and ranked first, its
// gathers are issued back to back, then the live ones are accumulated.  A
// group that is not live loads the thread's own row, which is always valid,
// and is not added; neither is a general group whose value is exactly zero.
template <typename R, typename ST, typename IT, int RK, bool SM, bool DIAG>
__global__ void __launch_bounds__(kU1Threads) k_u1_apply(U1Dev p, U1Apply a, size_t tab_bytes,
                                                         const typename Cplx<R>::T *__restrict__ x,
                                                         typename Cplx<R>::T *__restrict__ y, uint64_t row0,
                                                         uint64_t row1) {
    using C = typename Cplx<R>::T;
    using G = GRec<ST>;
    constexpr int U = kU1Unroll;
    extern __shared__ __align__(16) unsigned char sm[];
    const IT *tab;
    const G *grec;
    const C *ac;
    const ST *azo;
    const uint32_t *at;
    const ST *az;
    const C *aw;
    const void *tab_src = RK ? static_cast<const void *>(a.ftab) : p.tab;
    const uint32_t nab = a.na + a.nb, nall = nab + a.nc;
    if (SM) {
        const U1ApplySmem L = u1_apply_layout(tab_bytes, a.na, a.nb, a.nc, a.ta, sizeof(ST), sizeof(C));
        copy16(sm + L.tab, tab_src, tab_bytes);
        copy16(sm + L.grec, a.grec, sizeof(G) * nall);
        copy16(sm + L.ac, ApplyW<R>::consts(a), sizeof(C) * nab);
        copy16(sm + L.azo, a.azo, sizeof(ST) * a.nb);
        copy16(sm + L.at, a.at, 4ull * (a.nc + 1));
        copy16(sm + L.az, a.az, sizeof(ST) * a.ta);
        copy16(sm + L.aw, ApplyW<R>::terms(a), sizeof(C) * a.ta);
        __syncthreads();
        tab = reinterpret_cast<const IT *>(sm + L.tab);
        grec = reinterpret_cast<const G *>(sm + L.grec);
        ac = reinterpret_cast<const C *>(sm + L.ac);
        azo = reinterpret_cast<const ST *>(sm + L.azo);
        at = reinterpret_cast<const uint32_t *>(sm + L.at);
        az = reinterpret_cast<const ST *>(sm + L.az);
        aw = reinterpret_cast<const C *>(sm + L.aw);
    } else {
        tab = static_cast<const IT *>(tab_src);
        grec = static_cast<const G *>(a.grec);
        ac = ApplyW<R>::consts(a);
        azo = static_cast<const ST *>(a.azo);
        at = a.at;
        az = static_cast<const ST *>(a.az);
        aw = ApplyW<R>::terms(a);
    }
    const ST *basis = static_cast<const ST *>(p.basis);
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = row0 + static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < row1; i += stride) {
        const ST b = basis[i];
        R ar = 0, ai = 0, cr = 0, ci = 0;
        if (DIAG) {
            const double2 d = a.diag[i];
            const R dr = static_cast<R>(d.x), di = static_cast<R>(d.y);
            if (dr != R(0) || di != R(0)) {
                const C xv = x[i];
                ar = dr * xv.x - di * xv.y;
                ai = dr * xv.y + di * xv.x;
            }
        }
        // segments A and B: constant values
        for (uint32_t g0 = 0; g0 < nab; g0 += U) {
            bool live[U];
            uint64_t j[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const G r = grec[g0 + u];
                live[u] = popc_t<ST>(b & r.x) == r.half;
                j[u] = live[u] ? rank_any<RK, ST, IT>(b ^ r.x, tab, p, a) : i;
            }
            C xv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) xv[u] = x[j[u]];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (!live[u]) continue;
                const C c = ac[g0 + u];
                R vr = c.x, vi = c.y;
                if (g0 >= a.na && (popc_t<ST>(azo[g0 + u - a.na] & b) & 1u)) {
                    vr = -vr;
                    vi = -vi;
                }
                cmac<R, C>(ar, ai, cr, ci, vr, vi, xv[u]);
            }
        }
        // segment C: general groups, term by term
        for (uint32_t g0 = nab; g0 < nall; g0 += U) {
            bool live[U];
            uint64_t j[U];
            R vr[U], vi[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const G r = grec[g0 + u];
                vr[u] = 0;
                vi[u] = 0;
                j[u] = i;
                live[u] = popc_t<ST>(b & r.x) == r.half;
                if (!live[u]) continue;
                const ST s = b ^ r.x;
                const uint32_t te = at[g0 + u - nab + 1];
                for (uint32_t t = at[g0 + u - nab]; t < te; ++t) {
                    const C w = aw[t];
                    if (popc_t<ST>(az[t] & s) & 1u) {
                        vr[u] -= w.x;
                        vi[u] -= w.y;
                    } else {
                        vr[u] += w.x;
                        vi[u] += w.y;
                    }
                }
                live[u] = vr[u] != R(0) || vi[u] != R(0);
                if (live[u]) j[u] = rank_any<RK, ST, IT>(s, tab, p, a);
            }
            C xv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) xv[u] = x[j[u]];
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (live[u]) cmac<R, C>(ar, ai, cr, ci, vr[u], vi[u], xv[u]);
        }
        C out;
        out.x = ar;
        out.y = ai;
        y[i] = out;
    }
}

// Group value of group g at source s in FP64 (canonical term order, from 0).
__device__ __forceinline__ double2 group_value(const U1Dev &p, uint32_t g, uint64_t s) {
    double vr = 0, vi = 0;
    for (uint32_t t = p.gt[g]; t < p.gt[g + 1]; ++t) {
        const double2 w = p.tw[t];
        if (__popcll(p.tz[t] & s) & 1) {
            vr -= w.x;
            vi -= w.y;
        } else {
            vr += w.x;
            vi += w.y;
        }
    }
    return make_double2(vr, vi);
}

// Sector basis: thread t writes rows [t*R, (t+1)*R): unrank the first, then
// step to the next larger integer of the same weight.
template <typename BT>
__global__ void k_u1_basis(U1Dev p, uint32_t rows_per_thread, BT *__restrict__ out) {
    const uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t i0 = t * rows_per_thread;
    if (i0 >= p.dim) return;
    // unrank i0: integer bit e = n-1-q; walk from the top bit down
    uint64_t r = i0, v = 0;
    uint32_t left = p.k;
    for (int e = static_cast<int>(p.n) - 1; e >= 0 && left; --e) {
        const uint64_t zero_count = p.choose[static_cast<uint32_t>(e) * 65u + left];  // C(e, left)
        if (r >= zero_count) {
            r -= zero_count;
            v |= 1ull << e;
            --left;
        }
    }
    const uint64_t end = min(p.dim, i0 + rows_per_thread);
    for (uint64_t i = i0; i < end; ++i) {
        out[i] = static_cast<BT>(v);
        if (i + 1 < end) {
            const uint64_t tt = v | (v - 1);
            const uint32_t shift = static_cast<uint32_t>(__ffsll(static_cast<long long>(v)));  // ctz(v) + 1
            const uint64_t low = (~tt & (tt + 1)) - 1;
            v = (tt + 1) | (shift >= 64 ? 0ull : (low >> shift));
        }
    }
}

// Leakage scan (U1RestrictedOperator::new, sector.rs:362-388 with
// aggregate_source :1051-1127): for every source, a group whose destination
// leaves the sector must aggregate to exactly zero.  Records the smallest
// (source, group) pair that does not.
template <typename BT>
__global__ void k_u1_leak(U1Dev p, unsigned long long *first) {
    const BT *basis = static_cast<const BT *>(p.basis);
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < p.dim; i += stride) {
        const uint64_t b = static_cast<uint64_t>(basis[i]);
        for (uint32_t g = 0; g < p.ngroups; ++g) {
            const uint64_t d = b ^ p.gx[g];
            if (static_cast<uint32_t>(__popcll(d)) == p.k) continue;
            const double2 v = group_value(p, g, b);
            if (v.x != 0.0 || v.y != 0.0) {
                atomicMin(first, static_cast<unsigned long long>(i * p.ngroups + g));
                break;
            }
        }
    }
}

// Nonzero entries per destination row (and their total).
template <typename BT>
__global__ void k_u1_count(U1Dev p, uint64_t *row_counts, unsigned long long *total) {
    const BT *basis = static_cast<const BT *>(p.basis);
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    unsigned long long mine = 0;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < p.dim; i += stride) {
        const uint64_t b = static_cast<uint64_t>(basis[i]);
        uint32_t c = 0;
        for (uint32_t g = 0; g < p.ngroups; ++g) {
            const uint64_t s = b ^ p.gx[g];
            if (static_cast<uint32_t>(__popcll(s)) != p.k) continue;
            const double2 v = group_value(p, g, s);
            if (v.x != 0.0 || v.y != 0.0) ++c;
        }
        if (row_counts) row_counts[i] = c;
        mine += c;
    }
    typedef cub::BlockReduce<unsigned long long, kU1Threads> Reduce;
    __shared__ typename Reduce::TempStorage tmp;
    const unsigned long long sum = Reduce(tmp).Sum(mine);
    if (threadIdx.x == 0 && sum) atomicAdd(total, sum);
}

// CSR fill: entries of row i at indptr[i] ..., in group order (sorted after).
template <typename BT, typename IT>
__global__ void k_u1_fill(U1Dev p, const uint64_t *indptr, uint64_t *cols, double2 *vals) {
    const BT *basis = static_cast<const BT *>(p.basis);
    const IT *tab = static_cast<const IT *>(p.tab);
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < p.dim; i += stride) {
        const uint64_t b = static_cast<uint64_t>(basis[i]);
        uint64_t pos = indptr[i];
        for (uint32_t g = 0; g < p.ngroups; ++g) {
            const uint64_t s = b ^ p.gx[g];
            if (static_cast<uint32_t>(__popcll(s)) != p.k) continue;
            const double2 v = group_value(p, g, s);
            if (v.x == 0.0 && v.y == 0.0) continue;
            cols[pos] = (s == b) ? i : rank_state<IT>(s, tab, p);
            vals[pos] = v;
            ++pos;
        }
    }
}

template <typename BT>
__global__ void k_u1_diag(U1Dev p, int32_t gzero, double2 *out) {
    const BT *basis = static_cast<const BT *>(p.basis);
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < p.dim; i += stride) {
        out[i] = gzero < 0 ? make_double2(0.0, 0.0) : group_value(p, static_cast<uint32_t>(gzero), basis[i]);
    }
}

template <int W> struct WState {
    uint64_t w[W];
};

template <int W> __device__ __forceinline__ WState<W> wload(const uint64_t *p, uint64_t i) {
    WState<W> s;
#pragma unroll
    for (int q = 0; q < W; ++q) s.w[q] = p[i * W + q];
    return s;
}
template <int W> __device__ __forceinline__ WState<W> wxor(const WState<W> &a, const uint64_t *m) {
    WState<W> s;
#pragma unroll
    for (int q = 0; q < W; ++q) s.w[q] = a.w[q] ^ m[q];
    return s;
}
template <int W> __device__ __forceinline__ uint32_t wpopc(const WState<W> &a) {
    uint32_t c = 0;
#pragma unroll
    for (int q = 0; q < W; ++q) c += static_cast<uint32_t>(__popcll(a.w[q]));
    return c;
}
template <int W> __device__ __forceinline__ uint32_t wparity_and(const WState<W> &a, const uint64_t *m) {
    uint32_t c = 0;
#pragma unroll
    for (int q = 0; q < W; ++q) c += static_cast<uint32_t>(__popcll(a.w[q] & m[q]));
    return c & 1u;
}
template <int W> __device__ __forceinline__ bool wequal(const WState<W> &a, const WState<W> &b) {
    bool e = true;
#pragma unroll
    for (int q = 0; q < W; ++q) e = e && a.w[q] == b.w[q];
    return e;
}

template <int W, typename IT>
__device__ uint64_t wrank(const WState<W> &s, const U1WDev &d) {
    const IT *tab = static_cast<const IT *>(d.tab);
    WState<W> a = s;
    if (d.comp) {
#pragma unroll
        for (int q = 0; q < W; ++q) a.w[q] = ~s.w[q];
        const uint32_t top = (d.n - 1) / 64;
        for (int q = 0; q < W; ++q) {
            if (q > static_cast<int>(top)) a.w[q] = 0;
        }
        a.w[top] &= d.tail;
    }
    uint64_t r = 0;
    uint32_t ones = 0;
    const uint32_t row = d.kp + 1;
    for (int c = static_cast<int>(d.nchunk) - 1; c >= 0; --c) {
        const uint32_t v = static_cast<uint32_t>(a.w[c / 8] >> (8 * (c % 8))) & 255u;
        r += static_cast<uint64_t>(tab[(static_cast<size_t>(c) * row + ones) * 256u + v]);
        ones += __popc(v);
    }
    return d.comp ? d.dim - 1 - r : r;
}

__device__ __forceinline__ double2 wgroup_value(const U1WDev &d, uint32_t g, const uint64_t *s, int W) {
    double re = 0, im = 0;
    for (uint32_t t = d.gt[g]; t < d.gt[g + 1]; ++t) {
        uint32_t par = 0;
        for (int q = 0; q < W; ++q) par += static_cast<uint32_t>(__popcll(d.tz[static_cast<size_t>(t) * W + q] & s[q]));
        const double2 w = d.tw[t];
        if (par & 1u) {
            re -= w.x;
            im -= w.y;
        } else {
            re += w.x;
            im += w.y;
        }
    }
    return make_double2(re, im);
}

// Basis: one thread per index, unranked from the top integer bit down.
template <int W>
__global__ void k_u1w_basis(U1WDev d, uint64_t *__restrict__ out) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= d.dim) return;
    uint64_t r = i, v[W] = {};
    uint32_t left = d.k;
    for (int e = static_cast<int>(d.n) - 1; e >= 0 && left; --e) {
        const uint64_t zero_count = d.choose[static_cast<uint32_t>(e) * 257u + left];  // C(e, left)
        if (r >= zero_count) {
            r -= zero_count;
            v[e / 64] |= 1ull << (e % 64);
            --left;
        }
    }
#pragma unroll
    for (int q = 0; q < W; ++q) out[i * W + q] = v[q];
}

template <typename R, int W, typename IT>
__global__ void k_u1w_apply(U1WDev d, const typename Cplx<R>::T *__restrict__ x, typename Cplx<R>::T *__restrict__ y,
                            uint64_t row0, uint64_t row1) {
    using C = typename Cplx<R>::T;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = row0 + static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < row1; i += stride) {
        const WState<W> b = wload<W>(d.basis, i);
        R ar = 0, ai = 0, cr = 0, ci = 0;
        for (uint32_t g = 0; g < d.ngroups; ++g) {
            const WState<W> s = wxor<W>(b, d.gx + static_cast<size_t>(g) * W);
            if (wpopc<W>(s) != d.k) continue;
            R vr = 0, vi = 0;
            for (uint32_t t = d.gt[g]; t < d.gt[g + 1]; ++t) {
                const C w = sizeof(R) == 8 ? reinterpret_cast<const C *>(d.tw)[t] : reinterpret_cast<const C *>(d.twf)[t];
                if (wparity_and<W>(s, d.tz + static_cast<size_t>(t) * W)) {
                    vr -= w.x;
                    vi -= w.y;
                } else {
                    vr += w.x;
                    vi += w.y;
                }
            }
            if (vr == R(0) && vi == R(0)) continue;
            const uint64_t j = wequal<W>(s, b) ? i : wrank<W, IT>(s, d);
            const C xv = x[j];
            const R pr = vr * xv.x - vi * xv.y, pi = vr * xv.y + vi * xv.x;
            if (sizeof(R) == 8) {
                ar += pr;
                ai += pi;
            } else {
                const R yr = pr - cr, yi = pi - ci;
                const R tr = ar + yr, ti = ai + yi;
                cr = (tr - ar) - yr;
                ci = (ti - ai) - yi;
                ar = tr;
                ai = ti;
            }
        }
        C out;
        out.x = ar;
        out.y = ai;
        y[i] = out;
    }
}

template <int W>
__global__ void k_u1w_leak(U1WDev d, unsigned long long *first) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < d.dim; i += stride) {
        const WState<W> b = wload<W>(d.basis, i);
        for (uint32_t g = 0; g < d.ngroups; ++g) {
            const WState<W> s = wxor<W>(b, d.gx + static_cast<size_t>(g) * W);
            if (wpopc<W>(s) == d.k) continue;
            const double2 v = wgroup_value(d, g, b.w, W);
            if (v.x != 0.0 || v.y != 0.0) {
                atomicMin(first, static_cast<unsigned long long>(i * d.ngroups + g));
                break;
            }
        }
    }
}

template <int W>
__global__ void k_u1w_count(U1WDev d, uint64_t *row_counts, unsigned long long *total) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    unsigned long long mine = 0;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < d.dim; i += stride) {
        const WState<W> b = wload<W>(d.basis, i);
        uint64_t c = 0;
        for (uint32_t g = 0; g < d.ngroups; ++g) {
            const WState<W> s = wxor<W>(b, d.gx + static_cast<size_t>(g) * W);
            if (wpopc<W>(s) != d.k) continue;
            const double2 v = wgroup_value(d, g, s.w, W);
            c += (v.x != 0.0 || v.y != 0.0);
        }
        if (row_counts) row_counts[i] = c;
        mine += c;
    }
    typedef cub::BlockReduce<unsigned long long, kU1Threads> Reduce;
    __shared__ typename Reduce::TempStorage tmp;
    const unsigned long long sum = Reduce(tmp).Sum(mine);
    if (threadIdx.x == 0 && sum) atomicAdd(total, sum);
}

template <int W, typename IT>
__global__ void k_u1w_fill(U1WDev d, const uint64_t *indptr, uint64_t *cols, double2 *vals) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < d.dim; i += stride) {
        const WState<W> b = wload<W>(d.basis, i);
        uint64_t pos = indptr[i];
        for (uint32_t g = 0; g < d.ngroups; ++g) {
            const WState<W> s = wxor<W>(b, d.gx + static_cast<size_t>(g) * W);
            if (wpopc<W>(s) != d.k) continue;
            const double2 v = wgroup_value(d, g, s.w, W);
            if (v.x == 0.0 && v.y == 0.0) continue;
            cols[pos] = wequal<W>(s, b) ? i : wrank<W, IT>(s, d);
            vals[pos] = v;
            ++pos;
        }
    }
}

template <int W>
__global__ void k_u1w_diag(U1WDev d, int32_t gzero, double2 *out) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < d.dim; i += stride) {
        const WState<W> b = wload<W>(d.basis, i);
        out[i] = gzero < 0 ? make_double2(0.0, 0.0) : wgroup_value(d, static_cast<uint32_t>(gzero), b.w, W);
    }
}

int g_sms = 0;

}  // namespace

// --------------------------------- the plan ---------------------------------
struct tcp_u1_plan {
    uint32_t n = 0, k = 0, kp = 0, comp = 0, nchunk = 0;
    uint64_t dim = 0, mask = 0;
    int storage = 0, device = 0;
    int64_t transitions = -1;
    uint64_t term_count = 0, estimated = 0;
    bool basis32 = true, index32 = true, smem = false;
    size_t tab_bytes = 0, smem_c128 = 0, smem_c64 = 0;
    U1Terms terms;
    uint32_t W = 1;  // 64-bit words per state (2 or 4 for n > 64)
    U1Dev dev{};
    U1Apply app{};
    U1WDev wdev{};
    void *block = nullptr;
    size_t block_bytes = 0;
    mutable std::mutex ws_mutex;
    mutable std::vector<std::pair<void *, size_t>> ws_free;
    mutable std::vector<void *> ws_all;
};

namespace {

int check_u1(const tcp_u1_plan *p) {
    if (p == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "plan is null");
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev != p->device) {
        return fail(TCP_ERR_WRONG_DEVICE, "plan lives on device " + std::to_string(p->device) +
                                              " but the current device is " + std::to_string(dev));
    }
    return TCP_OK;
}

int grid_for(uint64_t rows) {
    if (g_sms == 0) cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, 0);
    uint64_t want = (rows + kU1Threads - 1) / kU1Threads;
    uint64_t cap = static_cast<uint64_t>(std::max(g_sms, 1)) * 8;
    return static_cast<int>(std::max<uint64_t>(1, std::min(want, cap)));
}

// estimate_compiled_terms_bytes (sector.rs:1243-1292): retained size of a
// lazy plan, with the choose table of (n + 1) * (active + 1) entries.
uint64_t estimate_compiled(const tcp_u1_plan *p) {
    const U1Terms &t = p->terms;
    const uint64_t G = t.gx.size() / p->W, T = t.tz.size() / p->W, wc = word_count_of(p->n);
    unsigned __int128 b = 0;
    b += static_cast<unsigned __int128>(G) * wc * 8 + t.x_support * 8 + static_cast<unsigned __int128>(T) * wc * 8;
    b += static_cast<unsigned __int128>(T) * 16 + (T + 1) * 8 + t.z_support * 8 + G * 40;
    b += static_cast<unsigned __int128>(p->n + 1) * (p->kp + 1) * 8;
    return b >> 64 ? ~0ull : static_cast<uint64_t>(b);
}

// transition_upper_bound + estimate_plan_bytes (sector.rs:1176-1241).
int estimate_eager(const tcp_u1_plan *p, unsigned __int128 &bytes) {
    unsigned __int128 total = 0;
    for (size_t g = 0; g < p->terms.gx.size() / p->W; ++g) {
        uint32_t w = 0;
        for (uint32_t i = 0; i < p->W; ++i) w += static_cast<uint32_t>(__builtin_popcountll(p->terms.gx[g * p->W + i]));
        if (w % 2) continue;
        const uint32_t half = w / 2;
        if (half > p->k || half > p->n - p->k) continue;
        uint64_t left = 0, right = 0;
        if (!choose_u64(w, half, left) || !choose_u64(p->n - w, p->k - half, right)) {
            return fail(TCP_ERR_OVERFLOW, "integer overflow while estimating U1 transition candidates");
        }
        total += static_cast<unsigned __int128>(left) * right;
    }
    if (total >> 64) return fail(TCP_ERR_OVERFLOW, "integer overflow while converting U1 transition candidate count");
    const unsigned __int128 D = p->dim;
    bytes = estimate_compiled(p) + D * 8 + (D + 1) * 8 + D * 8 + total * 24;
    return TCP_OK;
}

std::string bytes_str(unsigned __int128 v) {
    return v >> 64 ? std::string("more than 2^64") : std::to_string(static_cast<uint64_t>(v));
}

template <typename R, typename ST, typename IT, int RK, bool SM, bool DIAG>
int launch_apply_v(const tcp_u1_plan *p, const void *x, void *y, cudaStream_t s, uint64_t row0, uint64_t row1) {
    using C = typename Cplx<R>::T;
    auto kern = k_u1_apply<R, ST, IT, RK, SM, DIAG>;
    int grid = grid_for(row1 - row0);
    size_t smem = 0;
    const size_t tab_bytes = RK ? p->app.ftab_bytes : p->tab_bytes;
    if (SM) {
        // one wave of resident CTAs: each CTA stages the tables once
        smem = sizeof(R) == 8 ? p->smem_c128 : p->smem_c64;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
        int per_sm = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kU1Threads, smem);
        if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        grid = std::min<int>(grid, std::max(per_sm, 1) * std::max(g_sms, 1));
    }
    kern<<<grid, kU1Threads, smem, s>>>(p->dev, p->app, tab_bytes, static_cast<const C *>(x), static_cast<C *>(y), row0,
                                        row1);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "sector MVP kernel launch");
}

template <typename R, typename ST, typename IT, int RK>
int launch_apply_t(const tcp_u1_plan *p, const void *x, void *y, cudaStream_t s, uint64_t r0, uint64_t r1) {
    const bool diag = p->app.diag != nullptr;
    if (p->smem) {
        return diag ? launch_apply_v<R, ST, IT, RK, true, true>(p, x, y, s, r0, r1)
                    : launch_apply_v<R, ST, IT, RK, true, false>(p, x, y, s, r0, r1);
    }
    return diag ? launch_apply_v<R, ST, IT, RK, false, true>(p, x, y, s, r0, r1)
                : launch_apply_v<R, ST, IT, RK, false, false>(p, x, y, s, r0, r1);
}

// Apply on `s` to output rows [row0, row1) (row1 = 0: all rows).
template <typename R, int W, typename IT>
int launch_apply_w(const tcp_u1_plan *p, const void *x, void *y, cudaStream_t s, uint64_t row0, uint64_t row1) {
    using C = typename Cplx<R>::T;
    k_u1w_apply<R, W, IT><<<grid_for(row1 - row0), kU1Threads, 0, s>>>(p->wdev, static_cast<const C *>(x),
                                                                          static_cast<C *>(y), row0, row1);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "wide sector MVP kernel launch");
}

template <typename R>
int launch_apply(const tcp_u1_plan *p, const void *x, void *y, cudaStream_t s, uint64_t row0 = 0, uint64_t row1 = 0) {
    if (p->dim == 0) return TCP_OK;
    if (row1 == 0) row1 = p->dim;
    if (p->W == 2) return p->index32 ? launch_apply_w<R, 2, uint32_t>(p, x, y, s, row0, row1)
                                     : launch_apply_w<R, 2, uint64_t>(p, x, y, s, row0, row1);
    if (p->W == 4) return p->index32 ? launch_apply_w<R, 4, uint32_t>(p, x, y, s, row0, row1)
                                     : launch_apply_w<R, 4, uint64_t>(p, x, y, s, row0, row1);
    if (p->basis32) {
        return p->app.rk == 2 ? launch_apply_t<R, uint32_t, uint32_t, 2>(p, x, y, s, row0, row1)
                              : launch_apply_t<R, uint32_t, uint32_t, 3>(p, x, y, s, row0, row1);
    }
    if (p->index32) return launch_apply_t<R, uint64_t, uint32_t, 0>(p, x, y, s, row0, row1);
    return launch_apply_t<R, uint64_t, uint64_t, 0>(p, x, y, s, row0, row1);
}

int count_transitions(const tcp_u1_plan *p, uint64_t *row_counts, uint64_t &total, cudaStream_t s) {
    unsigned long long *d_total = nullptr;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(&d_total), sizeof(unsigned long long), s);
    if (e != cudaSuccess) return cuda_fail(e, "allocating the transition counter");
    cudaMemsetAsync(d_total, 0, sizeof(unsigned long long), s);
    const int grid = grid_for(p->dim);
    if (p->W == 2) k_u1w_count<2><<<grid, kU1Threads, 0, s>>>(p->wdev, row_counts, d_total);
    else if (p->W == 4) k_u1w_count<4><<<grid, kU1Threads, 0, s>>>(p->wdev, row_counts, d_total);
    else if (p->basis32) k_u1_count<uint32_t><<<grid, kU1Threads, 0, s>>>(p->dev, row_counts, d_total);
    else k_u1_count<uint64_t><<<grid, kU1Threads, 0, s>>>(p->dev, row_counts, d_total);
    unsigned long long h = 0;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d_total, sizeof(h), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(d_total, s);
    cudaError_t e2 = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "counting sector transitions");
    if (e2 != cudaSuccess) return cuda_fail(e2, "counting sector transitions");
    total = h;
    return TCP_OK;
}

int scan_leakage(const tcp_u1_plan *p) {
    unsigned long long *d_first = nullptr;
    cudaError_t e = cudaMalloc(reinterpret_cast<void **>(&d_first), sizeof(unsigned long long));
    if (e != cudaSuccess) return cuda_fail(e, "allocating the leakage flag");
    cudaMemset(d_first, 0xff, sizeof(unsigned long long));
    const int grid = grid_for(p->dim);
    if (p->W == 2) k_u1w_leak<2><<<grid, kU1Threads>>>(p->wdev, d_first);
    else if (p->W == 4) k_u1w_leak<4><<<grid, kU1Threads>>>(p->wdev, d_first);
    else if (p->basis32) k_u1_leak<uint32_t><<<grid, kU1Threads>>>(p->dev, d_first);
    else k_u1_leak<uint64_t><<<grid, kU1Threads>>>(p->dev, d_first);
    unsigned long long first = 0;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(&first, d_first, sizeof(first), cudaMemcpyDeviceToHost);
    cudaFree(d_first);
    if (e != cudaSuccess) return cuda_fail(e, "scanning for sector leakage");
    if (first == ~0ull) return TCP_OK;
    const uint64_t G = p->terms.gx.size() / p->W;
    const uint64_t source = first / G, g = first % G;
    std::vector<uint64_t> words(std::max<uint32_t>(word_count_of(p->n), 1), 0), b(p->W, 0);
    unrank_packed(p->n, p->k, p->dim, source, words.data(), word_count_of(p->n));
    for (uint32_t q = 0; q < p->n; ++q)  // packed qubit words -> integer bits
        if ((words[q / 64] >> (q % 64)) & 1) b[(p->n - 1 - q) / 64] |= 1ull << ((p->n - 1 - q) % 64);
    uint32_t actual = 0;
    for (uint32_t i = 0; i < p->W; ++i) actual += static_cast<uint32_t>(__builtin_popcountll(b[i] ^ p->terms.gx[g * p->W + i]));
    return tcp::fail_fields(TCP_ERR_SECTOR_LEAKAGE, leak_message(source, p->k, actual), source, actual);
}

// One device allocation: choose table, rank tables, groups, terms, basis.
int upload(tcp_u1_plan *p) {
    const U1Terms &t = p->terms;
    const uint32_t G = static_cast<uint32_t>(t.gx.size()), T = static_cast<uint32_t>(t.tz.size());
    // host tables
    std::vector<uint64_t> choose(65 * 65, 0);
    for (uint32_t a = 0; a <= 64; ++a)
        for (uint32_t b = 0; b <= 64; ++b) choose_u64(a, b, choose[a * 65 + b]);
    const uint32_t row = p->kp + 1;
    const size_t entries = static_cast<size_t>(p->nchunk) * row * 256;
    std::vector<uint64_t> tab(entries, 0);
    for (uint32_t c = 0; c < p->nchunk; ++c) {
        const uint32_t below = 8 * c;
        for (uint32_t a = 0; a < row; ++a) {
            uint64_t acc = 0;
            for (uint32_t v = 0; v < 256; ++v) {
                tab[(static_cast<size_t>(c) * row + a) * 256 + v] = acc;
                const int need = static_cast<int>(p->kp) - static_cast<int>(a) - __builtin_popcount(v);
                if (need >= 0 && static_cast<uint32_t>(need) <= below) acc += choose[below * 65 + need];
            }
        }
    }
    const size_t isz = p->index32 ? 4 : 8, bsz = p->basis32 ? 4 : 8;
    p->tab_bytes = entries * isz;
    struct Piece {
        const void *src;
        size_t bytes;
        size_t off;
    };
    std::vector<uint32_t> tab32;
    if (p->index32) tab32.assign(tab.begin(), tab.end());
    std::vector<float> twf(2 * static_cast<size_t>(T));
    for (size_t i = 0; i < twf.size(); ++i) twf[i] = static_cast<float>(t.tw[i]);
    // apply view: groups with x != 0 and an even number of flips, in three
    // segments (constant, constant with z_out, general); see U1Apply
    const size_t ssz = p->basis32 ? 4 : 8;
    struct SegGroup {
        uint64_t x, zout;
        uint32_t half, tb, te;
        double cr, ci;
    };
    std::vector<SegGroup> segA, segB, segC;
    for (uint32_t g = 0; g < G; ++g) {
        const uint64_t x = t.gx[g];
        const uint32_t w = static_cast<uint32_t>(__builtin_popcountll(x));
        if (x == 0 || (w & 1)) continue;
        const uint32_t tb = t.gt[g], te = t.gt[g + 1];
        bool constant = true;
        const uint64_t zout = t.tz[tb] & ~x;
        for (uint32_t q = tb; q < te && constant; ++q) {
            const uint64_t zin = t.tz[q] & x;
            constant = (zin == 0 || zin == x) && (t.tz[q] & ~x) == zout;
        }
        SegGroup sg{x, zout, w / 2, tb, te, 0.0, 0.0};
        if (!constant) {
            segC.push_back(sg);
            continue;
        }
        // the value where popcount(z_out & b) is even, summed from 0 in
        // canonical term order as aggregate_source sums it
        for (uint32_t q = tb; q < te; ++q) {
            if (((t.tz[q] & x) == x) && ((w / 2) & 1)) {
                sg.cr -= t.tw[2 * q];
                sg.ci -= t.tw[2 * q + 1];
            } else {
                sg.cr += t.tw[2 * q];
                sg.ci += t.tw[2 * q + 1];
            }
        }
        if (sg.cr == 0.0 && sg.ci == 0.0) continue;  // never contributes
        (zout ? segB : segA).push_back(sg);
    }
    auto pad = [](std::vector<SegGroup> &v) {
        while (v.size() % kU1Unroll) v.push_back(SegGroup{0, 0, 1, 0, 0, 0.0, 0.0});  // never live
    };
    pad(segA);
    pad(segB);
    pad(segC);
    std::vector<unsigned char> grec, azo, az;
    std::vector<double> ac, aw;
    std::vector<float> acf, awf;
    std::vector<uint32_t> at(1, 0);
    auto put = [&](std::vector<unsigned char> &v, uint64_t m) {
        const size_t o = v.size();
        v.resize(o + ssz);
        if (ssz == 4) {
            const uint32_t m32 = static_cast<uint32_t>(m);
            std::memcpy(v.data() + o, &m32, 4);
        } else {
            std::memcpy(v.data() + o, &m, 8);
        }
    };
    auto put_rec = [&](const SegGroup &sg) {
        put(grec, sg.x);
        const uint32_t half_pad[2] = {sg.half, 0};
        const size_t o = grec.size();
        grec.resize(o + ssz);  // half (and padding for 64-bit records)
        std::memcpy(grec.data() + o, half_pad, ssz);
    };
    for (auto *seg : {&segA, &segB}) {
        for (const SegGroup &sg : *seg) {
            put_rec(sg);
            ac.push_back(sg.cr);
            ac.push_back(sg.ci);
            acf.push_back(static_cast<float>(sg.cr));
            acf.push_back(static_cast<float>(sg.ci));
        }
    }
    for (const SegGroup &sg : segB) put(azo, sg.zout);
    for (const SegGroup &sg : segC) {
        put_rec(sg);
        for (uint32_t q = sg.tb; q < sg.te; ++q) {
            put(az, t.tz[q]);
            aw.push_back(t.tw[2 * q]);
            aw.push_back(t.tw[2 * q + 1]);
            awf.push_back(twf[2 * q]);
            awf.push_back(twf[2 * q + 1]);
        }
        at.push_back(static_cast<uint32_t>(aw.size() / 2));
    }
    const uint32_t NA = static_cast<uint32_t>(segA.size()), NB = static_cast<uint32_t>(segB.size()),
                   NC = static_cast<uint32_t>(segC.size()), TA = at.back();
    const bool has_diag = t.gzero >= 0;
    // fast rank tables (n <= 32): two levels up to 24 qubits, else three
    std::vector<uint32_t> ftab;
    U1Apply fast{};
    if (p->basis32) {
        const uint32_t n = p->n, k = p->k;
        uint32_t T_ = 0, M_ = 0, L_ = 0;
        if (n <= 24) {
            L_ = n / 2;
            T_ = n - L_;
        } else {
            size_t best = ~size_t(0);
            for (uint32_t a = 1; a + 2 <= n; ++a)
                for (uint32_t b = 1; a + b + 1 <= n; ++b) {
                    const uint32_t c = n - a - b;
                    const size_t e = (size_t(1) << a) + (std::min(k, a) + 1) * (size_t(1) << b) + (size_t(1) << c);
                    if (e < best) {
                        best = e;
                        T_ = a;
                        M_ = b;
                        L_ = c;
                    }
                }
        }
        const uint32_t lowbits = M_ + L_;  // bits below the top part
        std::vector<uint32_t> H(size_t(1) << T_), Lr(size_t(1) << L_), Mid;
        {
            std::vector<uint32_t> seen(L_ + 1, 0);
            for (uint32_t v = 0; v < (1u << L_); ++v) Lr[v] = seen[__builtin_popcount(v)]++;
            uint64_t acc = 0;
            for (uint32_t h = 0; h < (1u << T_); ++h) {
                H[h] = static_cast<uint32_t>(acc);
                const int need = static_cast<int>(k) - __builtin_popcount(h);
                if (need >= 0 && static_cast<uint32_t>(need) <= lowbits) acc += choose[lowbits * 65 + need];
            }
        }
        if (M_) {
            const uint32_t rows = std::min(k, T_) + 1;
            Mid.assign(size_t(rows) << M_, 0);
            for (uint32_t a = 0; a < rows; ++a) {
                uint64_t acc = 0;
                for (uint32_t v = 0; v < (1u << M_); ++v) {
                    Mid[(size_t(a) << M_) + v] = static_cast<uint32_t>(acc);
                    const int need = static_cast<int>(k) - static_cast<int>(a) - __builtin_popcount(v);
                    if (need >= 0 && static_cast<uint32_t>(need) <= L_) acc += choose[L_ * 65 + need];
                }
            }
        }
        fast.rk = M_ ? 3 : 2;
        fast.rL = L_;
        fast.rM = M_;
        fast.lmask = L_ ? ((1u << L_) - 1) : 0u;
        fast.mmask = M_ ? ((1u << M_) - 1) : 0u;
        fast.h_off = 0;
        fast.m_off = static_cast<uint32_t>(H.size());
        fast.l_off = static_cast<uint32_t>(H.size() + Mid.size());
        ftab.insert(ftab.end(), H.begin(), H.end());
        ftab.insert(ftab.end(), Mid.begin(), Mid.end());
        ftab.insert(ftab.end(), Lr.begin(), Lr.end());
        fast.ftab_bytes = 4 * ftab.size();
    }
    Piece pieces[] = {
        {choose.data(), choose.size() * 8, 0},
        {p->index32 ? static_cast<const void *>(tab32.data()) : tab.data(), p->tab_bytes, 0},
        {t.gx.data(), 8ull * G, 0},
        {t.gt.data(), 4ull * (G + 1), 0},
        {t.tz.data(), 8ull * T, 0},
        {t.tw.data(), 16ull * T, 0},
        {twf.data(), 8ull * T, 0},
        {nullptr, bsz * p->dim, 0},  // basis, generated on the device
        {grec.data(), grec.size(), 0},
        {nullptr, 0, 0},
        {azo.data(), azo.size(), 0},
        {ac.data(), 8ull * ac.size(), 0},
        {acf.data(), 4ull * acf.size(), 0},
        {at.data(), 4ull * at.size(), 0},
        {az.data(), az.size(), 0},
        {aw.data(), 8ull * aw.size(), 0},
        {awf.data(), 4ull * awf.size(), 0},
        {nullptr, has_diag ? 16 * p->dim : 0, 0},  // diagonal, evaluated on the device
        {ftab.data(), 4ull * ftab.size(), 0},
    };
    size_t off = 0;
    for (auto &pc : pieces) {
        pc.off = off;
        off += (pc.bytes + 255) / 256 * 256;
    }
    void *block = nullptr;
    cudaError_t e = tcp::injected_alloc_failure() ? cudaErrorMemoryAllocation : cudaMalloc(&block, std::max<size_t>(off, 256));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(TCP_ERR_ALLOCATION, "device allocation of the sector plan (" + std::to_string(off) + " bytes) failed");
    }
    unsigned char *base = static_cast<unsigned char *>(block);
    for (auto &pc : pieces) {
        if (pc.src && pc.bytes) {
            e = cudaMemcpy(base + pc.off, pc.src, pc.bytes, cudaMemcpyHostToDevice);
            if (e != cudaSuccess) {
                cudaFree(block);
                return cuda_fail(e, "uploading the sector plan");
            }
        }
    }
    p->block = block;
    p->block_bytes = off;
    U1Dev &d = p->dev;
    d.choose = reinterpret_cast<const uint64_t *>(base + pieces[0].off);
    d.tab = base + pieces[1].off;
    d.gx = reinterpret_cast<const uint64_t *>(base + pieces[2].off);
    d.gt = reinterpret_cast<const uint32_t *>(base + pieces[3].off);
    d.tz = reinterpret_cast<const uint64_t *>(base + pieces[4].off);
    d.tw = reinterpret_cast<const double2 *>(base + pieces[5].off);
    d.twf = reinterpret_cast<const float2 *>(base + pieces[6].off);
    d.basis = base + pieces[7].off;
    d.dim = p->dim;
    d.mask = p->mask;
    d.n = p->n;
    d.k = p->k;
    d.kp = p->kp;
    d.comp = p->comp;
    d.nchunk = p->nchunk;
    d.ngroups = G;
    d.nterms = T;
    U1Apply &ap = p->app;
    ap = fast;
    ap.grec = base + pieces[8].off;
    ap.azo = base + pieces[10].off;
    ap.ac = reinterpret_cast<const double2 *>(base + pieces[11].off);
    ap.acf = reinterpret_cast<const float2 *>(base + pieces[12].off);
    ap.at = reinterpret_cast<const uint32_t *>(base + pieces[13].off);
    ap.az = base + pieces[14].off;
    ap.aw = reinterpret_cast<const double2 *>(base + pieces[15].off);
    ap.awf = reinterpret_cast<const float2 *>(base + pieces[16].off);
    ap.diag = has_diag ? reinterpret_cast<const double2 *>(base + pieces[17].off) : nullptr;
    ap.ftab = p->basis32 ? reinterpret_cast<const uint32_t *>(base + pieces[18].off) : nullptr;
    ap.na = NA;
    ap.nb = NB;
    ap.nc = NC;
    ap.ta = TA;
    // basis generation
    const uint32_t rows_per_thread = 64;
    const uint64_t threads = (p->dim + rows_per_thread - 1) / rows_per_thread;
    const unsigned blocks = static_cast<unsigned>((threads + kU1Threads - 1) / kU1Threads);
    if (p->basis32) k_u1_basis<uint32_t><<<blocks, kU1Threads>>>(d, rows_per_thread, static_cast<uint32_t *>(const_cast<void *>(d.basis)));
    else k_u1_basis<uint64_t><<<blocks, kU1Threads>>>(d, rows_per_thread, static_cast<uint64_t *>(const_cast<void *>(d.basis)));
    e = cudaGetLastError();
    if (e == cudaSuccess && has_diag) {
        const int grid = grid_for(p->dim);
        double2 *diag = reinterpret_cast<double2 *>(base + pieces[17].off);
        if (p->basis32) k_u1_diag<uint32_t><<<grid, kU1Threads>>>(d, t.gzero, diag);
        else k_u1_diag<uint64_t><<<grid, kU1Threads>>>(d, t.gzero, diag);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        cudaFree(block);
        p->block = nullptr;
        return cuda_fail(e, "generating the sector basis and diagonal");
    }
    // shared-memory staging of the apply view
    const size_t apply_tab = p->basis32 ? ap.ftab_bytes : p->tab_bytes;
    p->smem_c128 = u1_apply_layout(apply_tab, NA, NB, NC, TA, ssz, 16).total;
    p->smem_c64 = u1_apply_layout(apply_tab, NA, NB, NC, TA, ssz, 8).total;
    p->smem = p->smem_c128 <= kU1SmemMax;
    return TCP_OK;
}

// Wide plans: one allocation with the saturated C(e, j) table, the 8-bit
// chunk rank tables, groups, terms and the basis (unranked on the device).
int upload_wide(tcp_u1_plan *p) {
    const U1Terms &t = p->terms;
    const uint32_t W = p->W;
    const uint32_t G = static_cast<uint32_t>(t.gx.size() / W), T = static_cast<uint32_t>(t.tz.size() / W);
    std::vector<uint64_t> choose(256 * 257, 0);
    for (uint32_t a = 0; a < 256; ++a)
        for (uint32_t b = 0; b <= 256; ++b) {
            uint64_t c = 0;
            choose[a * 257 + b] = choose_u64(a, b, c) ? c : ~0ull;
        }
    const uint32_t row = p->kp + 1;
    const size_t entries = static_cast<size_t>(p->nchunk) * row * 256;
    std::vector<uint64_t> tab(entries, 0);
    for (uint32_t c = 0; c < p->nchunk; ++c) {
        const uint32_t below = 8 * c;
        for (uint32_t a = 0; a < row; ++a) {
            uint64_t acc = 0;
            for (uint32_t v = 0; v < 256; ++v) {
                tab[(static_cast<size_t>(c) * row + a) * 256 + v] = acc;
                const int need = static_cast<int>(p->kp) - static_cast<int>(a) - __builtin_popcount(v);
                if (need >= 0 && static_cast<uint32_t>(need) <= below) {
                    uint64_t cnt = 0;
                    if (!choose_u64(below, static_cast<uint64_t>(need), cnt) || acc + cnt < acc) acc = ~0ull;
                    else acc += cnt;
                }
            }
        }
    }
    std::vector<uint32_t> tab32;
    if (p->index32) tab32.assign(tab.begin(), tab.end());
    std::vector<float> twf(2 * static_cast<size_t>(T));
    for (size_t i = 0; i < twf.size(); ++i) twf[i] = static_cast<float>(t.tw[i]);
    struct Piece {
        const void *src;
        size_t bytes;
        size_t off;
    };
    Piece pieces[] = {
        {choose.data(), choose.size() * 8, 0},
        {p->index32 ? static_cast<const void *>(tab32.data()) : tab.data(), entries * (p->index32 ? 4 : 8), 0},
        {t.gx.data(), 8ull * t.gx.size(), 0},
        {t.gt.data(), 4ull * (G + 1), 0},
        {t.tz.data(), 8ull * t.tz.size(), 0},
        {t.tw.data(), 16ull * T, 0},
        {twf.data(), 8ull * T, 0},
        {nullptr, 8ull * W * p->dim, 0},  // basis, generated on the device
    };
    size_t off = 0;
    for (auto &pc : pieces) {
        pc.off = off;
        off += (pc.bytes + 255) / 256 * 256;
    }
    void *block = nullptr;
    cudaError_t e = tcp::injected_alloc_failure() ? cudaErrorMemoryAllocation : cudaMalloc(&block, std::max<size_t>(off, 256));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(TCP_ERR_ALLOCATION, "device allocation of the sector plan (" + std::to_string(off) + " bytes) failed");
    }
    unsigned char *base = static_cast<unsigned char *>(block);
    for (auto &pc : pieces) {
        if (pc.src && pc.bytes) {
            e = cudaMemcpy(base + pc.off, pc.src, pc.bytes, cudaMemcpyHostToDevice);
            if (e != cudaSuccess) {
                cudaFree(block);
                return cuda_fail(e, "uploading the sector plan");
            }
        }
    }
    p->block = block;
    p->block_bytes = off;
    p->tab_bytes = entries * (p->index32 ? 4 : 8);
    U1WDev &d = p->wdev;
    d.choose = reinterpret_cast<const uint64_t *>(base + pieces[0].off);
    d.tab = base + pieces[1].off;
    d.gx = reinterpret_cast<const uint64_t *>(base + pieces[2].off);
    d.gt = reinterpret_cast<const uint32_t *>(base + pieces[3].off);
    d.tz = reinterpret_cast<const uint64_t *>(base + pieces[4].off);
    d.tw = reinterpret_cast<const double2 *>(base + pieces[5].off);
    d.twf = reinterpret_cast<const float2 *>(base + pieces[6].off);
    d.basis = reinterpret_cast<const uint64_t *>(base + pieces[7].off);
    d.dim = p->dim;
    d.tail = (p->n % 64) ? ((1ull << (p->n % 64)) - 1) : ~0ull;
    d.n = p->n;
    d.k = p->k;
    d.kp = p->kp;
    d.comp = p->comp;
    d.nchunk = p->nchunk;
    d.ngroups = G;
    d.nterms = T;
    const unsigned blocks = static_cast<unsigned>((p->dim + kU1Threads - 1) / kU1Threads);
    uint64_t *basis = reinterpret_cast<uint64_t *>(base + pieces[7].off);
    if (W == 2) k_u1w_basis<2><<<blocks, kU1Threads>>>(d, basis);
    else k_u1w_basis<4><<<blocks, kU1Threads>>>(d, basis);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        cudaFree(block);
        p->block = nullptr;
        return cuda_fail(e, "generating the wide sector basis");
    }
    p->smem = false;
    return TCP_OK;
}

template <typename R>
int apply_host(const tcp_u1_plan *plan, const R *state, uint64_t state_len, R *result, uint64_t result_len) {
    int st = check_u1(plan);
    if (st) return st;
    if (state_len != plan->dim) return tcp::length_error(plan->dim, state_len);
    if (result_len != plan->dim) return tcp::length_error(plan->dim, result_len);
    if (state == nullptr || result == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    const size_t bytes = plan->dim * 2 * sizeof(R);
    auto pa = reinterpret_cast<uintptr_t>(state), pb = reinterpret_cast<uintptr_t>(result);
    if (pa < pb + bytes && pb < pa + bytes) return fail(TCP_ERR_INVALID_ARGUMENT, "input and output must not overlap");
    void *ws = nullptr;
    {
        std::lock_guard<std::mutex> lock(plan->ws_mutex);
        for (size_t i = 0; i < plan->ws_free.size(); ++i) {
            if (plan->ws_free[i].second >= 2 * bytes) {
                ws = plan->ws_free[i].first;
                plan->ws_free.erase(plan->ws_free.begin() + static_cast<long>(i));
                break;
            }
        }
    }
    if (ws == nullptr) {
        cudaError_t e = tcp::injected_alloc_failure() ? cudaErrorMemoryAllocation : cudaMalloc(&ws, 2 * bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(TCP_ERR_ALLOCATION, "device allocation of the sector apply workspace failed");
        }
        std::lock_guard<std::mutex> lock(plan->ws_mutex);
        plan->ws_all.push_back(ws);
    }
    void *dx = ws, *dy = static_cast<unsigned char *>(ws) + bytes;
    cudaStream_t stream = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
    int status = e == cudaSuccess ? TCP_OK : cuda_fail(e, "cudaStreamCreate");
    if (!status && bytes) {
        e = cudaMemcpyAsync(dx, state, bytes, cudaMemcpyHostToDevice, stream);
        if (e != cudaSuccess) status = cuda_fail(e, "H2D copy");
    }
    // Large applies run in kSectorChunks row ranges; a second stream copies
    // each finished range of y to the host while the next one computes.  All
    // launches and copies are queued before the host waits on any of them.
    constexpr uint64_t kSectorChunks = 8;
    const uint64_t chunks = plan->dim >= (1ull << 22) ? kSectorChunks : 1;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t done[kSectorChunks] = {};
    if (!status && chunks > 1) {
        e = cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking);
        for (uint64_t c = 0; c < chunks && e == cudaSuccess; ++c) e = cudaEventCreateWithFlags(&done[c], cudaEventDisableTiming);
        if (e != cudaSuccess) status = cuda_fail(e, "creating the copy stream");
        const uint64_t per = plan->dim / chunks;
        for (uint64_t c = 0; c < chunks && !status; ++c) {
            const uint64_t r0 = c * per, r1 = (c + 1 == chunks) ? plan->dim : r0 + per;
            status = launch_apply<R>(plan, dx, dy, stream, r0, r1);
            if (!status) {
                e = cudaEventRecord(done[c], stream);
                if (e != cudaSuccess) status = cuda_fail(e, "chunk event");
            }
        }
        for (uint64_t c = 0; c < chunks && !status; ++c) {
            const uint64_t r0 = c * per, r1 = (c + 1 == chunks) ? plan->dim : r0 + per;
            const size_t off = r0 * 2 * sizeof(R), len = (r1 - r0) * 2 * sizeof(R);
            e = cudaStreamWaitEvent(copy_stream, done[c], 0);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(reinterpret_cast<unsigned char *>(result) + off,
                                    static_cast<const unsigned char *>(dy) + off, len, cudaMemcpyDeviceToHost,
                                    copy_stream);
            if (e != cudaSuccess) status = cuda_fail(e, "D2H copy");
        }
    } else if (!status) {
        status = launch_apply<R>(plan, dx, dy, stream);
        if (!status && bytes) {
            e = cudaMemcpyAsync(result, dy, bytes, cudaMemcpyDeviceToHost, stream);
            if (e != cudaSuccess) status = cuda_fail(e, "D2H copy");
        }
    }
    if (copy_stream) {
        e = cudaStreamSynchronize(copy_stream);
        if (!status && e != cudaSuccess) status = cuda_fail(e, "copy stream synchronize");
        cudaStreamDestroy(copy_stream);
    }
    for (auto &ev : done)
        if (ev) cudaEventDestroy(ev);
    if (stream) {
        e = cudaStreamSynchronize(stream);
        if (!status && e != cudaSuccess) status = cuda_fail(e, "stream synchronize");
        cudaStreamDestroy(stream);
    }
    {
        std::lock_guard<std::mutex> lock(plan->ws_mutex);
        plan->ws_free.emplace_back(ws, 2 * bytes);
    }
    return status;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" int tcp_u1_dimension(uint32_t nqubits, uint32_t particle_number, uint64_t *out_dimension) {
    if (out_dimension == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "null output");
    return sector_dimension(nqubits, particle_number, *out_dimension);
}

extern "C" int tcp_u1_rank_words(uint32_t nqubits, uint32_t particle_number, const uint64_t *words,
                                 uint32_t word_count, uint64_t *out_rank) {
    if (out_rank == nullptr || (word_count && words == nullptr)) return fail(TCP_ERR_INVALID_ARGUMENT, "null argument");
    uint64_t dim = 0;
    int st = sector_dimension(nqubits, particle_number, dim);
    if (st) return st;
    return rank_packed(nqubits, particle_number, words, word_count, *out_rank);
}

extern "C" int tcp_u1_unrank_words(uint32_t nqubits, uint32_t particle_number, uint64_t index, uint64_t *out_words,
                                   uint32_t word_count) {
    if (word_count && out_words == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "null output");
    uint64_t dim = 0;
    int st = sector_dimension(nqubits, particle_number, dim);
    if (st) return st;
    return unrank_packed(nqubits, particle_number, dim, index, out_words, word_count);
}

extern "C" int tcp_u1_basis_words(uint32_t nqubits, uint32_t particle_number, uint64_t *out, uint64_t capacity,
                                  uint64_t max_bytes) {
    uint64_t dim = 0;
    int st = sector_dimension(nqubits, particle_number, dim);
    if (st) return st;
    const uint32_t wc = nqubits <= 64 ? 1 : word_count_of(nqubits);
    const unsigned __int128 count = static_cast<unsigned __int128>(dim) * wc;
    const unsigned __int128 bytes = count * 8;
    if (bytes > max_bytes)
        return tcp::fail_fields(TCP_ERR_MEMORY_LIMIT,
                                "requested " + bytes_str(bytes) + " bytes exceeds memory limit " + std::to_string(max_bytes),
                                tcp::clamp_u64(bytes), max_bytes);
    if (count > capacity) return fail(TCP_ERR_INVALID_ARGUMENT, "basis output buffer is too small");
    if (dim && out == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "null output");
    const uint32_t pw = word_count_of(nqubits);
    std::vector<uint64_t> words(std::max<uint32_t>(pw, 1));
    for (uint64_t i = 0; i < dim; ++i) {
        st = unrank_packed(nqubits, particle_number, dim, i, words.data(), pw);
        if (st) return st;
        if (nqubits <= 64) {
            uint64_t v = 0;  // TensorCircuit integer
            for (uint32_t q = 0; q < nqubits; ++q)
                if ((words[0] >> q) & 1) v |= 1ull << (nqubits - 1 - q);
            out[i] = v;
        } else {
            std::memcpy(out + i * wc, words.data(), 8ull * wc);
        }
    }
    return TCP_OK;
}

extern "C" int tcp_pauli_number_commutator(uint32_t nqubits, uint64_t term_count, uint32_t word_count,
                                           const uint64_t *x_words, const uint64_t *z_words,
                                           const double *coefficients, uint64_t *out_nonzero) {
    // analyze_charge (operator.rs:396-444) with levels (0, 1): difference
    // l0 - l1 = -1.  Every X (Y) factor on qubit q contributes the word with
    // that factor swapped to Y (X), weighted by coefficient * (0 + i*scale),
    // scale = -difference for X and +difference for Y.  Contributions to one
    // word are summed from 0 in ascending (re bits, im bits) order; the
    // operator conserves the number iff every sum is exactly zero.
    if (out_nonzero == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "null output");
    const uint32_t wc = word_count_of(nqubits);
    if (word_count != wc) {
        return tcp::fail_fields(TCP_ERR_INVALID_WORD_LENGTH,
                                "expected " + std::to_string(wc) + " packed words, got " + std::to_string(word_count), wc,
                                word_count);
    }
    if (term_count && (x_words == nullptr || z_words == nullptr || coefficients == nullptr)) {
        return fail(TCP_ERR_INVALID_ARGUMENT, "null term arrays");
    }
    std::map<std::vector<uint64_t>, std::vector<std::pair<double, double>>> aggregate;
    const double difference = 0.0 - 1.0;
    for (uint64_t t = 0; t < term_count; ++t) {
        const double are = coefficients[2 * t], aim = coefficients[2 * t + 1];
        for (uint32_t q = 0; q < nqubits; ++q) {
            const uint64_t bit = 1ull << (q % 64);
            const bool x = x_words[t * wc + q / 64] & bit, z = z_words[t * wc + q / 64] & bit;
            if (!x) continue;  // I or Z
            const double scale = z ? difference : -difference;  // Y : X
            std::vector<uint64_t> key(2 * wc);
            for (uint32_t w = 0; w < wc; ++w) {
                key[w] = x_words[t * wc + w];
                key[wc + w] = z_words[t * wc + w];
            }
            key[wc + q / 64] ^= bit;  // X <-> Y
            // (are + i aim) * (0 + i scale), textbook product
            const double re = are * 0.0 - aim * scale;
            const double im = are * scale + aim * 0.0;
            aggregate[key].emplace_back(re, im);
        }
    }
    uint64_t nonzero = 0;
    for (auto &kv : aggregate) {
        auto &vals = kv.second;
        std::sort(vals.begin(), vals.end(), [](const std::pair<double, double> &a, const std::pair<double, double> &b) {
            uint64_t ar, ai, br, bi;
            std::memcpy(&ar, &a.first, 8);
            std::memcpy(&ai, &a.second, 8);
            std::memcpy(&br, &b.first, 8);
            std::memcpy(&bi, &b.second, 8);
            return ar != br ? ar < br : ai < bi;
        });
        double sr = 0.0, si = 0.0;
        for (auto &v : vals) {
            sr = sr + v.first;
            si = si + v.second;
        }
        if (sr != 0.0 || si != 0.0) ++nonzero;
    }
    *out_nonzero = nonzero;
    return TCP_OK;
}

extern "C" int tcp_u1_plan_create(uint32_t nqubits, uint32_t particle_number, uint64_t term_count,
                                  uint32_t word_count, const uint64_t *x_words, const uint64_t *z_words,
                                  const double *coefficients, int storage, uint64_t max_bytes,
                                  tcp_u1_plan **out_plan) {
    tcp::Range range("tcp_u1_plan_create");
    if (out_plan == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "out_plan is null");
    *out_plan = nullptr;
    if (storage != TCP_STORAGE_LAZY && storage != TCP_STORAGE_EAGER) {
        return fail(TCP_ERR_INVALID_SECTOR, "invalid sector: storage must be either 'eager' or 'lazy'");
    }
    if (term_count > 0 && (x_words == nullptr || z_words == nullptr || coefficients == nullptr)) {
        return fail(TCP_ERR_INVALID_ARGUMENT, "null term arrays");
    }
    if (term_count > 0xffffffffull) return fail(TCP_ERR_OVERFLOW, "integer overflow while counting plan terms");
    std::unique_ptr<tcp_u1_plan> p(new tcp_u1_plan());
    int st = sector_dimension(nqubits, particle_number, p->dim);
    if (st) return st;
    if (nqubits > 256) {
        return fail(TCP_ERR_OVERFLOW, "integer overflow while representing a sector state: the device sector plan "
                                      "supports at most 256 qubits");
    }
    p->W = nqubits <= 64 ? 1 : (nqubits <= 128 ? 2 : 4);
    st = compile_u1(nqubits, term_count, word_count, x_words, z_words, coefficients, p->W, p->terms);
    if (st) return st;
    p->n = nqubits;
    p->k = particle_number;
    p->kp = std::min(particle_number, nqubits - particle_number);
    p->comp = particle_number > nqubits - particle_number ? 1 : 0;
    p->nchunk = (nqubits + 7) / 8;
    p->mask = nqubits >= 64 ? ~0ull : ((1ull << nqubits) - 1);
    p->storage = storage;
    p->term_count = term_count;
    p->basis32 = nqubits <= 32;
    p->index32 = p->dim <= 0xffffffffull;
    if (storage == TCP_STORAGE_LAZY) {
        p->estimated = estimate_compiled(p.get());
        if (p->estimated > max_bytes) {
            return tcp::fail_fields(TCP_ERR_MEMORY_LIMIT,
                                    "requested " + std::to_string(p->estimated) + " bytes exceeds memory limit " +
                                        std::to_string(max_bytes),
                                    p->estimated, max_bytes);
        }
    } else {
        unsigned __int128 bytes = 0;
        st = estimate_eager(p.get(), bytes);
        if (st) return st;
        if (bytes > max_bytes) {
            return tcp::fail_fields(TCP_ERR_MEMORY_LIMIT,
                                    "requested " + bytes_str(bytes) + " bytes exceeds memory limit " +
                                        std::to_string(max_bytes),
                                    tcp::clamp_u64(bytes), max_bytes);
        }
        p->estimated = estimate_compiled(p.get());
    }
    cudaError_t e = cudaGetDevice(&p->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (g_sms == 0) cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, p->device);
    st = p->W > 1 ? upload_wide(p.get()) : upload(p.get());
    if (st) return st;
    // Both storages scan every source for leakage once.  The reference's lazy
    // plan finds a leaking group while it applies (aggregate_source); the
    // destination-major kernel never visits out-of-sector rows, so the scan
    // runs here instead and a lazy plan reports the same error at build.
    st = scan_leakage(p.get());
    if (!st && storage == TCP_STORAGE_EAGER) {
        uint64_t count = 0;
        st = count_transitions(p.get(), nullptr, count, nullptr);
        if (!st) p->transitions = static_cast<int64_t>(count);
    }
    if (st) {
        cudaFree(p->block);
        p->block = nullptr;
        return st;
    }
    *out_plan = p.release();
    return TCP_OK;
}

extern "C" int tcp_u1_plan_destroy(tcp_u1_plan *plan) {
    if (plan == nullptr) return TCP_OK;
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != plan->device) cudaSetDevice(plan->device);
    for (void *w : plan->ws_all) cudaFree(w);
    if (plan->block) cudaFree(plan->block);
    if (prev >= 0 && prev != plan->device) cudaSetDevice(prev);
    delete plan;
    return TCP_OK;
}

extern "C" int tcp_u1_plan_info(const tcp_u1_plan *plan, tcp_u1_plan_info_t *info) {
    if (plan == nullptr || info == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "null argument");
    std::memset(info, 0, sizeof(*info));
    info->nqubits = plan->n;
    info->particle_number = plan->k;
    info->dimension = plan->dim;
    info->term_count = plan->term_count;
    info->group_count = plan->terms.gx.size() / plan->W;
    info->storage = plan->storage;
    info->device = plan->device;
    info->transition_count = plan->transitions;
    info->device_bytes = plan->block_bytes;
    info->estimated_bytes = plan->estimated;
    info->complement = plan->comp;
    info->rank_chunks = plan->nchunk;
    info->tables_in_shared = plan->smem ? 1 : 0;
    return TCP_OK;
}

extern "C" int tcp_u1_apply_into_host(const tcp_u1_plan *plan, const double *state, uint64_t state_len,
                                      double *result, uint64_t result_len, uint64_t max_bytes) {
    tcp::Range range("tcp_u1_apply_into_host");
    (void)max_bytes;  // advisory: the output is caller-owned
    return apply_host<double>(plan, state, state_len, result, result_len);
}

extern "C" int tcp_u1_apply_into_device(const tcp_u1_plan *plan, const void *d_state, void *d_result, uint64_t len,
                                        uint32_t nrhs, int dtype, void *stream) {
    int st = check_u1(plan);
    if (st) return st;
    if (len != plan->dim) return tcp::length_error(plan->dim, len);
    if (dtype != TCP_DTYPE_C128 && dtype != TCP_DTYPE_C64) return fail(TCP_ERR_INVALID_ARGUMENT, "unknown dtype");
    if (nrhs == 0) return TCP_OK;
    if (d_state == nullptr || d_result == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    const size_t elem = dtype == TCP_DTYPE_C128 ? 16 : 8;
    const size_t bytes = static_cast<size_t>(len) * elem * nrhs;
    auto pa = reinterpret_cast<uintptr_t>(d_state), pb = reinterpret_cast<uintptr_t>(d_result);
    if (pa < pb + bytes && pb < pa + bytes) return fail(TCP_ERR_INVALID_ARGUMENT, "input and output must not overlap");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    for (uint32_t v = 0; v < nrhs; ++v) {
        const void *x = static_cast<const unsigned char *>(d_state) + static_cast<size_t>(v) * len * elem;
        void *y = static_cast<unsigned char *>(d_result) + static_cast<size_t>(v) * len * elem;
        st = dtype == TCP_DTYPE_C128 ? launch_apply<double>(plan, x, y, s) : launch_apply<float>(plan, x, y, s);
        if (st) return st;
    }
    return TCP_OK;
}

extern "C" int tcp_u1_diagonal_device(const tcp_u1_plan *plan, void *d_diag, uint64_t len, void *stream) {
    int st = check_u1(plan);
    if (st) return st;
    if (len != plan->dim) return tcp::length_error(plan->dim, len);
    if (d_diag == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (plan->W > 1) {
        double2 *out = static_cast<double2 *>(d_diag);
        if (plan->W == 2) k_u1w_diag<2><<<grid_for(plan->dim), kU1Threads, 0, s>>>(plan->wdev, plan->terms.gzero, out);
        else k_u1w_diag<4><<<grid_for(plan->dim), kU1Threads, 0, s>>>(plan->wdev, plan->terms.gzero, out);
        cudaError_t ew = cudaGetLastError();
        return ew == cudaSuccess ? TCP_OK : cuda_fail(ew, "wide sector diagonal kernel launch");
    }
    // the plan holds the diagonal of its x == 0 group (zero when it has none)
    cudaError_t e = plan->app.diag ? cudaMemcpyAsync(d_diag, plan->app.diag, 16 * plan->dim, cudaMemcpyDeviceToDevice, s)
                                   : cudaMemsetAsync(d_diag, 0, 16 * plan->dim, s);
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "copying the sector diagonal");
}

extern "C" int tcp_u1_transition_count(const tcp_u1_plan *plan, uint64_t *out_count) {
    int st = check_u1(plan);
    if (st) return st;
    if (out_count == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "null output");
    if (plan->transitions >= 0) {
        *out_count = static_cast<uint64_t>(plan->transitions);
        return TCP_OK;
    }
    return count_transitions(plan, nullptr, *out_count, nullptr);
}

extern "C" int tcp_u1_csr(const tcp_u1_plan *plan, uint64_t *indptr, uint64_t *columns, double *values,
                          uint64_t capacity, uint64_t *out_nnz) {
    int st = check_u1(plan);
    if (st) return st;
    if (indptr == nullptr || out_nnz == nullptr) return fail(TCP_ERR_INVALID_ARGUMENT, "null output");
    const uint64_t D = plan->dim;
    if (D >= (1ull << 31)) return fail(TCP_ERR_OVERFLOW, "integer overflow while sizing the CSR rows (at most 2^31 - 1 rows)");
    uint64_t *d_counts = nullptr;
    uint64_t *d_indptr = nullptr;
    cudaError_t e = cudaMalloc(&d_counts, sizeof(uint64_t) * (D + 1));
    if (e == cudaSuccess) e = cudaMalloc(&d_indptr, sizeof(uint64_t) * (D + 1));
    if (e != cudaSuccess) {
        cudaGetLastError();
        cudaFree(d_counts);
        return fail(TCP_ERR_ALLOCATION, "device allocation of the CSR row counts failed");
    }
    uint64_t nnz = 0;
    cudaMemset(d_counts, 0, sizeof(uint64_t) * (D + 1));
    st = count_transitions(plan, d_counts, nnz, nullptr);
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    uint64_t *d_cols = nullptr, *d_cols2 = nullptr;
    double2 *d_vals = nullptr, *d_vals2 = nullptr;
    if (!st) {
        *out_nnz = nnz;
        if (nnz >= (1ull << 31)) st = fail(TCP_ERR_OVERFLOW, "integer overflow while sizing the CSR entries (at most 2^31 - 1)");
        else if (nnz > capacity) st = fail(TCP_ERR_MEMORY_LIMIT, "CSR output needs " + std::to_string(nnz) + " entries, capacity is " + std::to_string(capacity));
        else if (nnz && (columns == nullptr || values == nullptr)) st = fail(TCP_ERR_INVALID_ARGUMENT, "null output");
    }
    if (!st) {
        // indptr = exclusive scan of the row counts (D + 1 entries, last count 0)
        cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, d_counts, d_indptr, static_cast<int>(D + 1));
        size_t sort_bytes = 0;
        cub::DeviceSegmentedSort::SortPairs(nullptr, sort_bytes, d_cols, d_cols2, d_vals, d_vals2,
                                            static_cast<int>(nnz), static_cast<int>(D), d_indptr, d_indptr + 1);
        tmp_bytes = std::max(tmp_bytes, sort_bytes);
        e = cudaMalloc(&tmp, std::max<size_t>(tmp_bytes, 16));
        if (e == cudaSuccess && nnz) e = cudaMalloc(&d_cols, 2 * 8 * nnz);
        if (e == cudaSuccess && nnz) e = cudaMalloc(&d_vals, 2 * 16 * nnz);
        if (e != cudaSuccess) {
            cudaGetLastError();
            st = fail(TCP_ERR_ALLOCATION, "device allocation of the CSR arrays failed");
        }
    }
    if (!st) {
        size_t scan_bytes = tmp_bytes;
        e = cub::DeviceScan::ExclusiveSum(tmp, scan_bytes, d_counts, d_indptr, static_cast<int>(D + 1));
        if (e == cudaSuccess && nnz) {
            d_cols2 = d_cols + nnz;
            d_vals2 = d_vals + nnz;
            const int grid = grid_for(D);
            if (plan->W == 2 && plan->index32) k_u1w_fill<2, uint32_t><<<grid, kU1Threads>>>(plan->wdev, d_indptr, d_cols, d_vals);
            else if (plan->W == 2) k_u1w_fill<2, uint64_t><<<grid, kU1Threads>>>(plan->wdev, d_indptr, d_cols, d_vals);
            else if (plan->W == 4 && plan->index32) k_u1w_fill<4, uint32_t><<<grid, kU1Threads>>>(plan->wdev, d_indptr, d_cols, d_vals);
            else if (plan->W == 4) k_u1w_fill<4, uint64_t><<<grid, kU1Threads>>>(plan->wdev, d_indptr, d_cols, d_vals);
            else if (plan->basis32) k_u1_fill<uint32_t, uint32_t><<<grid, kU1Threads>>>(plan->dev, d_indptr, d_cols, d_vals);
            else if (plan->index32) k_u1_fill<uint64_t, uint32_t><<<grid, kU1Threads>>>(plan->dev, d_indptr, d_cols, d_vals);
            else k_u1_fill<uint64_t, uint64_t><<<grid, kU1Threads>>>(plan->dev, d_indptr, d_cols, d_vals);
            e = cudaGetLastError();
            if (e == cudaSuccess) {
                size_t sort_bytes = tmp_bytes;
                e = cub::DeviceSegmentedSort::SortPairs(tmp, sort_bytes, d_cols, d_cols2, d_vals, d_vals2,
                                                        static_cast<int>(nnz), static_cast<int>(D), d_indptr,
                                                        d_indptr + 1);
            }
        }
        if (e == cudaSuccess) e = cudaMemcpy(indptr, d_indptr, 8 * (D + 1), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && nnz) e = cudaMemcpy(columns, d_cols2, 8 * nnz, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && nnz) e = cudaMemcpy(values, d_vals2, 16 * nnz, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) st = cuda_fail(e, "building the sector CSR arrays");
    }
    cudaFree(tmp);
    cudaFree(d_cols);
    cudaFree(d_vals);
    cudaFree(d_counts);
    cudaFree(d_indptr);
    return st;
}

extern "C" int tcp_u1_plan_device_status(const tcp_u1_plan *plan) {
    int st = check_u1(plan);
    if (st) return st;
    cudaError_t e = cudaDeviceSynchronize();
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "cudaDeviceSynchronize");
}
