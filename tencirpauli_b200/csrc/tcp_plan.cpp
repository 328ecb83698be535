// Host side of libtcpmvp.so: error slot, canonicalization, term compilation and
// the tile schedule.  Pure C++ (no CUDA); compiled by nvcc with the kernels.
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <numeric>

#include "tcp_internal.h"

namespace tcp {

namespace {
thread_local std::string g_last_error;
thread_local int g_last_status = 0;
thread_local uint64_t g_last_fields[2] = {0, 0};
std::atomic<long long> g_alloc_count{0};
}  // namespace

void set_error(const std::string &message) { g_last_error = message; }

int fail(int status, const std::string &message) { return fail_fields(status, message, 0, 0); }

int fail_fields(int status, const std::string &message, uint64_t a, uint64_t b) {
    g_last_error = message;
    g_last_status = status;
    g_last_fields[0] = a;
    g_last_fields[1] = b;
    return status;
}

uint64_t clamp_u64(unsigned __int128 v) { return (v >> 64) ? ~0ull : static_cast<uint64_t>(v); }

bool injected_alloc_failure() {
    const char *env = std::getenv("TCP_FAIL_ALLOC_AFTER");
    if (env == nullptr || *env == '\0') return false;
    long long limit = std::atoll(env);
    long long index = g_alloc_count.fetch_add(1);
    return index >= limit;
}

static inline uint32_t packed_word_count(uint32_t nqubits) { return nqubits / 64 + (nqubits % 64 != 0); }

int compile_terms(uint32_t nqubits, uint64_t count, uint32_t word_count, const uint64_t *x_words,
                  const uint64_t *z_words, const double *coefficients, std::vector<MatrixTerm> &out) {
    // pauli_action.rs:38-55 -- word-length and dimension checks
    uint32_t expected = packed_word_count(nqubits);
    if (word_count != expected) {
        return fail_fields(TCP_ERR_INVALID_WORD_LENGTH,
                           "expected " + std::to_string(expected) + " packed words, got " + std::to_string(word_count),
                           expected, word_count);
    }
    if (nqubits >= 64) return fail(TCP_ERR_OVERFLOW, "integer overflow while computing dense statevector dimension");
    out.clear();
    out.reserve(count);
    // word.rs:81-85: bits above nqubits in the final word are masked off
    uint64_t tail = (nqubits % 64) ? ((1ull << (nqubits % 64)) - 1) : ~0ull;
    for (uint64_t t = 0; t < count; ++t) {
        double re = coefficients[2 * t], im = coefficients[2 * t + 1];
        if (!std::isfinite(re) || !std::isfinite(im)) {
            return fail_fields(TCP_ERR_NON_FINITE_COEFFICIENT, "coefficient at index " + std::to_string(t) + " is not finite",
                               t, 0);
        }
        uint64_t xm = 0, zm = 0;
        uint32_t ny = 0;
        for (uint32_t q = 0; q < nqubits; ++q) {
            uint64_t packed = 1ull << (q % 64);
            uint64_t xw = x_words[t * word_count + q / 64];
            uint64_t zw = z_words[t * word_count + q / 64];
            if (q / 64 == word_count - 1) {
                xw &= tail;
                zw &= tail;
            }
            bool x = (xw & packed) != 0, z = (zw & packed) != 0;
            uint64_t bit = 1ull << (nqubits - 1 - q);
            if (x) xm |= bit;
            if (z) zm |= bit;
            if (x && z) ++ny;
        }
        // y_phase = i^{#Y mod 4}; weighted = coefficient * y_phase with the
        // textbook complex product (num-complex): (a c - b d, a d + b c).
        double pr = 0.0, pi = 0.0;
        switch (ny % 4) {
        case 0: pr = 1.0; break;
        case 1: pi = 1.0; break;
        case 2: pr = -1.0; break;
        default: pi = -1.0; break;
        }
        MatrixTerm mt;
        mt.x_mask = xm;
        mt.z_mask = zm;
        volatile double ac = re * pr, bd = im * pi, ad = re * pi, bc = im * pr;  // no contraction
        mt.w_re = ac - bd;
        mt.w_im = ad + bc;
        out.push_back(mt);
    }
    return TCP_OK;
}

uint64_t distinct_x_masks(const std::vector<MatrixTerm> &terms) {
    std::vector<uint64_t> m;
    m.reserve(terms.size());
    for (auto &t : terms) m.push_back(t.x_mask);
    std::sort(m.begin(), m.end());
    return static_cast<uint64_t>(std::unique(m.begin(), m.end()) - m.begin());
}

namespace {
template <typename T> void put(std::vector<uint8_t> &out, const T &v) {
    const uint8_t *p = reinterpret_cast<const uint8_t *>(&v);
    out.insert(out.end(), p, p + sizeof(T));
}
}  // namespace

Schedule build_schedule(const std::vector<MatrixTerm> &terms, uint32_t nqubits, uint32_t tile_bits,
                        uint32_t log_threads) {
    Schedule s;
    s.tile_bits = std::min(tile_bits, nqubits);
    s.log_threads = std::min(log_threads, s.tile_bits);
    const uint32_t S = s.tile_bits;
    const uint32_t L = s.log_threads;
    const uint64_t inner = (S >= 64) ? ~0ull : ((1ull << S) - 1);
    const uint32_t jcount = 1u << (S - L);
    // (outer, inner, canonical index): a stable order that keeps canonical
    // term order inside every x-mask group.
    std::vector<uint64_t> order(terms.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](uint64_t a, uint64_t b) {
        uint64_t da = terms[a].x_mask >> S, db = terms[b].x_mask >> S;
        if (da != db) return da < db;
        return (terms[a].x_mask & inner) < (terms[b].x_mask & inner);
    });
    // group view
    s.g_tbeg.push_back(0);
    for (size_t i = 0; i < order.size(); ++i) {
        const MatrixTerm &t = terms[order[i]];
        if (s.g_mask.empty() || s.g_mask.back() != t.x_mask) {
            if (!s.g_mask.empty()) s.g_tbeg.push_back(static_cast<uint32_t>(i));
            s.g_mask.push_back(t.x_mask);
        }
        s.t_z.push_back(t.z_mask);
        s.t_w.push_back(t.w_re);
        s.t_w.push_back(t.w_im);
        s.t_wf.push_back(static_cast<float>(t.w_re));
        s.t_wf.push_back(static_cast<float>(t.w_im));
    }
    if (!s.g_mask.empty()) s.g_tbeg.push_back(static_cast<uint32_t>(order.size()));

    // step view: walk the groups, packing blocks of at most kBlockBytesMax
    struct Pending {
        uint32_t m_in;
        size_t gid;                   // group index in the group view
        std::vector<uint64_t> terms;  // indices into `terms`
    };
    uint64_t cur_d = 0;
    std::vector<Pending> pend;
    size_t pend_bytes = 0;
    auto flush = [&]() {
        if (pend.empty()) return;
        const size_t off = s.blocks_c128.size();
        uint32_t nterms = 0;
        for (auto &g : pend) {
            put(s.blocks_c128, g.m_in);
            put(s.blocks_c128, nterms);
            nterms += static_cast<uint32_t>(g.terms.size());
            put(s.blocks_c128, nterms);
            put(s.blocks_c128, uint32_t(0));
        }
        for (auto &g : pend) {
            for (uint64_t ti : g.terms) {
                const MatrixTerm &t = terms[ti];
                const uint64_t zt = (S >= 64) ? 0 : (t.z_mask >> S);
                const uint32_t zlo = static_cast<uint32_t>(t.z_mask & ((1ull << L) - 1));
                const uint32_t zj = static_cast<uint32_t>((t.z_mask & inner) >> L);
                uint32_t pattern = 0;
                for (uint32_t jj = 0; jj < jcount; ++jj)
                    pattern |= (static_cast<uint32_t>(__builtin_popcount(zj & jj)) & 1u) << jj;
                const uint32_t kind = (t.w_im == 0.0) ? kKindReal : ((t.w_re == 0.0) ? kKindImag : kKindComplex);
                const uint64_t zrec = static_cast<uint64_t>(zlo) | (static_cast<uint64_t>(pattern) << 32) |
                                      (static_cast<uint64_t>(kind) << 56);
                // parity(zt & d), parity(zlo & m_lo) and parity(zj & jh) are
                // fixed for the term inside its step and group, so they are
                // folded into the weight.  (The kernel loads row j's source
                // j ^ jh into register j, so the remaining sign of row j is
                // bit j of the pattern, parity(zj & j), XOR the thread's base.)
                const uint32_t m_lo = g.m_in & ((1u << L) - 1u);
                const uint32_t jh = g.m_in >> L;
                const bool flip = ((__builtin_popcountll(zt & cur_d) + __builtin_popcount(zlo & m_lo) +
                                    __builtin_popcount(zj & jh)) & 1) != 0;
                const double wr = flip ? -t.w_re : t.w_re, wi = flip ? -t.w_im : t.w_im;
                put(s.blocks_c128, zrec);
                put(s.blocks_c128, zt);
                put(s.blocks_c128, wr);
                put(s.blocks_c128, wi);
            }
        }
        const size_t bytes = s.blocks_c128.size() - off;
        s.step_info.push_back(static_cast<uint32_t>(cur_d));
        s.step_info.push_back(static_cast<uint32_t>(cur_d >> 32));
        s.step_info.push_back(static_cast<uint32_t>(off / 16));
        s.step_info.push_back(static_cast<uint32_t>(pend.size()) | static_cast<uint32_t>((bytes / 16) << 16));
        pend.clear();
        pend_bytes = 0;
    };
    bool have_step = false;
    for (size_t g = 0; g < s.g_mask.size(); ++g) {
        const uint64_t d = s.g_mask[g] >> S;
        const uint32_t m_in = static_cast<uint32_t>(s.g_mask[g] & inner);
        if (!have_step || d != cur_d) {
            flush();
            cur_d = d;
            have_step = true;
            ++s.distinct_outer;
        }
        for (uint32_t t = s.g_tbeg[g]; t < s.g_tbeg[g + 1]; ++t) {
            bool opens = pend.empty() || pend.back().gid != g;
            if (pend_bytes + kTermRecBytes + (opens ? kGroupRecBytes : 0) > kBlockBytesMax) {
                flush();
                opens = true;
            }
            if (opens) {
                pend.push_back(Pending{m_in, g, {}});
                pend_bytes += kGroupRecBytes;
            }
            pend.back().terms.push_back(order[t]);
            pend_bytes += kTermRecBytes;
        }
    }
    flush();
    // complex64 blocks: same layout, weights as two floats + 8 pad bytes
    s.blocks_c64 = s.blocks_c128;
    for (size_t i = 0; i + 4 <= s.step_info.size(); i += 4) {
        const size_t off = static_cast<size_t>(s.step_info[i + 2]) * 16;
        const uint32_t ng = s.step_info[i + 3] & 0xffffu;
        const size_t bytes = static_cast<size_t>(s.step_info[i + 3] >> 16) * 16;
        for (size_t p = off + ng * kGroupRecBytes; p < off + bytes; p += kTermRecBytes) {
            double wr, wi;
            std::memcpy(&wr, &s.blocks_c128[p + 16], 8);
            std::memcpy(&wi, &s.blocks_c128[p + 24], 8);
            const float fr = static_cast<float>(wr), fi = static_cast<float>(wi);
            std::memcpy(&s.blocks_c64[p + 16], &fr, 4);
            std::memcpy(&s.blocks_c64[p + 20], &fi, 4);
            std::memset(&s.blocks_c64[p + 24], 0, 8);
        }
    }
    return s;
}

RingSchedule build_ring_schedule(const std::vector<MatrixTerm> &terms, uint32_t nqubits, uint32_t tile_bits,
                                 uint32_t log_threads) {
    RingSchedule r;
    // The ring kernel covers 512 threads x 8 rows per tile, and outer z bits
    // that fit 32 bits.
    if (log_threads != 9 || tile_bits != 12 || nqubits < tile_bits || nqubits - tile_bits > 32) return r;
    const uint32_t S = tile_bits, L = log_threads;
    const uint64_t inner = (1ull << S) - 1, tmask = (1ull << L) - 1;
    r.tile_bits = S;
    r.log_threads = L;

    // One record per real or imaginary weight part; canonical order inside a
    // group, real part before imaginary part.
    struct Item {
        uint64_t d;
        uint32_t m_lo, jh;
        uint64_t mask;
        uint64_t z;
        uint64_t canon;
        uint32_t imag;
        double w;
    };
    std::vector<Item> items;
    items.reserve(terms.size() + 8);
    for (uint64_t i = 0; i < terms.size(); ++i) {
        const MatrixTerm &t = terms[i];
        const uint64_t d = t.x_mask >> S;
        const uint32_t m_lo = static_cast<uint32_t>(t.x_mask & tmask);
        const uint32_t jh = static_cast<uint32_t>((t.x_mask & inner) >> L);
        if (t.w_re != 0.0 || t.w_im == 0.0) items.push_back({d, m_lo, jh, t.x_mask, t.z_mask, i, 0u, t.w_re});
        if (t.w_im != 0.0) items.push_back({d, m_lo, jh, t.x_mask, t.z_mask, i, 1u, t.w_im});
    }
    std::stable_sort(items.begin(), items.end(), [](const Item &a, const Item &b) {
        if (a.d != b.d) return a.d < b.d;
        if (a.m_lo != b.m_lo) return a.m_lo < b.m_lo;
        if (a.jh != b.jh) return a.jh < b.jh;
        return a.canon < b.canon;
    });

    struct PGroup {
        uint32_t a = 0;
        std::vector<size_t> items;
    };
    struct PCoset {
        uint32_t m_lo = 0, jh = 0;
        std::vector<PGroup> groups;
    };
    auto pattern_of = [&](const Item &it) {
        const uint32_t zj = static_cast<uint32_t>((it.z & inner) >> L);
        uint32_t pattern = 0;
        for (uint32_t j = 0; j < 8; ++j) pattern |= (static_cast<uint32_t>(__builtin_popcount(zj & j)) & 1u) << j;
        return pattern;
    };
    // run of a record: real / imaginary weight x uniform / patterned sign
    auto run_of = [&](const Item &it) { return (it.imag << 1) | (pattern_of(it) != 0u ? 1u : 0u); };
    std::vector<PCoset> pend;
    size_t pend_groups = 0, pend_terms = 0;
    uint64_t cur_d = 0;
    auto block_bytes = [](size_t c, size_t g, size_t t) { return 16 + 16 * c + (4 * g + 15) / 16 * 16 + 16 * t; };
    auto flush = [&]() {
        if (pend.empty()) return;
        const size_t off = r.blocks_c128.size();
        const size_t terms_off = 16 + 16 * pend.size() + (4 * pend_groups + 15) / 16 * 16;
        put(r.blocks_c128, static_cast<uint32_t>(pend.size()));
        put(r.blocks_c128, static_cast<uint32_t>(pend_groups));
        put(r.blocks_c128, static_cast<uint32_t>(terms_off / 16));
        put(r.blocks_c128, uint32_t(0));
        for (auto &c : pend) {
            put(r.blocks_c128, c.m_lo);
            put(r.blocks_c128, c.jh);
            put(r.blocks_c128, static_cast<uint32_t>(c.groups.size()));
            put(r.blocks_c128, uint32_t(0));
        }
        for (auto &c : pend)
            for (auto &g : c.groups) put(r.blocks_c128, g.a | static_cast<uint32_t>(g.items.size() << 4));
        while ((r.blocks_c128.size() - off) % 16) r.blocks_c128.push_back(0);
        for (auto &c : pend) {
            for (auto &g : c.groups) {
                // records of a group in four runs: real uniform-sign, real
                // patterned, imaginary uniform-sign, imaginary patterned
                std::stable_sort(g.items.begin(), g.items.end(),
                                 [&](size_t u, size_t v) { return run_of(items[u]) < run_of(items[v]); });
                for (size_t k : g.items) {
                    const Item &it = items[k];
                    const uint64_t zt = it.z >> S;
                    const uint32_t zlo = static_cast<uint32_t>(it.z & tmask);
                    const uint32_t zj = static_cast<uint32_t>((it.z & inner) >> L);
                    const uint32_t pattern = pattern_of(it);
                    const bool flip = ((__builtin_popcountll(zt & cur_d) + __builtin_popcount(zlo & it.m_lo) +
                                        __builtin_popcount(zj & it.jh)) & 1) != 0;
                    const double w = flip ? -it.w : it.w;
                    put(r.blocks_c128, zlo | (pattern << 9) | (it.imag << 17));
                    put(r.blocks_c128, static_cast<uint32_t>(zt));
                    put(r.blocks_c128, w);
                }
            }
        }
        const size_t bytes = r.blocks_c128.size() - off;
        r.max_block_bytes = std::max<uint32_t>(r.max_block_bytes, static_cast<uint32_t>(bytes));
        r.step_info.push_back(static_cast<uint32_t>(cur_d));
        r.step_info.push_back(static_cast<uint32_t>(cur_d >> 32));
        r.step_info.push_back(static_cast<uint32_t>(off / 16));
        r.step_info.push_back(static_cast<uint32_t>(bytes / 16));
        r.cosets += pend.size();
        pend.clear();
        pend_groups = pend_terms = 0;
    };
    bool have = false;
    for (size_t k = 0; k < items.size(); ++k) {
        const Item &it = items[k];
        if (!have || it.d != cur_d) {
            flush();
            cur_d = it.d;
            have = true;
        }
        bool new_coset = pend.empty() || pend.back().m_lo != it.m_lo;
        bool new_group = new_coset || items[pend.back().groups.back().items.back()].mask != it.mask;
        if (block_bytes(pend.size() + new_coset, pend_groups + new_group, pend_terms + 1) > kRingBlockBytes) {
            flush();
            new_coset = new_group = true;
        }
        if (new_coset) {
            PCoset c;
            c.m_lo = it.m_lo;
            c.jh = 0;  // row-order loads: the permutation lives in each group's a
            pend.push_back(c);
        }
        if (new_group) {
            PGroup g;
            g.a = it.jh;
            pend.back().groups.push_back(g);
            ++pend_groups;
        }
        pend.back().groups.back().items.push_back(k);
        ++pend_terms;
    }
    flush();
    // complex64 blocks: the same layout with the weight rounded to FP32
    r.blocks_c64 = r.blocks_c128;
    for (size_t i = 0; i + 4 <= r.step_info.size(); i += 4) {
        const size_t off = static_cast<size_t>(r.step_info[i + 2]) * 16;
        const size_t bytes = static_cast<size_t>(r.step_info[i + 3]) * 16;
        uint32_t terms_off;
        std::memcpy(&terms_off, &r.blocks_c128[off + 8], 4);
        for (size_t p = off + static_cast<size_t>(terms_off) * 16; p < off + bytes; p += 16) {
            double w;
            std::memcpy(&w, &r.blocks_c128[p + 8], 8);
            const float f = static_cast<float>(w);
            std::memcpy(&r.blocks_c64[p + 8], &f, 4);
            std::memset(&r.blocks_c64[p + 12], 0, 4);
        }
    }
    return r;
}

}  // namespace tcp

// ---------------------------------------------------------------------------
// C ABI: canonicalization (operator.rs:117-155)
// ---------------------------------------------------------------------------
namespace {
inline uint8_t code_at(const uint64_t *xw, const uint64_t *zw, uint32_t q) {
    uint64_t x = (xw[q / 64] >> (q % 64)) & 1u, z = (zw[q / 64] >> (q % 64)) & 1u;
    return x ? (z ? 2 : 1) : (z ? 3 : 0);
}
inline uint64_t bits_of(double v) {
    uint64_t b;
    std::memcpy(&b, &v, sizeof b);
    return b;
}
}  // namespace

extern "C" int tcp_pauli_canonicalize(uint32_t nqubits, uint64_t count, const uint8_t *codes,
                                      const double *coefficients, uint64_t *out_x, uint64_t *out_z,
                                      double *out_coefficients, uint64_t *out_count, uint64_t *bad_index) {
    using namespace tcp;
    if (out_count == nullptr || (count > 0 && (coefficients == nullptr || out_coefficients == nullptr ||
                                               out_x == nullptr || out_z == nullptr ||
                                               (nqubits > 0 && codes == nullptr)))) {
        return fail(TCP_ERR_INVALID_ARGUMENT, "null pointer argument");
    }
    const uint32_t w = packed_word_count(nqubits);
    // Validation in input order, coefficient before codes (operator.rs:130-136).
    for (uint64_t t = 0; t < count; ++t) {
        if (!std::isfinite(coefficients[2 * t]) || !std::isfinite(coefficients[2 * t + 1])) {
            if (bad_index) *bad_index = t;
            return fail_fields(TCP_ERR_NON_FINITE_COEFFICIENT, "coefficient at index " + std::to_string(t) + " is not finite",
                               t, 0);
        }
        for (uint32_t q = 0; q < nqubits; ++q) {
            uint8_t c = codes[t * nqubits + q];
            if (c > 3) {
                if (bad_index) *bad_index = q;
                return fail_fields(TCP_ERR_INVALID_CODE,
                                   "invalid Pauli code " + std::to_string(c) + " at index " + std::to_string(q) +
                                       "; expected 0..=3",
                                   c, q);
            }
        }
    }
    std::vector<uint64_t> xw(count * w + 1, 0), zw(count * w + 1, 0);
    for (uint64_t t = 0; t < count; ++t) {
        for (uint32_t q = 0; q < nqubits; ++q) {
            uint8_t c = codes[t * nqubits + q];
            uint64_t x = (c == 1 || c == 2), z = (c == 2 || c == 3);
            xw[t * w + q / 64] |= x << (q % 64);
            zw[t * w + q / 64] |= z << (q % 64);
        }
    }
    auto word_less = [&](uint64_t a, uint64_t b) -> int {
        for (uint32_t q = 0; q < nqubits; ++q) {
            uint8_t ca = code_at(&xw[a * w], &zw[a * w], q), cb = code_at(&xw[b * w], &zw[b * w], q);
            if (ca != cb) return ca < cb ? -1 : 1;
        }
        return 0;
    };
    std::vector<uint64_t> idx(count);
    std::iota(idx.begin(), idx.end(), 0);
    auto tie_break = [&](uint64_t a, uint64_t b) {
        uint64_t ar = bits_of(coefficients[2 * a]), br = bits_of(coefficients[2 * b]);
        if (ar != br) return ar < br;
        uint64_t ai = bits_of(coefficients[2 * a + 1]), bi = bits_of(coefficients[2 * b + 1]);
        if (ai != bi) return ai < bi;
        return a < b;
    };
    if (nqubits <= 64) {
        // Word order (word.rs:240-254) as a 128-bit integer key: the 2-bit code
        // of qubit 0 is the most significant digit.
        std::vector<std::pair<uint64_t, uint64_t>> key(count);
        for (uint64_t t = 0; t < count; ++t) {
            uint64_t hi = 0, lo = 0;
            for (uint32_t q = 0; q < nqubits; ++q) {
                const uint64_t c = codes[t * nqubits + q];
                const uint32_t pos = 2 * (63 - q);  // digit position inside 128 bits
                if (pos >= 64) hi |= c << (pos - 64); else lo |= c << pos;
            }
            key[t] = {hi, lo};
        }
        std::sort(idx.begin(), idx.end(), [&](uint64_t a, uint64_t b) {
            if (key[a] != key[b]) return key[a] < key[b];
            return tie_break(a, b);
        });
    } else {
        std::sort(idx.begin(), idx.end(), [&](uint64_t a, uint64_t b) {
            int r = word_less(a, b);
            if (r) return r < 0;
            return tie_break(a, b);
        });
    }
    uint64_t out = 0;
    for (uint64_t i = 0; i < count;) {
        uint64_t j = i;
        double sr = 0.0, si = 0.0;
        while (j < count && word_less(idx[i], idx[j]) == 0) {
            sr = sr + coefficients[2 * idx[j]];
            si = si + coefficients[2 * idx[j] + 1];
            ++j;
        }
        if (!(sr == 0.0 && si == 0.0)) {
            for (uint32_t k = 0; k < w; ++k) {
                out_x[out * w + k] = xw[idx[i] * w + k];
                out_z[out * w + k] = zw[idx[i] * w + k];
            }
            out_coefficients[2 * out] = sr;
            out_coefficients[2 * out + 1] = si;
            ++out;
        }
        i = j;
    }
    *out_count = out;
    return TCP_OK;
}

extern "C" size_t tcp_last_error(char *buffer, size_t capacity) {
    const std::string &m = tcp::g_last_error;
    if (buffer != nullptr && capacity > 0) {
        size_t n = std::min(capacity - 1, m.size());
        std::memcpy(buffer, m.data(), n);
        buffer[n] = '\0';
    }
    return m.size();
}

extern "C" int tcp_abi_version(void) { return TCP_ABI_VERSION; }

extern "C" int tcp_last_error_fields(uint64_t *fields) {
    if (fields != nullptr) {
        fields[0] = tcp::g_last_fields[0];
        fields[1] = tcp::g_last_fields[1];
    }
    return tcp::g_last_status;
}
