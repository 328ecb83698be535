/*
 * u1_oracle.c -- TEST INFRASTRUCTURE ONLY: a plain-C restatement of
 * TenCirPauli's fixed-Hamming-weight (U(1)) sector path, the checker of the
 * CUDA sector plan.  Only tests, smoke() and the bench's CPU arms use it.
 *
 * Reference items (paths inside crates/tencir-pauli-core/src):
 *   sector.rs:79-99      U1Sector::new (active number, complement flag)
 *   sector.rs:141-167,310-341  rank_words / rank_active_words
 *   sector.rs:184-238    unrank_into
 *   sector.rs:579-643    U1LazyMvpPlan::apply_into (source-major)
 *   sector.rs:926-1021   compile_terms (x-mask groups in first-appearance order)
 *   sector.rs:1051-1127  aggregate_source (group value, zero skip, leakage)
 *   sector.rs:1147-1170  pauli_z_parity (complement-aware parity)
 *   sector.rs:345-431,699-730  U1RestrictedOperator::new / csr (destination-major CSR)
 *   operator.rs:396-444  analyze_charge (number-charge selection rule)
 *
 * States are packed occupation words: qubit q at word q / 64, bit q % 64.
 * Any qubit count is accepted.  Error returns: 10 invalid sector, 11 sector
 * leakage (*leak_source / *leak_weight set), 13 invalid index, 8 overflow.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    double re, im;
} ucplx;

static uint32_t wcount(uint32_t n) { return n / 64 + (n % 64 != 0); }

/* C(n, k) with a 128-bit running product; returns 0 on overflow of u64. */
static int binom(uint64_t n, uint64_t k, uint64_t *out) {
    if (k > n) {
        *out = 0;
        return 1;
    }
    if (k > n - k) k = n - k;
    unsigned __int128 v = 1;
    for (uint64_t i = 1; i <= k; ++i) {
        v = v * (n - k + i) / i;
        if (v > (unsigned __int128)UINT64_MAX) return 0;
    }
    *out = (uint64_t)v;
    return 1;
}

int oracle_u1_dimension(uint32_t n, uint32_t k, uint64_t *dim) {
    if (k > n) return 10;
    return binom(n, k, dim) ? 0 : 8;
}

/* rank over the "active" qubits: set qubits, or clear qubits when the sector
 * is complemented (k > n - k), each adding C(n - position - 1, still needed). */
int oracle_u1_rank(uint32_t n, uint32_t k, const uint64_t *words, uint64_t *rank) {
    uint64_t dim;
    int st = oracle_u1_dimension(n, k, &dim);
    if (st) return st;
    const uint32_t W = wcount(n);
    uint64_t weight = 0;
    for (uint32_t w = 0; w < W; ++w) weight += (uint64_t)__builtin_popcountll(words[w]);
    if (W && (n % 64) && (words[W - 1] >> (n % 64))) return 13;
    if (weight != k) return 13;
    const int complement = k > n - k;
    const uint32_t active = complement ? n - k : k;
    uint64_t r = 0;
    uint32_t selected = 0;
    for (uint32_t q = 0; q < n; ++q) {
        int bit = (int)((words[q / 64] >> (q % 64)) & 1);
        if (complement) bit = !bit;
        if (!bit) continue;
        uint64_t c = 0;
        binom(n - q - 1, active - selected, &c);
        r += c;
        ++selected;
    }
    *rank = complement ? dim - 1 - r : r;
    return 0;
}

int oracle_u1_unrank(uint32_t n, uint32_t k, uint64_t index, uint64_t *words) {
    uint64_t dim;
    int st = oracle_u1_dimension(n, k, &dim);
    if (st) return st;
    if (index >= dim) return 13;
    const uint32_t W = wcount(n);
    memset(words, 0, sizeof(uint64_t) * W);
    const int complement = k > n - k;
    uint32_t remaining = complement ? n - k : k;
    uint64_t a = complement ? dim - 1 - index : index;
    for (uint32_t q = 0; q < n; ++q) {
        uint64_t zero_count = 0;
        binom(n - q - 1, remaining, &zero_count);
        if (a >= zero_count) {
            a -= zero_count;
            if (remaining == 0) return 13;
            words[q / 64] |= 1ull << (q % 64);
            --remaining;
        }
    }
    if (remaining || a) return 13;
    if (complement) {
        for (uint32_t w = 0; w < W; ++w) words[w] = ~words[w];
        if (n % 64) words[W - 1] &= (1ull << (n % 64)) - 1;
    }
    return 0;
}

/* ------------------------------- terms ----------------------------------- */
typedef struct {
    uint32_t n, W;
    uint64_t ngroups;
    uint64_t *gx;      /* [G * W] */
    uint64_t *gstart;  /* [G + 1] */
    uint64_t *tz;      /* [T * W] grouped */
    ucplx *tw;         /* [T] grouped */
} u1terms;

static ucplx weighted(const uint64_t *x, const uint64_t *z, uint32_t W, double re, double im) {
    uint64_t ny = 0;
    for (uint32_t w = 0; w < W; ++w) ny += (uint64_t)__builtin_popcountll(x[w] & z[w]);
    double pr = 0, pi = 0;
    switch (ny % 4) {
    case 0: pr = 1; break;
    case 1: pi = 1; break;
    case 2: pr = -1; break;
    default: pi = -1; break;
    }
    ucplx out = {re * pr - im * pi, re * pi + im * pr};
    return out;
}

static int build_terms(uint32_t n, uint64_t count, const uint64_t *xw, const uint64_t *zw, const double *coef,
                       u1terms *t) {
    const uint32_t W = wcount(n);
    t->n = n;
    t->W = W;
    uint64_t *group_of = malloc(sizeof(uint64_t) * (count ? count : 1));
    t->gx = malloc(sizeof(uint64_t) * (count * W + 1));
    uint64_t *counts = calloc(count + 1, sizeof(uint64_t));
    uint64_t G = 0;
    for (uint64_t i = 0; i < count; ++i) {  /* first appearance order; linear lookup */
        uint64_t g;
        for (g = 0; g < G; ++g)
            if (!memcmp(t->gx + g * W, xw + i * W, sizeof(uint64_t) * W)) break;
        if (g == G) {
            memcpy(t->gx + G * W, xw + i * W, sizeof(uint64_t) * W);
            ++G;
        }
        group_of[i] = g;
        ++counts[g];
    }
    t->ngroups = G;
    t->gstart = calloc(G + 1, sizeof(uint64_t));
    for (uint64_t g = 0; g < G; ++g) t->gstart[g + 1] = t->gstart[g] + counts[g];
    uint64_t *next = malloc(sizeof(uint64_t) * (G + 1));
    memcpy(next, t->gstart, sizeof(uint64_t) * (G + 1));
    t->tz = malloc(sizeof(uint64_t) * (count * W + 1));
    t->tw = malloc(sizeof(ucplx) * (count + 1));
    for (uint64_t i = 0; i < count; ++i) {
        uint64_t slot = next[group_of[i]]++;
        memcpy(t->tz + slot * W, zw + i * W, sizeof(uint64_t) * W);
        t->tw[slot] = weighted(xw + i * W, zw + i * W, W, coef[2 * i], coef[2 * i + 1]);
    }
    free(next);
    free(counts);
    free(group_of);
    return 0;
}

static void free_terms(u1terms *t) {
    free(t->gx);
    free(t->gstart);
    free(t->tz);
    free(t->tw);
}

/* pauli_z_parity: parity of |z support ∩ active qubits|, corrected by the
 * parity of |z support| when the active qubits are the holes. */
static int z_parity(const uint64_t *state, const uint64_t *z, uint32_t W, int complement, uint32_t n) {
    uint64_t inter = 0, zs = 0;
    for (uint32_t w = 0; w < W; ++w) {
        uint64_t tail = (w == W - 1 && (n % 64)) ? ((1ull << (n % 64)) - 1) : ~0ull;
        uint64_t active = complement ? (~state[w] & tail) : state[w];
        inter += (uint64_t)__builtin_popcountll(active & z[w]);
        zs += (uint64_t)__builtin_popcountll(z[w]);
    }
    int p = (int)(inter & 1);
    return complement ? p ^ (int)(zs & 1) : p;
}

/* One source: (destination index, value) pairs in group order, zero values
 * skipped, leakage reported. */
typedef struct {
    uint64_t dest;
    ucplx value;
} u1entry;

static int aggregate(const u1terms *t, uint32_t k, uint64_t source_index, const uint64_t *src, uint64_t *dst,
                     u1entry *out, uint64_t *nout, uint64_t *leak_weight) {
    const uint32_t W = t->W, n = t->n;
    const int complement = k > n - k;
    *nout = 0;
    for (uint64_t g = 0; g < t->ngroups; ++g) {
        ucplx v = {0.0, 0.0};
        for (uint64_t i = t->gstart[g]; i < t->gstart[g + 1]; ++i) {
            if (z_parity(src, t->tz + i * W, W, complement, n)) {
                v.re -= t->tw[i].re;
                v.im -= t->tw[i].im;
            } else {
                v.re += t->tw[i].re;
                v.im += t->tw[i].im;
            }
        }
        if (v.re == 0.0 && v.im == 0.0) continue;
        uint64_t weight = 0;
        for (uint32_t w = 0; w < W; ++w) {
            dst[w] = src[w] ^ t->gx[g * W + w];
            weight += (uint64_t)__builtin_popcountll(dst[w]);
        }
        if (weight != k) {
            (void)source_index;
            *leak_weight = weight;
            return 11;
        }
        uint64_t r;
        int st = oracle_u1_rank(n, k, dst, &r);
        if (st) return st;
        out[*nout].dest = r;
        out[*nout].value = v;
        ++*nout;
    }
    return 0;
}

/* U1LazyMvpPlan::apply_into: output zeroed, then sources in ascending order
 * accumulate value * state[source] into their destinations. */
int oracle_u1_apply(uint32_t n, uint32_t k, uint64_t count, const uint64_t *xw, const uint64_t *zw,
                    const double *coef, const double *state, double *out, uint64_t *leak_source,
                    uint64_t *leak_weight) {
    uint64_t dim;
    int st = oracle_u1_dimension(n, k, &dim);
    if (st) return st;
    u1terms t;
    build_terms(n, count, xw, zw, coef, &t);
    const uint32_t W = wcount(n);
    uint64_t *src = calloc(W + 1, sizeof(uint64_t)), *dst = calloc(W + 1, sizeof(uint64_t));
    u1entry *agg = malloc(sizeof(u1entry) * (t.ngroups + 1));
    memset(out, 0, sizeof(double) * 2 * dim);
    for (uint64_t s = 0; s < dim && !st; ++s) {
        oracle_u1_unrank(n, k, s, src);
        uint64_t m = 0, lw = 0;
        st = aggregate(&t, k, s, src, dst, agg, &m, &lw);
        if (st == 11) {
            if (leak_source) *leak_source = s;
            if (leak_weight) *leak_weight = lw;
            break;
        }
        const double xr = state[2 * s], xi = state[2 * s + 1];
        for (uint64_t e = 0; e < m; ++e) {
            const ucplx v = agg[e].value;
            /* output[dest] += value * state, textbook product then add */
            const double pr = v.re * xr - v.im * xi, pi = v.re * xi + v.im * xr;
            out[2 * agg[e].dest] += pr;
            out[2 * agg[e].dest + 1] += pi;
        }
    }
    free(agg);
    free(src);
    free(dst);
    free_terms(&t);
    return st;
}

/* Destination-major CSR of U1RestrictedOperator::new: rows = destinations,
 * entries appended while the sources ascend.  Call with capacity 0 to get
 * *nnz; indptr has dim + 1 entries. */
int oracle_u1_csr(uint32_t n, uint32_t k, uint64_t count, const uint64_t *xw, const uint64_t *zw, const double *coef,
                  uint64_t *indptr, uint64_t *cols, double *vals, uint64_t capacity, uint64_t *nnz,
                  uint64_t *leak_source, uint64_t *leak_weight) {
    uint64_t dim;
    int st = oracle_u1_dimension(n, k, &dim);
    if (st) return st;
    u1terms t;
    build_terms(n, count, xw, zw, coef, &t);
    const uint32_t W = wcount(n);
    uint64_t *src = calloc(W + 1, sizeof(uint64_t)), *dst = calloc(W + 1, sizeof(uint64_t));
    u1entry *agg = malloc(sizeof(u1entry) * (t.ngroups + 1));
    uint64_t *rows = calloc(dim + 1, sizeof(uint64_t));
    for (int pass = 0; pass < 2 && !st; ++pass) {
        uint64_t *next = NULL;
        if (pass == 1) {
            indptr[0] = 0;
            for (uint64_t r = 0; r < dim; ++r) indptr[r + 1] = indptr[r] + rows[r];
            *nnz = indptr[dim];
            if (*nnz > capacity) break;
            next = malloc(sizeof(uint64_t) * (dim + 1));
            memcpy(next, indptr, sizeof(uint64_t) * dim);
        }
        for (uint64_t s = 0; s < dim; ++s) {
            oracle_u1_unrank(n, k, s, src);
            uint64_t m = 0, lw = 0;
            st = aggregate(&t, k, s, src, dst, agg, &m, &lw);
            if (st == 11) {
                if (leak_source) *leak_source = s;
                if (leak_weight) *leak_weight = lw;
                break;
            }
            if (st) break;
            for (uint64_t e = 0; e < m; ++e) {
                if (pass == 0) {
                    ++rows[agg[e].dest];
                } else {
                    uint64_t pos = next[agg[e].dest]++;
                    cols[pos] = s;
                    vals[2 * pos] = agg[e].value.re;
                    vals[2 * pos + 1] = agg[e].value.im;
                }
            }
        }
        free(next);
    }
    free(rows);
    free(agg);
    free(src);
    free(dst);
    free_terms(&t);
    return st;
}

/* analyze_charge with qubit levels (0, 1): commutator words with their
 * contributions; sums run from 0 over contributions sorted by their bit
 * patterns (re, then im).  Returns the number of nonzero sums. */
typedef struct {
    uint64_t *key;  /* 2W words: x then z */
    double re, im;
    uint64_t rb, ib;
} u1contrib;

static uint32_t g_keyw;

static int contrib_cmp(const void *pa, const void *pb) {
    const u1contrib *a = pa, *b = pb;
    int c = memcmp(a->key, b->key, sizeof(uint64_t) * g_keyw);
    if (c) return c;
    if (a->rb != b->rb) return a->rb < b->rb ? -1 : 1;
    if (a->ib != b->ib) return a->ib < b->ib ? -1 : 1;
    return 0;
}

int oracle_number_commutator(uint32_t n, uint64_t count, const uint64_t *xw, const uint64_t *zw, const double *coef,
                             uint64_t *nonzero) {
    const uint32_t W = wcount(n);
    uint64_t total = 0;
    for (uint64_t i = 0; i < count; ++i)
        for (uint32_t w = 0; w < W; ++w) total += (uint64_t)__builtin_popcountll(xw[i * W + w]);
    u1contrib *c = malloc(sizeof(u1contrib) * (total + 1));
    uint64_t *keys = malloc(sizeof(uint64_t) * (2 * W * total + 1));
    uint64_t m = 0;
    const double difference = 0.0 - 1.0;
    for (uint64_t i = 0; i < count; ++i) {
        for (uint32_t q = 0; q < n; ++q) {
            const uint64_t bit = 1ull << (q % 64);
            if (!(xw[i * W + q / 64] & bit)) continue;
            const int is_y = (zw[i * W + q / 64] & bit) != 0;
            const double scale = is_y ? difference : -difference;
            uint64_t *key = keys + 2 * W * m;
            memcpy(key, xw + i * W, sizeof(uint64_t) * W);
            memcpy(key + W, zw + i * W, sizeof(uint64_t) * W);
            key[W + q / 64] ^= bit;
            const double re = coef[2 * i], im = coef[2 * i + 1];
            c[m].key = key;
            c[m].re = re * 0.0 - im * scale;
            c[m].im = re * scale + im * 0.0;
            memcpy(&c[m].rb, &c[m].re, 8);
            memcpy(&c[m].ib, &c[m].im, 8);
            ++m;
        }
    }
    g_keyw = 2 * W;
    qsort(c, m, sizeof(u1contrib), contrib_cmp);
    uint64_t nz = 0;
    for (uint64_t a = 0; a < m;) {
        uint64_t b = a;
        double sr = 0.0, si = 0.0;
        while (b < m && !memcmp(c[a].key, c[b].key, sizeof(uint64_t) * 2 * W)) {
            sr = sr + c[b].re;
            si = si + c[b].im;
            ++b;
        }
        if (sr != 0.0 || si != 0.0) ++nz;
        a = b;
    }
    *nonzero = nz;
    free(keys);
    free(c);
    return 0;
}

/* Selected destination rows of the restricted MVP, pulled from their sources
 * (the destination-major reading of aggregate_source, used to time the CPU
 * baseline on a row sample).  rows: restricted indices; out[2*i] receives
 * row rows[i].  Leakage is not checked here.  OpenMP over rows. */
int oracle_u1_apply_rows(uint32_t n, uint32_t k, uint64_t count, const uint64_t *xw, const uint64_t *zw,
                         const double *coef, const double *state, uint64_t nrows, const uint64_t *rows,
                         double *out, int threads) {
    uint64_t dim;
    int st = oracle_u1_dimension(n, k, &dim);
    if (st) return st;
    u1terms t;
    build_terms(n, count, xw, zw, coef, &t);
    const uint32_t W = wcount(n);
    const int complement = k > n - k;
    int bad = 0;
#pragma omp parallel num_threads(threads > 0 ? threads : 1)
    {
        uint64_t *dst = calloc(W + 1, sizeof(uint64_t)), *src = calloc(W + 1, sizeof(uint64_t));
#pragma omp for schedule(static)
        for (uint64_t r = 0; r < nrows; ++r) {
            double yr = 0.0, yi = 0.0;
            if (rows[r] >= dim || oracle_u1_unrank(n, k, rows[r], dst)) {
                bad = 1;
                continue;
            }
            for (uint64_t g = 0; g < t.ngroups; ++g) {
                uint64_t weight = 0;
                for (uint32_t w = 0; w < W; ++w) {
                    src[w] = dst[w] ^ t.gx[g * W + w];
                    weight += (uint64_t)__builtin_popcountll(src[w]);
                }
                if (weight != k) continue;
                double vr = 0.0, vi = 0.0;
                for (uint64_t i = t.gstart[g]; i < t.gstart[g + 1]; ++i) {
                    if (z_parity(src, t.tz + i * W, W, complement, n)) {
                        vr -= t.tw[i].re;
                        vi -= t.tw[i].im;
                    } else {
                        vr += t.tw[i].re;
                        vi += t.tw[i].im;
                    }
                }
                if (vr == 0.0 && vi == 0.0) continue;
                uint64_t s;
                oracle_u1_rank(n, k, src, &s);
                const double xr = state[2 * s], xi = state[2 * s + 1];
                yr += vr * xr - vi * xi;
                yi += vr * xi + vi * xr;
            }
            out[2 * r] = yr;
            out[2 * r + 1] = yi;
        }
        free(dst);
        free(src);
    }
    free_terms(&t);
    return bad ? 13 : 0;
}
