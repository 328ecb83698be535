/*
 * CPU ORACLE -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of TenCirPauli's CPU matrix-free Pauli MVP (the Rust
 * `tencir-pauli-core` crate, workspace version 0.5.0).  It exists so that the
 * CUDA product path can be checked against the reference's algorithm on the
 * same inputs, and so that `bench.py` can time the reference's CPU loop on the
 * host cores.  Nothing in the product library links, loads or calls this file.
 *
 * Build: `make -C oracle` (gcc -O3 -fopenmp -ffp-contract=off).  Floating-point
 * contraction is disabled because rustc never fuses `a*b + c` into an FMA, and
 * the restatement must round exactly as the Rust loop does.
 *
 * Parity pinning: `tests/test_oracle_golden.py` checks every entry point below
 * against the golden vectors in `tests/golden/` (made from the reference's own
 * dense Kronecker oracle `tests/reference.py` and its fixed vectors).
 *
 * Restated reference items (paths inside the reference project):
 *   crates/tencir-pauli-core/src/word.rs:94-110     PauliWord::from_codes
 *   crates/tencir-pauli-core/src/word.rs:227-254    code_at, Ord for PauliWord
 *   crates/tencir-pauli-core/src/word.rs:291-308    packed_word_count, code_bits
 *   crates/tencir-pauli-core/src/operator.rs:117-155 PauliOperator::from_terms
 *   crates/tencir-pauli-core/src/scalar.rs:5-7      is_exact_zero
 *   crates/tencir-pauli-core/src/pauli_action.rs:24-88 from_packed (masks, phase)
 *   crates/tencir-pauli-core/src/hamiltonian.rs:564-571 matrix_term
 *   crates/tencir-pauli-core/src/hamiltonian.rs:573-582 group_matrix_terms
 *   crates/tencir-pauli-core/src/hamiltonian.rs:79-147  from_operator_reusable
 *   crates/tencir-pauli-core/src/hamiltonian.rs:166-179 transition_count
 *   crates/tencir-pauli-core/src/hamiltonian.rs:204-270 apply_into (hot loop)
 * Complex arithmetic follows num-complex 0.4.6 (Cargo.lock): textbook
 * (ac-bd, ad+bc) products and componentwise sums.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    double re, im;
} cplx;

static inline cplx c_mul(cplx a, cplx b) {
    /* num-complex `Mul for Complex<T>`: (a.re*b.re - a.im*b.im, a.re*b.im + a.im*b.re) */
    cplx r;
    r.re = a.re * b.re - a.im * b.im;
    r.im = a.re * b.im + a.im * b.re;
    return r;
}

static inline cplx c_add(cplx a, cplx b) {
    cplx r;
    r.re = a.re + b.re;
    r.im = a.im + b.im;
    return r;
}

static inline cplx c_neg(cplx a) {
    cplx r;
    r.re = -a.re;
    r.im = -a.im;
    return r;
}

/* Status codes match include/tcp_mvp.h (PauliError variants). */
enum {
    OR_OK = 0,
    OR_INVALID_CODE = 1,
    OR_INVALID_STRUCTURE_LENGTH = 4,
    OR_NON_FINITE_COEFFICIENT = 5,
    OR_OVERFLOW = 8,
    OR_MEMORY_LIMIT = 9,
    OR_ALLOC = 100,
};

/* word.rs:291-293 */
uint32_t oracle_packed_word_count(uint32_t nqubits) {
    return nqubits / 64 + (nqubits % 64 != 0);
}

/* word.rs:94-110 with code_bits (word.rs:296-304): I=(0,0) X=(1,0) Y=(1,1) Z=(0,1). */
int oracle_encode_codes(uint32_t nqubits, uint64_t count, const uint8_t *codes,
                        uint64_t *x_words, uint64_t *z_words) {
    uint32_t w = oracle_packed_word_count(nqubits);
    for (uint64_t t = 0; t < count; ++t) {
        uint64_t *xw = x_words + t * w;
        uint64_t *zw = z_words + t * w;
        for (uint32_t i = 0; i < w; ++i) xw[i] = zw[i] = 0;
        for (uint32_t q = 0; q < nqubits; ++q) {
            uint8_t c = codes[t * nqubits + q];
            uint64_t x, z;
            switch (c) {
            case 0: x = 0; z = 0; break;
            case 1: x = 1; z = 0; break;
            case 2: x = 1; z = 1; break;
            case 3: x = 0; z = 1; break;
            default: return OR_INVALID_CODE;
            }
            xw[q / 64] |= x << (q % 64);
            zw[q / 64] |= z << (q % 64);
        }
    }
    return OR_OK;
}

/* word.rs:227-237 */
static inline uint8_t code_at(const uint64_t *xw, const uint64_t *zw, uint32_t q) {
    uint64_t x = (xw[q / 64] >> (q % 64)) & 1u;
    uint64_t z = (zw[q / 64] >> (q % 64)) & 1u;
    if (!x && !z) return 0;
    if (x && !z) return 1;
    if (x && z) return 2;
    return 3;
}

/* Ord for PauliWord (word.rs:240-254): lexicographic in qubit order on codes. */
static int word_cmp(uint32_t n, const uint64_t *xa, const uint64_t *za,
                    const uint64_t *xb, const uint64_t *zb) {
    for (uint32_t q = 0; q < n; ++q) {
        uint8_t a = code_at(xa, za, q), b = code_at(xb, zb, q);
        if (a != b) return a < b ? -1 : 1;
    }
    return 0;
}

typedef struct {
    uint32_t n, w;
    const uint64_t *xw, *zw;
    const double *coeffs; /* interleaved re, im */
} canon_ctx;

static canon_ctx g_ctx; /* qsort has no context argument in C99 */

static uint64_t dbits(double v) {
    uint64_t b;
    memcpy(&b, &v, sizeof b);
    return b;
}

static int cmp_term_index(const void *pa, const void *pb) {
    uint64_t a = *(const uint64_t *)pa, b = *(const uint64_t *)pb;
    const canon_ctx *c = &g_ctx;
    int r = word_cmp(c->n, c->xw + a * c->w, c->zw + a * c->w, c->xw + b * c->w, c->zw + b * c->w);
    if (r) return r;
    /* operator.rs:141: duplicates are summed in ascending (re.to_bits(), im.to_bits()) order. */
    uint64_t ar = dbits(c->coeffs[2 * a]), br = dbits(c->coeffs[2 * b]);
    if (ar != br) return ar < br ? -1 : 1;
    uint64_t ai = dbits(c->coeffs[2 * a + 1]), bi = dbits(c->coeffs[2 * b + 1]);
    if (ai != bi) return ai < bi ? -1 : 1;
    return a < b ? -1 : (a > b); /* equal keys are equal values: order is immaterial */
}

/*
 * PauliOperator::from_terms (operator.rs:117-155): validate, group duplicate
 * words, sort words by the canonical order, sum each word's contributions in
 * IEEE-bit order starting from 0+0i, and drop exact zeros (scalar.rs:5-7).
 * Outputs are written to caller buffers of capacity `count`; *out_count gets
 * the canonical term count.  Not thread-safe (qsort context).
 */
int oracle_canonicalize(uint32_t nqubits, uint64_t count, const uint8_t *codes,
                        const double *coeffs, uint64_t *out_x, uint64_t *out_z,
                        double *out_coeffs, uint64_t *out_count, uint64_t *bad_index) {
    uint32_t w = oracle_packed_word_count(nqubits);
    for (uint64_t t = 0; t < count; ++t) {
        double re = coeffs[2 * t], im = coeffs[2 * t + 1];
        if (!(re - re == 0.0) || !(im - im == 0.0)) { /* !is_finite */
            if (bad_index) *bad_index = t;
            return OR_NON_FINITE_COEFFICIENT;
        }
        for (uint32_t q = 0; q < nqubits; ++q) {
            if (codes[t * nqubits + q] > 3) {
                if (bad_index) *bad_index = q;
                return OR_INVALID_CODE;
            }
        }
    }
    uint64_t *xw = (uint64_t *)malloc(sizeof(uint64_t) * (count * w + 1));
    uint64_t *zw = (uint64_t *)malloc(sizeof(uint64_t) * (count * w + 1));
    uint64_t *idx = (uint64_t *)malloc(sizeof(uint64_t) * (count + 1));
    if (!xw || !zw || !idx) {
        free(xw); free(zw); free(idx);
        return OR_ALLOC;
    }
    oracle_encode_codes(nqubits, count, codes, xw, zw);
    for (uint64_t t = 0; t < count; ++t) idx[t] = t;
    g_ctx.n = nqubits; g_ctx.w = w; g_ctx.xw = xw; g_ctx.zw = zw; g_ctx.coeffs = coeffs;
    qsort(idx, count, sizeof(uint64_t), cmp_term_index);
    uint64_t out = 0;
    uint64_t i = 0;
    while (i < count) {
        uint64_t j = i;
        cplx sum = {0.0, 0.0};
        while (j < count && word_cmp(nqubits, xw + idx[i] * w, zw + idx[i] * w,
                                     xw + idx[j] * w, zw + idx[j] * w) == 0) {
            cplx v = {coeffs[2 * idx[j]], coeffs[2 * idx[j] + 1]};
            sum = c_add(sum, v);
            ++j;
        }
        if (!(sum.re == 0.0 && sum.im == 0.0)) {
            for (uint32_t k = 0; k < w; ++k) {
                out_x[out * w + k] = xw[idx[i] * w + k];
                out_z[out * w + k] = zw[idx[i] * w + k];
            }
            out_coeffs[2 * out] = sum.re;
            out_coeffs[2 * out + 1] = sum.im;
            ++out;
        }
        i = j;
    }
    *out_count = out;
    free(xw); free(zw); free(idx);
    return OR_OK;
}

/*
 * StatevectorPauliAction::from_packed (pauli_action.rs:24-88) followed by
 * matrix_term (hamiltonian.rs:564-571): qubit q maps to matrix bit
 * 1 << (n-1-q); weighted_phase = coefficient * (i^(#Y mod 4) * 1.0).
 */
int oracle_matrix_terms(uint32_t nqubits, uint64_t count, const uint64_t *x_words,
                        const uint64_t *z_words, const double *coeffs,
                        uint64_t *x_mask, uint64_t *z_mask, double *weighted) {
    if (nqubits >= 64) return OR_OVERFLOW;
    uint32_t w = oracle_packed_word_count(nqubits);
    for (uint64_t t = 0; t < count; ++t) {
        uint64_t xm = 0, zm = 0;
        uint32_t ny = 0;
        for (uint32_t q = 0; q < nqubits; ++q) {
            uint64_t packed = 1ull << (q % 64);
            int x = (x_words[t * w + q / 64] & packed) != 0;
            int z = (z_words[t * w + q / 64] & packed) != 0;
            uint64_t mm = 1ull << (nqubits - 1 - q);
            if (x) xm |= mm;
            if (z) zm |= mm;
            if (x && z) ny += 1;
        }
        cplx yp;
        switch (ny % 4) {
        case 0: yp.re = 1.0; yp.im = 0.0; break;
        case 1: yp.re = 0.0; yp.im = 1.0; break;
        case 2: yp.re = -1.0; yp.im = 0.0; break;
        default: yp.re = 0.0; yp.im = -1.0; break;
        }
        /* `y_phase * sign` with sign = 1.0 (Complex * f64 scales both parts). */
        yp.re = yp.re * 1.0;
        yp.im = yp.im * 1.0;
        cplx c = {coeffs[2 * t], coeffs[2 * t + 1]};
        cplx wp = c_mul(c, yp);
        x_mask[t] = xm;
        z_mask[t] = zm;
        weighted[2 * t] = wp.re;
        weighted[2 * t + 1] = wp.im;
    }
    return OR_OK;
}

static inline int parity64(uint64_t v) { return __builtin_popcountll(v) & 1; }

/*
 * MvpPlan::apply_into, TermDirect strategy (hamiltonian.rs:204-270, default
 * lazy plan).  For every row: value = 0; for each term in canonical order,
 * column = row ^ x_mask, contribution = weighted_phase * state[column],
 * negated when popcount(z_mask & column) is odd; output overwritten.
 * Rows run in parallel (OpenMP in place of rayon) when work >= 1 << 16; the
 * per-row arithmetic is identical either way.
 */
int oracle_apply_term_direct(uint32_t nqubits, uint64_t count, const uint64_t *x_mask,
                             const uint64_t *z_mask, const double *weighted,
                             const double *state, double *result, int threads) {
    if (nqubits >= 64) return OR_OVERFLOW;
    uint64_t dim = 1ull << nqubits;
    const cplx *x = (const cplx *)state;
    cplx *y = (cplx *)result;
    const cplx *wp = (const cplx *)weighted;
    uint64_t work = count * dim;
    int par = work >= (1ull << 16);
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(threads) if (par)
#endif
    for (int64_t row = 0; row < (int64_t)dim; ++row) {
        cplx value = {0.0, 0.0};
        for (uint64_t t = 0; t < count; ++t) {
            uint64_t column = (uint64_t)row ^ x_mask[t];
            cplx contribution = c_mul(wp[t], x[column]);
            if (parity64(z_mask[t] & column)) contribution = c_neg(contribution);
            value = c_add(value, contribution);
        }
        y[row] = value;
    }
    (void)par;
    (void)threads;
    return OR_OK;
}

/*
 * Row-sampled TermDirect: the same per-row arithmetic as above for the listed
 * rows only (for state sizes whose full CPU MVP is too slow to run).
 */
int oracle_apply_rows(uint32_t nqubits, uint64_t count, const uint64_t *x_mask,
                      const uint64_t *z_mask, const double *weighted, const double *state,
                      uint64_t nrows, const uint64_t *rows, double *result, int threads) {
    if (nqubits >= 64) return OR_OVERFLOW;
    const cplx *x = (const cplx *)state;
    cplx *y = (cplx *)result;
    const cplx *wp = (const cplx *)weighted;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(threads)
#endif
    for (int64_t i = 0; i < (int64_t)nrows; ++i) {
        uint64_t row = rows[i];
        cplx value = {0.0, 0.0};
        for (uint64_t t = 0; t < count; ++t) {
            uint64_t column = row ^ x_mask[t];
            cplx contribution = c_mul(wp[t], x[column]);
            if (parity64(z_mask[t] & column)) contribution = c_neg(contribution);
            value = c_add(value, contribution);
        }
        y[i] = value;
    }
    (void)threads;
    return OR_OK;
}

/* group_matrix_terms (hamiltonian.rs:573-582): BTreeMap by x_mask, so groups
 * come out in ascending x_mask order with terms in canonical order inside. */
static int cmp_u64_pair(const void *pa, const void *pb) {
    const uint64_t *a = (const uint64_t *)pa, *b = (const uint64_t *)pb;
    if (a[0] != b[0]) return a[0] < b[0] ? -1 : 1;
    if (a[1] != b[1]) return a[1] < b[1] ? -1 : 1;
    return 0;
}

/* Returns the number of groups; fills order[] (term indices, grouped, stable)
 * and group_begin[G+1]. */
static uint64_t group_terms(uint64_t count, const uint64_t *x_mask, uint64_t *order,
                            uint64_t *group_begin) {
    uint64_t *pairs = (uint64_t *)malloc(sizeof(uint64_t) * 2 * (count + 1));
    for (uint64_t t = 0; t < count; ++t) {
        pairs[2 * t] = x_mask[t];
        pairs[2 * t + 1] = t;
    }
    qsort(pairs, count, 2 * sizeof(uint64_t), cmp_u64_pair);
    uint64_t g = 0;
    for (uint64_t t = 0; t < count; ++t) {
        order[t] = pairs[2 * t + 1];
        if (t == 0 || pairs[2 * t] != pairs[2 * t - 2]) group_begin[g++] = t;
    }
    group_begin[g] = count;
    free(pairs);
    return g;
}

/* Number of distinct x masks (BTreeSet size, hamiltonian.rs:86-90). */
uint64_t oracle_group_count(uint64_t count, const uint64_t *x_mask) {
    if (count == 0) return 0;
    uint64_t *order = (uint64_t *)malloc(sizeof(uint64_t) * (count + 1));
    uint64_t *gb = (uint64_t *)malloc(sizeof(uint64_t) * (count + 2));
    uint64_t g = group_terms(count, x_mask, order, gb);
    free(order);
    free(gb);
    return g;
}

/* Fill one group's diagonal: hamiltonian.rs:123-133. */
static void fill_diagonal(uint64_t dim, uint64_t b, uint64_t e, const uint64_t *order,
                          const uint64_t *z_mask, const cplx *wp, cplx *diag) {
    for (uint64_t column = 0; column < dim; ++column) {
        cplx value = {0.0, 0.0};
        for (uint64_t i = b; i < e; ++i) {
            uint64_t t = order[i];
            cplx contribution = wp[t];
            if (parity64(z_mask[t] & column)) contribution = c_neg(contribution);
            value = c_add(value, contribution);
        }
        diag[column] = value;
    }
}

/*
 * MvpPlan::from_operator_reusable + apply_into, XMaskDiagonal strategy
 * (hamiltonian.rs:79-147, 233-235): one precomputed 2^n diagonal per x mask,
 * then y[row] = sum over groups (ascending x_mask) of D_m[row^m] * x[row^m].
 * Needs G * 2^n * 16 bytes; only for small n.  *transitions receives the
 * eager transition_count (hamiltonian.rs:166-179) when non-null.
 */
int oracle_apply_xmask_diagonal(uint32_t nqubits, uint64_t count, const uint64_t *x_mask,
                                const uint64_t *z_mask, const double *weighted,
                                const double *state, double *result, uint64_t *transitions,
                                int threads) {
    if (nqubits >= 64) return OR_OVERFLOW;
    uint64_t dim = 1ull << nqubits;
    const cplx *x = (const cplx *)state;
    cplx *y = (cplx *)result;
    const cplx *wp = (const cplx *)weighted;
    uint64_t *order = (uint64_t *)malloc(sizeof(uint64_t) * (count + 1));
    uint64_t *gb = (uint64_t *)malloc(sizeof(uint64_t) * (count + 2));
    uint64_t groups = count ? group_terms(count, x_mask, order, gb) : 0;
    cplx *diag = (cplx *)malloc(sizeof(cplx) * (groups * dim + 1));
    uint64_t *gmask = (uint64_t *)malloc(sizeof(uint64_t) * (groups + 1));
    if (!order || !gb || !diag || !gmask) {
        free(order); free(gb); free(diag); free(gmask);
        return OR_ALLOC;
    }
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic) num_threads(threads)
#endif
    for (int64_t g = 0; g < (int64_t)groups; ++g) {
        gmask[g] = x_mask[order[gb[g]]];
        fill_diagonal(dim, gb[g], gb[g + 1], order, z_mask, wp, diag + (uint64_t)g * dim);
    }
    if (transitions) {
        uint64_t nz = 0;
        for (uint64_t i = 0; i < groups * dim; ++i)
            if (diag[i].re != 0.0 || diag[i].im != 0.0) ++nz;
        *transitions = nz;
    }
    uint64_t work = groups * dim;
    int par = work >= (1ull << 16);
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(threads) if (par)
#endif
    for (int64_t row = 0; row < (int64_t)dim; ++row) {
        cplx value = {0.0, 0.0};
        for (uint64_t g = 0; g < groups; ++g) {
            uint64_t column = (uint64_t)row ^ gmask[g];
            value = c_add(value, c_mul(diag[g * dim + column], x[column]));
        }
        y[row] = value;
    }
    (void)par;
    free(order); free(gb); free(diag); free(gmask);
    return OR_OK;
}

/* Eager transition count without applying (hamiltonian.rs:166-179). */
int oracle_transition_count(uint32_t nqubits, uint64_t count, const uint64_t *x_mask,
                            const uint64_t *z_mask, const double *weighted,
                            uint64_t *transitions, int threads) {
    if (nqubits >= 64) return OR_OVERFLOW;
    uint64_t dim = 1ull << nqubits;
    const cplx *wp = (const cplx *)weighted;
    uint64_t *order = (uint64_t *)malloc(sizeof(uint64_t) * (count + 1));
    uint64_t *gb = (uint64_t *)malloc(sizeof(uint64_t) * (count + 2));
    uint64_t groups = count ? group_terms(count, x_mask, order, gb) : 0;
    uint64_t total = 0;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic) num_threads(threads) reduction(+ : total)
#endif
    for (int64_t g = 0; g < (int64_t)groups; ++g) {
        uint64_t nz = 0;
        for (uint64_t column = 0; column < dim; ++column) {
            cplx value = {0.0, 0.0};
            for (uint64_t i = gb[g]; i < gb[g + 1]; ++i) {
                uint64_t t = order[i];
                cplx contribution = wp[t];
                if (parity64(z_mask[t] & column)) contribution = c_neg(contribution);
                value = c_add(value, contribution);
            }
            if (value.re != 0.0 || value.im != 0.0) ++nz;
        }
        total += nz;
    }
    *transitions = total;
    free(order);
    free(gb);
    (void)threads;
    return OR_OK;
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* PauliOperator::dense_matrix (hamiltonian.rs:313-355): row-major dense
 * matrix; every row walks the terms in canonical order and adds (or
 * subtracts) the weighted phase at column row ^ x_mask, the sign taken on the
 * column.  out: complex128[dim * dim], zeroed here. */
int oracle_dense(uint32_t nqubits, uint64_t count, const uint64_t *x_mask, const uint64_t *z_mask,
                 const double *weighted, double *out) {
    const uint64_t dim = 1ull << nqubits;
    memset(out, 0, sizeof(double) * 2 * dim * dim);
    for (uint64_t row = 0; row < dim; ++row) {
        double *o = out + 2 * row * dim;
        for (uint64_t t = 0; t < count; ++t) {
            const uint64_t column = row ^ x_mask[t];
            if (parity64(z_mask[t] & column)) {
                o[2 * column] -= weighted[2 * t];
                o[2 * column + 1] -= weighted[2 * t + 1];
            } else {
                o[2 * column] += weighted[2 * t];
                o[2 * column + 1] += weighted[2 * t + 1];
            }
        }
    }
    return 0;
}

typedef struct {
    uint64_t column;
    double re, im;
} sparse_entry;

static int entry_cmp(const void *a, const void *b) {
    const sparse_entry *x = a, *y = b;
    return x->column < y->column ? -1 : (x->column > y->column ? 1 : 0);
}

/* sparse_entries / fill_sparse_row (hamiltonian.rs:584-752): per row, one
 * entry per x-mask group (groups ascending by mask) whose value -- the group's
 * weighted phases summed from 0 in canonical order with the column's signs --
 * is not exactly zero, sorted by column.  Call with capacity 0 for *nnz;
 * indptr has dim + 1 entries. */
int oracle_csr(uint32_t nqubits, uint64_t count, const uint64_t *x_mask, const uint64_t *z_mask,
               const double *weighted, uint64_t *indptr, uint64_t *columns, double *values, uint64_t capacity,
               uint64_t *nnz) {
    const uint64_t dim = 1ull << nqubits;
    uint64_t *order = malloc(sizeof(uint64_t) * (count + 1));
    uint64_t *gstart = malloc(sizeof(uint64_t) * (count + 1));
    const uint64_t groups = group_terms(count, x_mask, order, gstart);
    sparse_entry *row_entries = malloc(sizeof(sparse_entry) * (groups + 1));
    uint64_t total = 0;
    indptr[0] = 0;
    for (uint64_t row = 0; row < dim; ++row) {
        uint64_t m = 0;
        for (uint64_t gi = 0; gi < groups; ++gi) {
            const uint64_t column = row ^ x_mask[order[gstart[gi]]];
            double re = 0.0, im = 0.0;
            for (uint64_t i = gstart[gi]; i < gstart[gi + 1]; ++i) {
                const uint64_t t = order[i];
                double cr = weighted[2 * t], ci = weighted[2 * t + 1];
                if (parity64(z_mask[t] & column)) {
                    cr = -cr;
                    ci = -ci;
                }
                re = re + cr;
                im = im + ci;
            }
            if (re != 0.0 || im != 0.0) {
                row_entries[m].column = column;
                row_entries[m].re = re;
                row_entries[m].im = im;
                ++m;
            }
        }
        qsort(row_entries, m, sizeof(sparse_entry), entry_cmp);
        if (capacity) {
            for (uint64_t e = 0; e < m && total + e < capacity; ++e) {
                columns[total + e] = row_entries[e].column;
                values[2 * (total + e)] = row_entries[e].re;
                values[2 * (total + e) + 1] = row_entries[e].im;
            }
        }
        total += m;
        indptr[row + 1] = total;
    }
    *nnz = total;
    free(row_entries);
    free(gstart);
    free(order);
    return 0;
}
