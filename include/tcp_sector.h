/*
 * tcp_sector.h -- C ABI of the fixed-Hamming-weight (U(1)) sector MVP in
 * `libtcpmvp.so`.
 *
 * A U(1) sector of n qubits and particle number k holds the C(n, k)
 * computational basis states with exactly k ones, in ascending TensorCircuit
 * integer order (qubit 0 is the most significant bit), the ordering of
 * `U1Sector::unrank` (crates/tencir-pauli-core/src/sector.rs:169-238 in the
 * reference).  A sector plan applies a number-conserving Pauli operator to a
 * restricted state of length C(n, k):
 *
 *   y[r] = sum over x-groups m with popcount(b_r ^ m) == k of
 *          v_m(b_r ^ m) * x[rank(b_r ^ m)],
 *   v_m(s) = sum_{terms t of m} c_t i^{#Y_t} (-1)^{popcount(z_t & s)},
 *
 * the destination-major form of `aggregate_source` (sector.rs:1051-1127).
 * The device plan covers n <= 256 (states of up to four 64-bit words); the
 * host rank, unrank and basis entries take any n.  Status codes are those of
 * tcp_mvp.h, plus the two PauliError variants of this path.
 */
#ifndef TCP_SECTOR_H
#define TCP_SECTOR_H

#include <stddef.h>
#include <stdint.h>

#include "tcp_mvp.h"

#ifdef __cplusplus
extern "C" {
#endif

enum tcp_sector_status {
    TCP_ERR_SECTOR_LEAKAGE = 11, /* PauliError::SectorLeakage (error.rs:30-35) */
    TCP_ERR_INVALID_INDEX = 13   /* PauliError::InvalidIndex (error.rs:38-39) */
};

typedef struct tcp_u1_plan tcp_u1_plan;

typedef struct tcp_u1_plan_info_t {
    uint32_t nqubits;
    uint32_t particle_number;
    uint64_t dimension;        /* C(n, k) */
    uint64_t term_count;       /* canonical terms held by the plan */
    uint64_t group_count;      /* distinct x masks */
    int32_t storage;           /* enum tcp_storage */
    int32_t device;            /* CUDA ordinal the plan lives on */
    int64_t transition_count;  /* eager nonzero count, -1 for lazy plans (None) */
    uint64_t device_bytes;     /* device memory retained by the plan */
    uint64_t estimated_bytes;  /* the reference's retained-size estimate (sector.rs:1208-1292) */
    uint32_t complement;       /* 1 when ranks run over the n - k holes (k > n - k) */
    uint32_t rank_chunks;      /* 8-bit chunks of one rank lookup */
    uint32_t tables_in_shared; /* 1 when rank tables, groups and terms are staged in shared memory */
    uint32_t reserved;
} tcp_u1_plan_info_t;

/* C(n, k) as U1Sector::new computes it (sector.rs:79-99, choose_u64 :1342-1362).
 * TCP_ERR_INVALID_SECTOR when k > n, TCP_ERR_OVERFLOW past uint64. */
int tcp_u1_dimension(uint32_t nqubits, uint32_t particle_number, uint64_t *out_dimension);

/* U1Sector::rank_words (sector.rs:141-167): rank of one packed occupation word
 * (qubit q at word q/64, bit q%64; `word_count` words).  Any n. */
int tcp_u1_rank_words(uint32_t nqubits, uint32_t particle_number, const uint64_t *words,
                      uint32_t word_count, uint64_t *out_rank);

/* U1Sector::unrank_into (sector.rs:184-238): packed occupation words of a
 * restricted index.  Any n. */
int tcp_u1_unrank_words(uint32_t nqubits, uint32_t particle_number, uint64_t index, uint64_t *out_words,
                        uint32_t word_count);

/* U1Sector::basis_words_packed (sector.rs:241-265) and the PyO3 entry
 * `u1_basis_words` (crates/tencirpauli-native/src/symmetry.rs:395-436): for
 * n <= 64 one TensorCircuit integer per state, else `word_count` packed words
 * per state.  `capacity` is in uint64 elements; max_bytes bounds the output. */
int tcp_u1_basis_words(uint32_t nqubits, uint32_t particle_number, uint64_t *out, uint64_t capacity,
                       uint64_t max_bytes);

/*
 * Number-charge conservation of a canonical operator: the selection rule of
 * PauliOperator::analyze_charge (crates/tencir-pauli-core/src/operator.rs:396-444)
 * for qubit levels (0, 1), which `_restrict_u1` (python/tencirpauli/symmetry.py,
 * lazy storage) calls before it builds a lazy plan.  *out_nonzero receives
 * the number of nonzero aggregated commutator words; the operator conserves
 * the particle number iff it is 0.  Any n.
 */
int tcp_pauli_number_commutator(uint32_t nqubits, uint64_t term_count, uint32_t word_count,
                                const uint64_t *x_words, const uint64_t *z_words, const double *coefficients,
                                uint64_t *out_nonzero);

/*
 * Build a sector plan on the current CUDA device from a canonical operator
 * (same arrays as tcp_mvp_plan_create).  Replaces U1LazyMvpPlan::new
 * (storage LAZY, sector.rs:515-534) and U1RestrictedOperator::new (storage
 * EAGER, sector.rs:345-431), reached from the PyO3 entries
 * `pauli_restrict_u1_lazy_handle` / `pauli_restrict_u1_handle`
 * (crates/tencirpauli-native/src/symmetry.rs:370-393).
 *  - LAZY: max_bytes bounds the compiled-term estimate.
 *  - EAGER: max_bytes bounds the reference's construction estimate and the
 *    transition count is computed.
 * Both scan every source for leakage: a group whose destination leaves the
 * sector must aggregate to exactly zero (TCP_ERR_SECTOR_LEAKAGE names the
 * lowest leaking source index, as the reference's ascending scan does; the
 * reference's lazy plan reports the same error from its first apply).
 */
int tcp_u1_plan_create(uint32_t nqubits, uint32_t particle_number, uint64_t term_count, uint32_t word_count,
                       const uint64_t *x_words, const uint64_t *z_words, const double *coefficients,
                       int storage, uint64_t max_bytes, tcp_u1_plan **out_plan);

int tcp_u1_plan_destroy(tcp_u1_plan *plan);
int tcp_u1_plan_info(const tcp_u1_plan *plan, tcp_u1_plan_info_t *info);

/* U1MvpPlan::apply_into / U1LazyMvpPlan::apply_into (sector.rs:579-643,681-691):
 * host complex128 buffers of length C(n, k), blocking, output overwritten. */
int tcp_u1_apply_into_host(const tcp_u1_plan *plan, const double *state, uint64_t state_len, double *result,
                           uint64_t result_len, uint64_t max_bytes);

/* Device buffers: nrhs contiguous vectors of `len` elements, dtype
 * enum tcp_dtype, stream-ordered on `stream` (a cudaStream_t). */
int tcp_u1_apply_into_device(const tcp_u1_plan *plan, const void *d_state, void *d_result, uint64_t len,
                             uint32_t nrhs, int dtype, void *stream);

/* Diagonal of the restricted operator (complex128, len C(n, k)). */
int tcp_u1_diagonal_device(const tcp_u1_plan *plan, void *d_diag, uint64_t len, void *stream);

/* Nonzero entries of the restricted matrix (the eager transition count). */
int tcp_u1_transition_count(const tcp_u1_plan *plan, uint64_t *out_count);

/*
 * Restricted CSR arrays (U1RestrictedOperator::csr, sector.rs:509-511 and
 * :699-730): rows are destinations, columns ascending inside a row, values
 * the aggregated group values.  indptr: uint64[dimension + 1]; columns:
 * uint64[capacity]; values: complex128[capacity] as doubles.  *out_nnz
 * receives the entry count; TCP_ERR_MEMORY_LIMIT when capacity is short.
 */
int tcp_u1_csr(const tcp_u1_plan *plan, uint64_t *indptr, uint64_t *columns, double *values, uint64_t capacity,
               uint64_t *out_nnz);

/* Sticky device status of the plan (TCP_ERR_DEVICE_TIMEOUT is never set by
 * the sector kernels; CUDA errors are reported). */
int tcp_u1_plan_device_status(const tcp_u1_plan *plan);

#ifdef __cplusplus
}
#endif

#endif /* TCP_SECTOR_H */
