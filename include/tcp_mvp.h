/*
 * tcp_mvp.h -- C ABI of the B200 (sm_100a) matrix-free Pauli MVP library
 * `libtcpmvp.so`.
 *
 * The library computes y = sum_k c_k P_k x over a 2^n complex statevector for
 * a canonical Pauli operator, the path behind TenCirPauli's
 * `PauliOperator.native_mvp_plan()` / `.mvp()`.  Every entry point returns an
 * `int` status (TCP_OK == 0) and never aborts; `tcp_last_error` returns the
 * calling thread's last message.  No torch or CUDA-runtime C++ types appear in
 * the signatures: CUDA streams travel as `void*` (a `cudaStream_t`).
 *
 * Conventions (identical to the reference, paths inside the reference project):
 *  - packed words: qubit q is bit q%64 of word q/64
 *    (crates/tencir-pauli-core/src/word.rs:94-110);
 *  - codes 0=I 1=X 2=Y 3=Z (word.rs:296-304);
 *  - state index: qubit 0 is the most significant bit, matrix bit of qubit q
 *    is 1 << (n-1-q) (crates/tencir-pauli-core/src/pauli_action.rs:65);
 *  - y[r] = sum_k c_k i^{#Y_k} (-1)^{popcount(z_k & (r ^ x_k))} x[r ^ x_k]
 *    (crates/tencir-pauli-core/src/hamiltonian.rs:238-243);
 *  - complex128 buffers are interleaved (re, im) doubles, complex64 buffers
 *    interleaved floats.
 */
#ifndef TCP_MVP_H
#define TCP_MVP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TCP_ABI_VERSION 1

/* Status codes.  1..10 mirror the PauliError variants used on this path
 * (crates/tencir-pauli-core/src/error.rs:5-74), in declaration order. */
enum tcp_status {
    TCP_OK = 0,
    TCP_ERR_INVALID_CODE = 1,             /* PauliError::InvalidCode */
    TCP_ERR_INVALID_WORD_LENGTH = 2,      /* PauliError::InvalidWordLength */
    TCP_ERR_INCOMPATIBLE_QUBITS = 3,      /* PauliError::IncompatibleQubitCounts */
    TCP_ERR_INVALID_STRUCTURE_LENGTH = 4, /* PauliError::InvalidStructureLength */
    TCP_ERR_NON_FINITE_COEFFICIENT = 5,   /* PauliError::NonFiniteCoefficient */
    TCP_ERR_NON_CANONICAL_TERMS = 7,      /* PauliError::NonCanonicalTerms */
    TCP_ERR_OVERFLOW = 8,                 /* PauliError::Overflow */
    TCP_ERR_MEMORY_LIMIT = 9,             /* PauliError::MemoryLimit */
    TCP_ERR_INVALID_SECTOR = 10,          /* PauliError::InvalidSector (bad storage label) */
    /* Library-specific statuses. */
    TCP_ERR_INVALID_ARGUMENT = 32, /* null pointer, bad enum, overlapping buffers */
    TCP_ERR_CUDA = 33,             /* a CUDA runtime call failed */
    TCP_ERR_DEVICE_TIMEOUT = 34,   /* a bounded device-side wait expired */
    TCP_ERR_ALLOCATION = 35,       /* device or host allocation failed */
    TCP_ERR_WRONG_DEVICE = 36      /* plan used on a device other than its own */
};

enum tcp_storage {
    TCP_STORAGE_LAZY = 0, /* MvpStrategy::TermDirect label (hamiltonian.rs:63-76) */
    TCP_STORAGE_EAGER = 1 /* MvpStrategy::XMaskDiagonal label (hamiltonian.rs:79-147) */
};

enum tcp_dtype {
    TCP_DTYPE_C128 = 0, /* complex128 state, FP64 arithmetic */
    TCP_DTYPE_C64 = 1   /* complex64 state, FP32 products, Kahan sum over groups */
};

/* The calling thread's last status and the numeric fields of its PauliError
 * variant, so that a binding can rebuild the variant without parsing the
 * message of tcp_last_error (crates/tencir-pauli-core/src/error.rs:5-74):
 *   TCP_ERR_INVALID_CODE             fields = {code, index}
 *   TCP_ERR_INVALID_WORD_LENGTH,
 *   TCP_ERR_INVALID_STRUCTURE_LENGTH fields = {expected, actual}
 *   TCP_ERR_NON_FINITE_COEFFICIENT   fields = {index, 0}
 *   TCP_ERR_MEMORY_LIMIT             fields = {requested, limit} (requested
 *                                    saturates at 2^64 - 1)
 *   TCP_ERR_SECTOR_LEAKAGE (11)      fields = {source_index, actual}; the
 *                                    expected weight is the sector's k
 * Other statuses carry no fields (both 0).  Returns the last status (0 when
 * the thread has had no error). */
int tcp_last_error_fields(uint64_t fields[2]);

/* Opaque, immutable-after-create plan.  Thread-safe for concurrent apply. */
typedef struct tcp_mvp_plan tcp_mvp_plan;

typedef struct tcp_mvp_plan_info_t {
    uint32_t nqubits;
    uint32_t word_count;
    uint64_t dimension;        /* 2^n */
    uint64_t term_count;       /* canonical terms held by the plan */
    uint64_t group_count;      /* distinct x masks */
    int32_t storage;           /* enum tcp_storage */
    int32_t device;            /* CUDA ordinal the plan lives on */
    int64_t transition_count;  /* eager nonzero count, -1 for lazy plans (None) */
    uint64_t device_bytes;     /* device memory retained by the plan */
    uint32_t tile_bits;        /* log2 rows of one tile of the tiled kernel */
    uint32_t log_threads;      /* log2 threads per tile (rows per thread = 2^(tile_bits - log_threads)) */
    uint64_t steps;            /* tile loads per output tile (outer patterns, split at 16 KiB of term data) */
    uint64_t outer_patterns;   /* distinct outer patterns d = x_mask >> tile_bits */
    uint64_t ring_steps;       /* tile loads per output tile of the ring kernel (0: not used) */
    uint64_t cosets;           /* operand loads per output tile of the ring kernel (groups sharing them) */
} tcp_mvp_plan_info_t;

/* Library version (TCP_ABI_VERSION) */
int tcp_abi_version(void);

/* Copy the calling thread's last error message (NUL-terminated, truncated to
 * `capacity`).  Returns the full message length. */
size_t tcp_last_error(char *buffer, size_t capacity);

/*
 * Canonicalize a term batch: replaces PauliOperator::from_terms
 * (crates/tencir-pauli-core/src/operator.rs:117-155) and the PyO3 entry
 * `pauli_operator_native_array` (crates/tencirpauli-native/src/operator.rs:205-243).
 * codes: uint8[count * nqubits] (0..3); coefficients: double[2*count] (re, im).
 * Duplicate words are summed in ascending (re bits, im bits) order from 0+0i,
 * exact zeros are dropped, words are sorted by their code tuple.
 * Outputs (capacity `count` terms): out_x/out_z uint64[count * word_count],
 * out_coefficients double[2*count]; *out_count receives the canonical count.
 * On TCP_ERR_INVALID_CODE / TCP_ERR_NON_FINITE_COEFFICIENT, *bad_index (if
 * non-null) receives the offending qubit / term index.
 */
int tcp_pauli_canonicalize(uint32_t nqubits, uint64_t count, const uint8_t *codes,
                           const double *coefficients, uint64_t *out_x, uint64_t *out_z,
                           double *out_coefficients, uint64_t *out_count, uint64_t *bad_index);

/*
 * Build a plan on the current CUDA device.  Replaces MvpPlan::from_operator
 * (storage LAZY, hamiltonian.rs:63-76) and MvpPlan::from_operator_reusable
 * (storage EAGER, hamiltonian.rs:79-147), reached from the PyO3 entry
 * `pauli_mvp_plan_handle` (crates/tencirpauli-native/src/hamiltonian.rs:98-116).
 * x_words / z_words: uint64[term_count * word_count], coefficients:
 * double[2*term_count]; the term list is the canonical operator's.
 * max_bytes is the reference's eager construction budget (u128 there; here
 * UINT64_MAX means unlimited); lazy plans ignore it.
 */
int tcp_mvp_plan_create(uint32_t nqubits, uint64_t term_count, uint32_t word_count,
                        const uint64_t *x_words, const uint64_t *z_words,
                        const double *coefficients, int storage, uint64_t max_bytes,
                        tcp_mvp_plan **out_plan);

/* Release a plan and its device memory.  NULL is accepted. */
int tcp_mvp_plan_destroy(tcp_mvp_plan *plan);

/* Metadata: nqubits / term_count / transition_count mirror the getters of
 * MvpPlan (hamiltonian.rs:149-179) and the PyO3 NativeMvpPlan properties. */
int tcp_mvp_plan_info(const tcp_mvp_plan *plan, tcp_mvp_plan_info_t *info);

/*
 * Drop-in for MvpPlan::apply_into (hamiltonian.rs:204-270) and the PyO3
 * NativeMvpPlan.apply_into (crates/tencirpauli-native/src/hamiltonian.rs:176-193):
 * host complex128 buffers, blocking.  Copies `state` to the device, applies,
 * copies the result back and overwrites every element of `result`.
 * Lengths are in complex elements; a length other than 2^n returns
 * TCP_ERR_INVALID_STRUCTURE_LENGTH ("expected structure length E, got A").
 * max_bytes is accepted and ignored, as in the reference (hamiltonian.rs:223).
 * States of 2^25 or more amplitudes (8192 output tiles) are copied in
 * quarters, each followed by the kernel pass that reads it, and copied back
 * in chunks of output tiles while later chunks compute; page-locked host
 * buffers let the copies overlap the kernel.  The FP64 sums are then grouped
 * by quarter, so the result can differ from tcp_mvp_apply_into_device in the
 * last bits.  After TCP_ERR_DEVICE_TIMEOUT the contents of `result` are
 * undefined.
 */
int tcp_mvp_apply_into_host(const tcp_mvp_plan *plan, const double *state, uint64_t state_len,
                            double *result, uint64_t result_len, uint64_t max_bytes);

/* Same, complex64 host buffers (FP32 arithmetic with Kahan group sums). */
int tcp_mvp_apply_into_host_c64(const tcp_mvp_plan *plan, const float *state,
                                uint64_t state_len, float *result, uint64_t result_len);

/*
 * Device-resident apply, asynchronous on `stream` (a cudaStream_t, NULL for
 * the legacy default stream).  d_state / d_result hold `nrhs` vectors of
 * `len` == 2^n complex elements each, vector v at offset v * len.  dtype is
 * enum tcp_dtype.  Buffers must not overlap.  Device-side timeouts are
 * reported by tcp_mvp_plan_device_status after the stream is synchronised.
 */
int tcp_mvp_apply_into_device(const tcp_mvp_plan *plan, const void *d_state, void *d_result,
                              uint64_t len, uint32_t nrhs, int dtype, void *stream);
/* The same with d_result += H d_state instead of overwriting (no counterpart
 * in the reference, whose apply_into always overwrites): the shard-exchange
 * path adds every partner's contribution to its output shard this way. */
int tcp_mvp_apply_add_device(const tcp_mvp_plan *plan, const void *d_state, void *d_result,
                             uint64_t len, uint32_t nrhs, int dtype, void *stream);

/*
 * Batched MVP: many plans (Hamiltonians of uneven qubit and term counts), each
 * applied to a block of `nrhs` right-hand sides, replayed from one CUDA graph:
 * one persistent kernel launch, or (the ring configuration below) one
 * ring-kernel launch per member.  No counterpart in the reference (its
 * MvpPlan::apply_into, hamiltonian.rs:204-270, takes one state per call);
 * per vector the arithmetic is that of tcp_mvp_apply_into_device.
 * Buffers: d_x[h] / d_y[h] hold member h's nrhs vectors, RHS-major (vector v at
 * offset v * 2^n_h), complex128 or complex64 per `dtype`, 16-byte aligned.
 * Every member needs at least 8 qubits.  The batch keeps pointers to its plans,
 * which must outlive it.  Work items are (member, tile of 2^tile_rows_log2
 * rows, block of rhs_block vectors), largest member first.
 * The ring configuration (tile_rows_log2 = 12, rhs_block = 1; the default
 * when every member has at least 12 qubits) instead records one ring-kernel
 * launch per member with a term, over all its tiles and all nrhs vectors
 * (nrhs <= 65535), in the same graph; its graph captures the buffers, so it
 * is rebuilt when they change.  tcp_mvp_batch_info then reports the total
 * CTAs as `items` and the number of launches as `grid`.
 */
typedef struct tcp_mvp_batch tcp_mvp_batch;
int tcp_mvp_batch_create(uint32_t count, const tcp_mvp_plan *const *plans, uint32_t nrhs, int dtype,
                         tcp_mvp_batch **out_batch);
int tcp_mvp_batch_destroy(tcp_mvp_batch *batch);
/* Choose the tile rows (2^8..2^10) and RHS block (1, 2, 4, 8; divides nrhs),
 * or the ring configuration (12, 1). */
int tcp_mvp_batch_configure(tcp_mvp_batch *batch, uint32_t tile_rows_log2, uint32_t rhs_block);
/* Time every kernel variant on these buffers (`repeats` launches each) and keep
 * the fastest; with a non-empty cache_path the choice is read from / appended
 * to that file, keyed by device, dtype, nrhs and every member's (n, T, G). */
int tcp_mvp_batch_autotune(tcp_mvp_batch *batch, const void *const *d_x, void *const *d_y,
                           const char *cache_path, uint32_t repeats, void *stream);
/* y_h = H_h x_h for every member; asynchronous on `stream` (graph launch). */
int tcp_mvp_batch_apply(tcp_mvp_batch *batch, const void *const *d_x, void *const *d_y, void *stream);
int tcp_mvp_batch_info(const tcp_mvp_batch *batch, uint32_t *tile_rows_log2, uint32_t *rhs_block,
                       uint64_t *items, uint32_t *grid);
/* Synchronise and report (then clear) a device-side error of the batch. */
int tcp_mvp_batch_device_status(tcp_mvp_batch *batch);

/*
 * Allocation-free host apply.  This entry point has no counterpart in the
 * reference; it exists for callers that must not allocate device memory while
 * they apply, such as applications whose own allocator owns the GPU's memory
 * and forbids allocations behind its back, or services that reserve every
 * allocation at start-up and may not touch the allocator afterwards.
 * tcp_mvp_apply_into_host allocates a device workspace on its first call;
 * this variant calls no cudaMalloc/cudaFree (nor any allocating routine) and
 * instead stages the state and the result through one fixed device array that
 * is part of the library image: TCP_NOALLOC_MAX_QUBITS = 20, i.e. two vectors
 * of 2^20 complex128 (32 MiB + 256 bytes), which every GPU that loads the
 * library holds until the process exits.  Plans with more qubits are rejected
 * with TCP_ERR_MEMORY_LIMIT.  The plan itself must still be created
 * beforehand (tcp_mvp_plan_create allocates it).
 *  - The first call on a device looks up the array's device address
 *    (set-up); make that first call before any stream capture.
 *  - Every call shares the one array: calls that overlap on the GPU (from
 *    several host threads, or several streams) race and must be serialised
 *    by the caller.  The array keeps the last call's contents.
 *  - Runs on `stream` (a cudaStream_t, NULL for the legacy default stream) and
 *    returns after the result is in `result`.  Semantics otherwise equal
 *    tcp_mvp_apply_into_host (lengths, overwrite, errors).
 *  - When it returns TCP_ERR_DEVICE_TIMEOUT, `result` has been set to zero.
 */
#define TCP_NOALLOC_MAX_QUBITS 20
int tcp_mvp_apply_into_host_noalloc(const tcp_mvp_plan *plan, const double *state,
                                    uint64_t state_len, double *result, uint64_t result_len,
                                    void *stream);

/* Self-test of the bounded device waits (no counterpart in the reference): a
 * kernel waits, with a limit of `limit_ns` (at most 100 ms), on an mbarrier
 * that nothing completes, and reports the expiry through the plan's status
 * word.  Returns TCP_ERR_DEVICE_TIMEOUT when the wait gave up as designed. */
int tcp_selftest_bounded_wait(const tcp_mvp_plan *plan, uint64_t limit_ns);

/* Synchronise the plan's device and report (then clear) any device-side error
 * flag raised by kernels of this plan. */
int tcp_mvp_plan_device_status(const tcp_mvp_plan *plan);

/*
 * Eager transition count on the device: the number of nonzero entries of the
 * per-x-mask diagonals D_m[c] = sum_{k in m} w_k (-1)^{popcount(z_k & c)}
 * summed in canonical term order (hamiltonian.rs:121-139,166-179).
 */
int tcp_mvp_transition_count(const tcp_mvp_plan *plan, uint64_t *out_count);

/*
 * Diagonal extraction: writes H_ii (the x_mask == 0 group, complex128) for
 * every basis state into d_diag (2^n elements), asynchronous on `stream`.
 * Used by Jacobi-type preconditioners.
 */
int tcp_mvp_diagonal_device(const tcp_mvp_plan *plan, void *d_diag, uint64_t len, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* TCP_MVP_H */
