/*
 * tcp_matrix.h -- dense, COO and CSR materialisation of a full-space plan in
 * `libtcpmvp.so` (the reference's `PauliOperator.dense()`, `.coo()`, `.csr()`:
 * python/tencirpauli/pauli.py:866-930 over
 * crates/tencir-pauli-core/src/hamiltonian.rs:311-478,584-770).
 *
 * Entries come from the plan's x-mask groups (ascending mask): row r and
 * group m give column r ^ m with the value sum_{k in m} c_k i^{#Y_k}
 * (-1)^{popcount(z_k & column)}, summed from 0 in canonical term order.  Dense
 * output keeps every group value (exact zeros included); COO/CSR skip exact
 * zeros and order the columns of a row ascending; rows ascend.  The budget
 * checks are the reference's (TCP_ERR_MEMORY_LIMIT, "requested R bytes
 * exceeds memory limit L").
 */
#ifndef TCP_MATRIX_H
#define TCP_MATRIX_H

#include <stdint.h>

#include "tcp_mvp.h"

#ifdef __cplusplus
extern "C" {
#endif

enum tcp_matrix_target {
    TCP_MATRIX_COO = 0, /* budget of PauliOperator::coo_matrix (hamiltonian.rs:358-414) */
    TCP_MATRIX_CSR = 1  /* budget of PauliOperator::csr_matrix (hamiltonian.rs:417-478) */
};

/* Row-major complex128 dense matrix (dimension^2 elements, interleaved
 * doubles) into host memory; capacity in complex elements.  Budget:
 * dimension^2 * 16 bytes against max_bytes (hamiltonian.rs:313-320). */
int tcp_mvp_dense(const tcp_mvp_plan *plan, double *out, uint64_t capacity, uint64_t max_bytes);

/* Entry count of the sparse targets (nonzero group values over all rows),
 * after the target's budget check. */
int tcp_mvp_sparse_count(const tcp_mvp_plan *plan, int target, uint64_t max_bytes, uint64_t *out_nnz);

/* CSR arrays into host memory: indptr uint64[dimension + 1], columns
 * uint64[capacity], values complex128[capacity] (interleaved doubles).
 * COO rows are indptr expanded.  *out_nnz receives the entry count;
 * TCP_ERR_INVALID_ARGUMENT when capacity is short. */
int tcp_mvp_csr(const tcp_mvp_plan *plan, int target, uint64_t max_bytes, uint64_t *indptr, uint64_t *columns,
                double *values, uint64_t capacity, uint64_t *out_nnz);

#ifdef __cplusplus
}
#endif

#endif /* TCP_MATRIX_H */
