/*
 * tcp_solver.h -- eigensolver kernels of libtcpmvp.so built on the MVP
 * (include/tcp_mvp.h): FP64 block inner products and combinations over
 * complex64 / complex128 vector storage, per-basis-state features, the Jacobi
 * and learned (MLP) Davidson preconditioners, and the MLP training kernels.
 * No counterpart in the reference: TenCirPauli hands its MVP plan to SciPy's
 * `eigsh` (python/tencirpauli/integrations/scipy.py:13-49); these kernels
 * serve the Davidson solver in tencirpauli_b200/davidson.py.
 *
 * Vectors are RHS-major on the device (vector v at offset v * n), complex64
 * (dtype TCP_DTYPE_C64) or complex128 (TCP_DTYPE_C128); small matrices
 * (Gram blocks, coefficient blocks) are complex128, column-major, on the
 * device.  All calls are asynchronous on `stream` and return a tcp_status.
 */
#ifndef TCP_SOLVER_H
#define TCP_SOLVER_H

#include "tcp_mvp.h"

#ifdef __cplusplus
extern "C" {
#endif

#define TCP_FEATURES 8          /* floats per basis state from tcp_state_features */
#define TCP_MLP_IN 8            /* network inputs */
#define TCP_MLP_HIDDEN 16       /* width of both hidden layers */
#define TCP_MLP_PARAMS 433      /* 16*8 + 16 + 16*16 + 16 + 16 + 1 */
#define TCP_MLP_TRAIN_BLOCKS 296

/* Scratch bytes for tcp_gram with p and q vectors. */
size_t tcp_gram_work_bytes(uint32_t p, uint32_t q);

/* G = A^H B (p x q complex128, column-major), accumulated in FP64 with a
 * fixed-order (deterministic) reduction.  p + q <= 96, p * q <= 512. */
int tcp_gram(const void *A, int a_dtype, uint32_t p, const void *B, int b_dtype, uint32_t q, uint64_t n,
             void *d_G, void *d_work, void *stream);

/* out[:, j] = alpha * sum_i A[:, i] S[i, j] + beta * out[:, j] in FP64
 * arithmetic (S: p x k complex128 column-major on the device, k <= 32,
 * p * k <= 6144 after k is padded to the next of 4, 8, 16, 32). */
int tcp_block_combine(const void *A, int a_dtype, uint32_t p, const void *d_S, uint32_t k, uint64_t n,
                      double alpha, double beta, void *out, int out_dtype, void *stream);

/* Jacobi correction T[:, j] = -R[:, j] / (diag - theta_j), |diag - theta_j|
 * clamped below by eps.  diag: complex128 H_ii (tcp_mvp_diagonal_device);
 * d_theta: k doubles on the device. */
int tcp_precond_jacobi(const void *R, int r_dtype, uint64_t n, uint32_t k, const void *d_diag,
                       const double *d_theta, double eps, void *T, int t_dtype, void *stream);

/* TCP_FEATURES floats per basis state (independent of the Ritz value):
 * H_ii, mean and minimum H_jj over the states j the row couples to,
 * sum_j |H_ij|, sum_j |H_ij|^2, the number of couplings, Hamming weight / n
 * - 1/2, and 0 (padding). */
int tcp_state_features(const tcp_mvp_plan *plan, float *d_features, uint64_t n, void *stream);

/* Learned correction T[:, j] = -exp(c) R[:, j] / den with c the MLP output for
 * the state's features at Ritz value theta_j (clamped to [-clamp, clamp]) and
 * den = H_ii - theta_j from the complex128 diagonal d_diag, clamped by eps as
 * in tcp_precond_jacobi (c = 0 gives the Jacobi correction bit for bit).
 * `scale` normalises energies. */
int tcp_precond_mlp(const void *R, int r_dtype, uint64_t n, uint32_t k, const float *d_features,
                    const void *d_diag, const double *d_theta, double scale, double eps, float clamp,
                    const float *d_params, void *T, int t_dtype, void *stream);

/* Network inputs (count x TCP_MLP_IN) and denominators for training samples:
 * sample s is basis state d_rows[s] at Ritz value d_theta[d_which[s]]. */
int tcp_mlp_inputs(const float *d_features, const uint64_t *d_rows, const double *d_theta,
                   const uint32_t *d_which, uint32_t count, double scale, double eps, float *d_X,
                   float *d_den, void *stream);

/* Scratch bytes for tcp_mlp_train_step. */
size_t tcp_mlp_train_work_bytes(void);

/* One training step over `count` samples: loss sum_s wt (g^2 a - 2 g b + e2)
 * with g = -exp(c) / den; writes the summed gradient to d_grad_out (if
 * non-null) and the loss to d_loss_out (if non-null); with lr > 0 applies one
 * Adam step (beta1 0.9, beta2 0.999, eps 1e-8) to d_params using d_m, d_v and
 * the 1-based step number. */
int tcp_mlp_train_step(const float *d_X, const float *d_den, const float *d_a, const float *d_b,
                       const float *d_e2, const float *d_wt, uint32_t count, float *d_params, float *d_m,
                       float *d_v, float *d_work, float lr, uint32_t step, float *d_grad_out,
                       float *d_loss_out, void *stream);

/* Network output c for `count` input rows (count x TCP_MLP_IN floats). */
int tcp_mlp_forward(const float *d_X, uint32_t count, const float *d_params, float *d_out, void *stream);

/* Gradient of any loss from its derivatives dL/dc (d_dc, one per sample):
 * back-propagates through the network, writes the summed gradient to
 * d_grad_out (if non-null) and, with lr > 0, applies one Adam step. */
int tcp_mlp_backward_step(const float *d_X, const float *d_dc, uint32_t count, float *d_params, float *d_m,
                          float *d_v, float *d_work, float lr, uint32_t step, float *d_grad_out, void *stream);

/* Scratch bytes for tcp_mlp_alignment_grad: six doubles per training set. */
size_t tcp_mlp_alignment_work_bytes(uint32_t nsets);

/* Derivative of the alignment objective with respect to the network outputs.
 * Training set s covers states [d_seg_begin[s], d_seg_begin[s + 1]) (d_seg
 * holds each state's set index).  Per state: network output d_c, denominator
 * d_den (H_ii - theta), alpha = conj(e_i) r_i and gamma = conj(u_i) r_i
 * (complex128), a = |r_i|^2; per set: E = ||e||^2, with r the residual, u the
 * Ritz vector and e the direction Davidson is missing.  With
 * g = -exp(clamp(c)) / den, A = sum g alpha, B = sum g^2 a, C = sum g gamma,
 * the set's loss is 1 - |A|^2 / (E (B - |C|^2)), the objective their mean.
 * Writes dL/dc to d_dc (zero where the clamp is active) and, if d_loss is
 * non-null, the objective to d_loss[0].  Sums are reduced in a fixed order. */
int tcp_mlp_alignment_grad(const float *d_c, const float *d_den, const void *d_alpha, const double *d_a,
                           const void *d_gamma, const double *d_E, const int64_t *d_seg, const uint64_t *d_seg_begin,
                           uint32_t nsets, uint64_t count, float clamp, double *d_work, float *d_dc, double *d_loss,
                           void *stream);

#ifdef __cplusplus
}
#endif

#endif /* TCP_SOLVER_H */
