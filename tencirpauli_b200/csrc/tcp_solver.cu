// libtcpmvp.so -- eigensolver kernels built on the MVP: FP64 block
// inner products and block combinations over complex64 or complex128 vector
// storage, per-basis-state features, the Jacobi and learned (MLP)
// preconditioners, and the MLP's training kernels (forward, backward, Adam).
//
// Vectors are stored RHS-major (vector v at offset v * n) as complex64 or
// complex128; every reduction and combination accumulates in FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/tcp_solver.h"
#include "tcp_device.cuh"
#include "tcp_plan_impl.h"

using namespace tcpdev;
using tcp::cuda_fail;
using tcp::fail;

namespace {

constexpr int kGramThreads = 256;
constexpr int kGramRows = 32;          // rows staged per chunk
constexpr int kGramMaxVectors = 96;    // p + q
constexpr int kGramBlocks = 296;       // 2 per SM

__device__ __forceinline__ double2 load_c(const void *base, int c64, uint64_t idx) {
    if (c64) {
        const float2 v = static_cast<const float2 *>(base)[idx];
        return make_double2(v.x, v.y);
    }
    return static_cast<const double2 *>(base)[idx];
}
__device__ __forceinline__ void store_c(void *base, int c64, uint64_t idx, double2 v) {
    if (c64) {
        static_cast<float2 *>(base)[idx] = make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
    } else {
        static_cast<double2 *>(base)[idx] = v;
    }
}

// Per-block partial sums of conj(A_i) . B_j over a grid-strided set of row
// chunks; partial[block][i + p*j].
__global__ void __launch_bounds__(kGramThreads)
    k_gram_partial(const void *__restrict__ A, int a64, uint32_t p, const void *__restrict__ B, int b64, uint32_t q,
                   uint64_t n, double2 *__restrict__ partial) {
    __shared__ double2 sa[kGramRows][kGramMaxVectors];
    const uint32_t pairs = p * q;
    double2 acc[2] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
    const uint64_t chunks = (n + kGramRows - 1) / kGramRows;
    for (uint64_t c = blockIdx.x; c < chunks; c += gridDim.x) {
        const uint64_t r0 = c * kGramRows;
        __syncthreads();
        for (uint32_t e = threadIdx.x; e < kGramRows * (p + q); e += blockDim.x) {
            const uint32_t v = e / kGramRows, rr = e % kGramRows;
            const uint64_t row = r0 + rr;
            double2 val = make_double2(0.0, 0.0);
            if (row < n) val = v < p ? load_c(A, a64, v * n + row) : load_c(B, b64, (v - p) * n + row);
            sa[rr][v] = val;
        }
        __syncthreads();
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            const uint32_t pr = threadIdx.x + s * kGramThreads;
            if (pr < pairs) {
                const uint32_t i = pr % p, j = pr / p;
                double re = acc[s].x, im = acc[s].y;
#pragma unroll 4
                for (int rr = 0; rr < kGramRows; ++rr) {
                    const double2 a = sa[rr][i], b = sa[rr][p + j];
                    re = fma(a.x, b.x, fma(a.y, b.y, re));
                    im = fma(a.x, b.y, fma(-a.y, b.x, im));
                }
                acc[s] = make_double2(re, im);
            }
        }
    }
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const uint32_t pr = threadIdx.x + s * kGramThreads;
        if (pr < pairs) partial[static_cast<size_t>(blockIdx.x) * pairs + pr] = acc[s];
    }
}

// Deterministic reduction of the per-block partials (fixed order).
__global__ void k_gram_reduce(const double2 *__restrict__ partial, uint32_t blocks, uint32_t pairs,
                              double2 *__restrict__ out) {
    const uint32_t pr = blockIdx.x * blockDim.x + threadIdx.x;
    if (pr >= pairs) return;
    double re = 0.0, im = 0.0;
    for (uint32_t b = 0; b < blocks; ++b) {
        const double2 v = partial[static_cast<size_t>(b) * pairs + pr];
        re += v.x;
        im += v.y;
    }
    out[pr] = make_double2(re, im);
}

// out[:, j] = alpha * sum_i A[:, i] S[i, j] + beta * out[:, j]  (FP64 arithmetic)
template <int KMAX>
__global__ void k_combine(const void *__restrict__ A, int a64, uint32_t p, const double2 *__restrict__ S, uint32_t k,
                          uint64_t n, double alpha, double beta, void *__restrict__ out, int o64) {
    extern __shared__ double2 ss[];  // S, p x k column-major
    for (uint32_t e = threadIdx.x; e < p * k; e += blockDim.x) ss[e] = S[e];
    __syncthreads();
    for (uint64_t r = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; r < n;
         r += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        double2 acc[KMAX];
#pragma unroll
        for (int j = 0; j < KMAX; ++j) acc[j] = make_double2(0.0, 0.0);
        for (uint32_t i = 0; i < p; ++i) {
            const double2 a = load_c(A, a64, i * n + r);
#pragma unroll
            for (int j = 0; j < KMAX; ++j) {
                if (j < static_cast<int>(k)) {
                    const double2 s = ss[i + p * j];
                    acc[j].x = fma(a.x, s.x, fma(-a.y, s.y, acc[j].x));
                    acc[j].y = fma(a.x, s.y, fma(a.y, s.x, acc[j].y));
                }
            }
        }
#pragma unroll
        for (int j = 0; j < KMAX; ++j) {
            if (j < static_cast<int>(k)) {
                double2 v = make_double2(alpha * acc[j].x, alpha * acc[j].y);
                if (beta != 0.0) {
                    const double2 o = load_c(out, o64, j * n + r);
                    v.x = fma(beta, o.x, v.x);
                    v.y = fma(beta, o.y, v.y);
                }
                store_c(out, o64, j * n + r, v);
            }
        }
    }
}

// Jacobi correction t = -r / (d - theta), |d - theta| clamped below by eps.
__global__ void k_jacobi(const void *__restrict__ R, int r64, uint64_t n, uint32_t k, const double2 *__restrict__ diag,
                         const double *__restrict__ theta, double eps, void *__restrict__ T, int t64) {
    for (uint64_t r = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; r < n;
         r += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const double d = diag[r].x;
        for (uint32_t j = 0; j < k; ++j) {
            double den = d - theta[j];
            if (fabs(den) < eps) den = den < 0.0 ? -eps : eps;
            const double2 v = load_c(R, r64, j * n + r);
            store_c(T, t64, j * n + r, make_double2(-v.x / den, -v.y / den));
        }
    }
}

// Per-basis-state features that do not depend on the Ritz value (see
// tcp_solver.h): H_ii, the mean and minimum diagonal of the states the row
// couples to, sum |H_ij|, sum |H_ij|^2, the number of couplings, and the
// normalised Hamming weight of the basis state.
__global__ void k_features(DevSchedule s, uint32_t gzero, uint32_t nqubits, uint64_t n, float *__restrict__ feat) {
    for (uint64_t r = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; r < n;
         r += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        auto diag_at = [&](uint64_t c) -> double {
            double re = 0.0;
            if (gzero != 0xffffffffu) {
                for (uint32_t t = s.g_tbeg[gzero]; t < s.g_tbeg[gzero + 1]; ++t) {
                    const double2 w = s.t_w[t];
                    re += (__popcll(s.t_z[t] & c) & 1) ? -w.x : w.x;
                }
            }
            return re;
        };
        const double hii = diag_at(r);
        double sum_abs = 0.0, sum_sq = 0.0, sum_nd = 0.0, min_nd = 1e300;
        uint32_t count = 0;
        for (uint32_t g = 0; g < s.ngroups; ++g) {
            if (g == gzero) continue;
            const uint64_t c = r ^ s.g_mask[g];
            double dre = 0.0, dim = 0.0;
            for (uint32_t t = s.g_tbeg[g]; t < s.g_tbeg[g + 1]; ++t) {
                const double2 w = s.t_w[t];
                const bool neg = __popcll(s.t_z[t] & c) & 1;
                dre += neg ? -w.x : w.x;
                dim += neg ? -w.y : w.y;
            }
            const double a2 = dre * dre + dim * dim;
            if (a2 == 0.0) continue;
            const double dj = diag_at(c);
            sum_abs += sqrt(a2);
            sum_sq += a2;
            sum_nd += dj;
            min_nd = fmin(min_nd, dj);
            ++count;
        }
        float *f = feat + r * TCP_FEATURES;
        f[0] = static_cast<float>(hii);
        f[1] = static_cast<float>(count ? sum_nd / count : hii);
        f[2] = static_cast<float>(count ? min_nd : hii);
        f[3] = static_cast<float>(sum_abs);
        f[4] = static_cast<float>(sum_sq);
        f[5] = static_cast<float>(count);
        f[6] = static_cast<float>(static_cast<double>(__popcll(r)) / fmax(1.0, static_cast<double>(nqubits)) - 0.5);
        f[7] = 0.f;
    }
}

// ---------------------------------- MLP -------------------------------------
// Network: x (TCP_MLP_IN inputs, built from the features and the Ritz value)
// -> tanh(W1 x + b1) (TCP_MLP_HIDDEN) -> tanh(W2 h1 + b2) (TCP_MLP_HIDDEN)
// -> c = w3 . h2 + b3.  The correction is t = -exp(c) r / max(d - theta, eps):
// c = 0 is the Jacobi correction, and the network learns a per-state factor.
constexpr int IN = TCP_MLP_IN, HID = TCP_MLP_HIDDEN;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + HID * IN, OFF_W2 = OFF_B1 + HID, OFF_B2 = OFF_W2 + HID * HID,
              OFF_W3 = OFF_B2 + HID, OFF_B3 = OFF_W3 + HID, NPARAM = OFF_B3 + 1;
static_assert(NPARAM == TCP_MLP_PARAMS, "parameter count mismatch");

// Network inputs of one basis state for Ritz value theta; `scale` normalises
// energies (a spread of the spectrum).  Also returns den = max(d - theta, eps).
__device__ __forceinline__ void mlp_inputs(const float *__restrict__ f, double theta, double scale, double eps,
                                           float (&x)[IN], double &den) {
    const double inv = 1.0 / scale;
    double d = static_cast<double>(f[0]) - theta;
    den = fabs(d) < eps ? (d < 0.0 ? -eps : eps) : d;
    x[0] = static_cast<float>(d * inv);
    x[1] = static_cast<float>((static_cast<double>(f[1]) - theta) * inv);
    x[2] = static_cast<float>((static_cast<double>(f[2]) - theta) * inv);
    x[3] = static_cast<float>(static_cast<double>(f[3]) * inv);
    x[4] = static_cast<float>(static_cast<double>(f[4]) * inv * inv);
    x[5] = static_cast<float>(static_cast<double>(f[5]) * 0.05);
    x[6] = f[6];
    // size of the second-order (one coupling out and back) term relative to the
    // first-order denominator, squashed to [0, 1)
    const double ratio = static_cast<double>(f[4]) / (fabs(den) * fmax(fabs(static_cast<double>(f[1]) - theta), eps));
    x[7] = static_cast<float>(ratio / (1.0 + ratio));
}

__device__ __forceinline__ float mlp_forward(const float *__restrict__ w, const float (&x)[IN], float (&h1)[HID],
                                             float (&h2)[HID]) {
#pragma unroll 4
    for (int o = 0; o < HID; ++o) {
        float a = w[OFF_B1 + o];
#pragma unroll
        for (int i = 0; i < IN; ++i) a = fmaf(w[OFF_W1 + o * IN + i], x[i], a);
        h1[o] = tanhf(a);
    }
#pragma unroll 4
    for (int o = 0; o < HID; ++o) {
        float a = w[OFF_B2 + o];
#pragma unroll 8
        for (int i = 0; i < HID; ++i) a = fmaf(w[OFF_W2 + o * HID + i], h1[i], a);
        h2[o] = tanhf(a);
    }
    float c = w[OFF_B3];
#pragma unroll 8
    for (int i = 0; i < HID; ++i) c = fmaf(w[OFF_W3 + i], h2[i], c);
    return c;
}

// Learned correction for k residual vectors: t_j = -exp(c) r_j / den with
// den = H_ii - theta_j (FP64 diagonal, clamped by eps, exactly as k_jacobi).
__global__ void k_mlp_precond(const void *__restrict__ R, int r64, uint64_t n, uint32_t k,
                              const float *__restrict__ feat, const double2 *__restrict__ diag,
                              const double *__restrict__ theta, double scale, double eps, float clamp,
                              const float *__restrict__ wglob, void *__restrict__ T, int t64) {
    __shared__ float w[NPARAM];
    for (int e = threadIdx.x; e < NPARAM; e += blockDim.x) w[e] = wglob[e];
    __syncthreads();
    for (uint64_t r = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; r < n;
         r += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const float *f = feat + r * TCP_FEATURES;
        const double d = diag[r].x;
        for (uint32_t j = 0; j < k; ++j) {
            float x[IN], h1[HID], h2[HID];
            double den_f;
            mlp_inputs(f, theta[j], scale, eps, x, den_f);
            double den = d - theta[j];
            if (fabs(den) < eps) den = den < 0.0 ? -eps : eps;
            const float c = fminf(fmaxf(mlp_forward(w, x, h1, h2), -clamp), clamp);
            const double2 v = load_c(R, r64, j * n + r);
            if (c == 0.f) {  // the Jacobi correction, rounded exactly as k_jacobi
                store_c(T, t64, j * n + r, make_double2(-v.x / den, -v.y / den));
            } else {
                const double g = -exp(static_cast<double>(c)) / den;
                store_c(T, t64, j * n + r, make_double2(g * v.x, g * v.y));
            }
        }
    }
}

// Training: per sample s the network sees inputs X[s] (TCP_MLP_IN floats) and
// predicts c; the correction is g = -exp(c) / den[s].  With a = |r|^2 and
// b = Re(conj(e) r) (e: the exact correction), the sample loss is
// wt[s] * (g^2 a - 2 g b + |e|^2).  A block takes kTrainChunk samples at a
// time: each thread runs one sample forward and back to the hidden layers and
// stages its activations in shared memory, then every thread accumulates the
// weight gradients of the parameters it owns over the chunk (no atomics; the
// result is deterministic).  Each block writes its gradient partial sum.
constexpr int kTrainChunk = 128;
constexpr int kTrainStride = IN + 4 * HID + 1;  // x, h1, h2, dh1, dh2, dc
__global__ void __launch_bounds__(kTrainChunk)
    k_mlp_train(const float *__restrict__ X, const float *__restrict__ den, const float *__restrict__ a,
                const float *__restrict__ b, const float *__restrict__ e2, const float *__restrict__ wt,
                const float *__restrict__ dc_in, uint32_t count, const float *__restrict__ wglob,
                float *__restrict__ grad_partial, float *__restrict__ loss_partial) {
    __shared__ float w[NPARAM];
    __shared__ float act[kTrainChunk][kTrainStride];
    __shared__ float lsum[kTrainChunk];
    constexpr int kOwn = (NPARAM + kTrainChunk - 1) / kTrainChunk;
    for (int e = threadIdx.x; e < NPARAM; e += blockDim.x) w[e] = wglob[e];
    float gacc[kOwn];
#pragma unroll
    for (int q = 0; q < kOwn; ++q) gacc[q] = 0.f;
    float loss = 0.f;
    __syncthreads();
    const uint32_t chunks = (count + kTrainChunk - 1) / kTrainChunk;
    for (uint32_t ch = blockIdx.x; ch < chunks; ch += gridDim.x) {
        const uint32_t sidx = ch * kTrainChunk + threadIdx.x;
        float *my = act[threadIdx.x];
        if (sidx < count) {
            float x[IN], h1[HID], h2[HID];
#pragma unroll
            for (int i = 0; i < IN; ++i) x[i] = X[static_cast<size_t>(sidx) * IN + i];
            const float c = mlp_forward(w, x, h1, h2);
            float dc;
            if (dc_in != nullptr) {  // caller-supplied dL/dc (any loss on the outputs)
                dc = dc_in[sidx];
            } else {
                const float g = -expf(c) / den[sidx];
                const float as = a[sidx], bs = b[sidx], ws = wt[sidx];
                loss += ws * (g * g * as - 2.f * g * bs + e2[sidx]);
                dc = ws * (2.f * g * as - 2.f * bs) * g;  // dL/dc
            }
            float dh2[HID];
#pragma unroll
            for (int i = 0; i < HID; ++i) dh2[i] = dc * w[OFF_W3 + i] * (1.f - h2[i] * h2[i]);
#pragma unroll
            for (int i = 0; i < IN; ++i) my[i] = x[i];
#pragma unroll
            for (int i = 0; i < HID; ++i) {
                float d1 = 0.f;
#pragma unroll
                for (int o = 0; o < HID; ++o) d1 = fmaf(dh2[o], w[OFF_W2 + o * HID + i], d1);
                my[IN + i] = h1[i];
                my[IN + HID + i] = h2[i];
                my[IN + 2 * HID + i] = d1 * (1.f - h1[i] * h1[i]);
                my[IN + 3 * HID + i] = dh2[i];
            }
            my[IN + 4 * HID] = dc;
        } else {
            for (int i = 0; i < kTrainStride; ++i) my[i] = 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < kOwn; ++q) {
            const int pidx = threadIdx.x + q * kTrainChunk;
            if (pidx >= NPARAM) break;
            float acc = 0.f;
            if (pidx < OFF_B1) {  // W1[o][i] += dh1[o] * x[i]
                const int o = pidx / IN, i = pidx % IN;
                for (int r = 0; r < kTrainChunk; ++r) acc = fmaf(act[r][IN + 2 * HID + o], act[r][i], acc);
            } else if (pidx < OFF_W2) {  // b1[o]
                const int o = pidx - OFF_B1;
                for (int r = 0; r < kTrainChunk; ++r) acc += act[r][IN + 2 * HID + o];
            } else if (pidx < OFF_B2) {  // W2[o][i] += dh2[o] * h1[i]
                const int o = (pidx - OFF_W2) / HID, i = (pidx - OFF_W2) % HID;
                for (int r = 0; r < kTrainChunk; ++r) acc = fmaf(act[r][IN + 3 * HID + o], act[r][IN + i], acc);
            } else if (pidx < OFF_W3) {  // b2[o]
                const int o = pidx - OFF_B2;
                for (int r = 0; r < kTrainChunk; ++r) acc += act[r][IN + 3 * HID + o];
            } else if (pidx < OFF_B3) {  // w3[i] += dc * h2[i]
                const int i = pidx - OFF_W3;
                for (int r = 0; r < kTrainChunk; ++r) acc = fmaf(act[r][IN + 4 * HID], act[r][IN + HID + i], acc);
            } else {  // b3
                for (int r = 0; r < kTrainChunk; ++r) acc += act[r][IN + 4 * HID];
            }
            gacc[q] += acc;
        }
        __syncthreads();
    }
#pragma unroll
    for (int q = 0; q < kOwn; ++q) {
        const int pidx = threadIdx.x + q * kTrainChunk;
        if (pidx < NPARAM) grad_partial[static_cast<size_t>(blockIdx.x) * NPARAM + pidx] = gacc[q];
    }
    lsum[threadIdx.x] = loss;
    __syncthreads();
    if (threadIdx.x == 0) {
        float l = 0.f;
        for (int i = 0; i < kTrainChunk; ++i) l += lsum[i];
        loss_partial[blockIdx.x] = l;
    }
}

// Fixed-order sum of per-block losses.
__global__ void k_sum_losses(const float *__restrict__ partial, uint32_t blocks, float *__restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        float l = 0.f;
        for (uint32_t b = 0; b < blocks; ++b) l += partial[b];
        *out = l;
    }
}

// Network output c for every sample.
__global__ void k_mlp_forward(const float *__restrict__ X, uint32_t count, const float *__restrict__ wglob,
                              float *__restrict__ out) {
    __shared__ float w[NPARAM];
    for (int e = threadIdx.x; e < NPARAM; e += blockDim.x) w[e] = wglob[e];
    __syncthreads();
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < count; s += gridDim.x * blockDim.x) {
        float x[IN], h1[HID], h2[HID];
#pragma unroll
        for (int i = 0; i < IN; ++i) x[i] = X[static_cast<size_t>(s) * IN + i];
        out[s] = mlp_forward(w, x, h1, h2);
    }
}

// Sum the per-block gradient partials (fixed order) and apply one Adam step.
__global__ void k_adam(float *__restrict__ w, float *__restrict__ m, float *__restrict__ v,
                       const float *__restrict__ grad_partial, uint32_t blocks, float scale, float lr, float b1,
                       float b2, float eps, uint32_t step, float *__restrict__ grad_out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= NPARAM) return;
    float gsum = 0.f;
    for (uint32_t b = 0; b < blocks; ++b) gsum += grad_partial[static_cast<size_t>(b) * NPARAM + e];
    const float g = gsum * scale;
    if (grad_out) grad_out[e] = g;
    if (lr == 0.f) return;  // gradient only
    m[e] = b1 * m[e] + (1.f - b1) * g;
    v[e] = b2 * v[e] + (1.f - b2) * g * g;
    const float mh = m[e] / (1.f - powf(b1, static_cast<float>(step)));
    const float vh = v[e] / (1.f - powf(b2, static_cast<float>(step)));
    w[e] -= lr * mh / (sqrtf(vh) + eps);
}

// Network inputs and denominators for training samples taken from features.
__global__ void k_mlp_inputs(const float *__restrict__ feat, const uint64_t *__restrict__ rows, const double *__restrict__ theta,
                             const uint32_t *__restrict__ which, uint32_t count, double scale, double eps,
                             float *__restrict__ X, float *__restrict__ den) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < count; s += gridDim.x * blockDim.x) {
        float x[IN];
        double d;
        mlp_inputs(feat + rows[s] * TCP_FEATURES, theta[which[s]], scale, eps, x, d);
#pragma unroll
        for (int i = 0; i < IN; ++i) X[static_cast<size_t>(s) * IN + i] = x[i];
        den[s] = static_cast<float>(d);
    }
}

int grid_for(uint64_t n, int threads) {
    return static_cast<int>(std::min<uint64_t>((n + threads - 1) / threads, 148ull * 16));
}

bool valid_dtype(int d) { return d == TCP_DTYPE_C128 || d == TCP_DTYPE_C64; }

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" size_t tcp_gram_work_bytes(uint32_t p, uint32_t q) {
    return static_cast<size_t>(kGramBlocks) * p * q * sizeof(double2);
}

extern "C" int tcp_gram(const void *A, int a_dtype, uint32_t p, const void *B, int b_dtype, uint32_t q, uint64_t n,
                        void *d_G, void *d_work, void *stream) {
    if (!valid_dtype(a_dtype) || !valid_dtype(b_dtype)) return fail(TCP_ERR_INVALID_ARGUMENT, "unknown dtype");
    if (p == 0 || q == 0) return TCP_OK;
    if (p + q > kGramMaxVectors || p * q > 2 * kGramThreads) {
        return fail(TCP_ERR_INVALID_ARGUMENT, "tcp_gram supports p + q <= 96 and p * q <= 512");
    }
    if (!A || !B || !d_G || !d_work) return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    auto *partial = static_cast<double2 *>(d_work);
    k_gram_partial<<<kGramBlocks, kGramThreads, 0, s>>>(A, a_dtype == TCP_DTYPE_C64, p, B, b_dtype == TCP_DTYPE_C64, q,
                                                        n, partial);
    const uint32_t pairs = p * q;
    k_gram_reduce<<<(pairs + 127) / 128, 128, 0, s>>>(partial, kGramBlocks, pairs, static_cast<double2 *>(d_G));
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "gram kernel launch");
}

extern "C" int tcp_block_combine(const void *A, int a_dtype, uint32_t p, const void *d_S, uint32_t k, uint64_t n,
                                 double alpha, double beta, void *out, int out_dtype, void *stream) {
    if (!valid_dtype(a_dtype) || !valid_dtype(out_dtype)) return fail(TCP_ERR_INVALID_ARGUMENT, "unknown dtype");
    if (k == 0) return TCP_OK;
    if (k > 16) return fail(TCP_ERR_INVALID_ARGUMENT, "tcp_block_combine supports k <= 16");
    if (p * k * sizeof(double2) > 96 * 1024) return fail(TCP_ERR_INVALID_ARGUMENT, "coefficient block too large");
    if (!A || !d_S || !out) return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t smem = p * k * sizeof(double2);
    const int threads = 256;
    const int grid = grid_for(n, threads);
    const int a64 = a_dtype == TCP_DTYPE_C64, o64 = out_dtype == TCP_DTYPE_C64;
    const auto *S = static_cast<const double2 *>(d_S);
    cudaError_t e;
    if (k <= 4) {
        cudaFuncSetAttribute(k_combine<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
        k_combine<4><<<grid, threads, smem, s>>>(A, a64, p, S, k, n, alpha, beta, out, o64);
    } else if (k <= 8) {
        cudaFuncSetAttribute(k_combine<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
        k_combine<8><<<grid, threads, smem, s>>>(A, a64, p, S, k, n, alpha, beta, out, o64);
    } else {
        cudaFuncSetAttribute(k_combine<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
        k_combine<16><<<grid, threads, smem, s>>>(A, a64, p, S, k, n, alpha, beta, out, o64);
    }
    e = cudaGetLastError();
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "combine kernel launch");
}

extern "C" int tcp_precond_jacobi(const void *R, int r_dtype, uint64_t n, uint32_t k, const void *d_diag,
                                  const double *d_theta, double eps, void *T, int t_dtype, void *stream) {
    if (!valid_dtype(r_dtype) || !valid_dtype(t_dtype)) return fail(TCP_ERR_INVALID_ARGUMENT, "unknown dtype");
    if (!R || !d_diag || !d_theta || !T) return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    k_jacobi<<<grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        R, r_dtype == TCP_DTYPE_C64, n, k, static_cast<const double2 *>(d_diag), d_theta, eps, T, t_dtype == TCP_DTYPE_C64);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "jacobi kernel launch");
}

extern "C" int tcp_state_features(const tcp_mvp_plan *plan, float *d_features, uint64_t n, void *stream) {
    int st = tcp::check_plan(plan);
    if (st) return st;
    if (n != plan->dim) return tcp::length_error(plan->dim, n);
    if (!d_features) return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    const tcp::Schedule &h = plan->sched.host;
    uint32_t gzero = 0xffffffffu;
    for (size_t g = 0; g < h.g_mask.size(); ++g)
        if (h.g_mask[g] == 0) gzero = static_cast<uint32_t>(g);
    k_features<<<grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(plan->sched.dev, gzero, plan->nqubits, n,
                                                                              d_features);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "feature kernel launch");
}

extern "C" int tcp_precond_mlp(const void *R, int r_dtype, uint64_t n, uint32_t k, const float *d_features,
                               const void *d_diag, const double *d_theta, double scale, double eps, float clamp,
                               const float *d_params, void *T, int t_dtype, void *stream) {
    if (!valid_dtype(r_dtype) || !valid_dtype(t_dtype)) return fail(TCP_ERR_INVALID_ARGUMENT, "unknown dtype");
    if (!R || !d_features || !d_diag || !d_theta || !d_params || !T) return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    k_mlp_precond<<<grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        R, r_dtype == TCP_DTYPE_C64, n, k, d_features, static_cast<const double2 *>(d_diag), d_theta, scale, eps, clamp,
        d_params, T, t_dtype == TCP_DTYPE_C64);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "mlp preconditioner launch");
}

extern "C" int tcp_mlp_inputs(const float *d_features, const uint64_t *d_rows, const double *d_theta,
                              const uint32_t *d_which, uint32_t count, double scale, double eps, float *d_X,
                              float *d_den, void *stream) {
    if (!d_features || !d_rows || !d_theta || !d_which || !d_X || !d_den) return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    if (count == 0) return TCP_OK;
    k_mlp_inputs<<<grid_for(count, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(d_features, d_rows, d_theta, d_which,
                                                                                   count, scale, eps, d_X, d_den);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "mlp input kernel launch");
}

extern "C" int tcp_mlp_forward(const float *d_X, uint32_t count, const float *d_params, float *d_out, void *stream) {
    if (!d_X || !d_params || !d_out) return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    if (count == 0) return TCP_OK;
    k_mlp_forward<<<grid_for(count, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(d_X, count, d_params, d_out);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "mlp forward launch");
}

extern "C" int tcp_mlp_backward_step(const float *d_X, const float *d_dc, uint32_t count, float *d_params, float *d_m,
                                     float *d_v, float *d_work, float lr, uint32_t step, float *d_grad_out,
                                     void *stream) {
    if (!d_X || !d_dc || !d_params || !d_work) return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    if (lr != 0.f && (!d_m || !d_v || step == 0)) return fail(TCP_ERR_INVALID_ARGUMENT, "Adam state missing");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    float *grad_partial = d_work;
    float *loss_partial = d_work + static_cast<size_t>(TCP_MLP_TRAIN_BLOCKS) * TCP_MLP_PARAMS;
    k_mlp_train<<<TCP_MLP_TRAIN_BLOCKS, kTrainChunk, 0, s>>>(d_X, nullptr, nullptr, nullptr, nullptr, nullptr, d_dc,
                                                             count, d_params, grad_partial, loss_partial);
    k_adam<<<(TCP_MLP_PARAMS + 255) / 256, 256, 0, s>>>(d_params, d_m, d_v, grad_partial, TCP_MLP_TRAIN_BLOCKS, 1.f, lr,
                                                       0.9f, 0.999f, 1e-8f, step, d_grad_out);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "mlp backward launch");
}

extern "C" size_t tcp_mlp_train_work_bytes(void) {
    return static_cast<size_t>(TCP_MLP_TRAIN_BLOCKS) * (TCP_MLP_PARAMS + 1) * sizeof(float);
}

extern "C" int tcp_mlp_train_step(const float *d_X, const float *d_den, const float *d_a, const float *d_b,
                                  const float *d_e2, const float *d_wt, uint32_t count, float *d_params, float *d_m,
                                  float *d_v, float *d_work, float lr, uint32_t step, float *d_grad_out,
                                  float *d_loss_out, void *stream) {
    if (!d_X || !d_den || !d_a || !d_b || !d_e2 || !d_wt || !d_params || !d_work) {
        return fail(TCP_ERR_INVALID_ARGUMENT, "null buffer");
    }
    if (lr != 0.f && (!d_m || !d_v || step == 0)) return fail(TCP_ERR_INVALID_ARGUMENT, "Adam state missing");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    float *grad_partial = d_work;
    float *loss_partial = d_work + static_cast<size_t>(TCP_MLP_TRAIN_BLOCKS) * TCP_MLP_PARAMS;
    k_mlp_train<<<TCP_MLP_TRAIN_BLOCKS, kTrainChunk, 0, s>>>(d_X, d_den, d_a, d_b, d_e2, d_wt, nullptr, count,
                                                             d_params, grad_partial, loss_partial);
    k_adam<<<(TCP_MLP_PARAMS + 255) / 256, 256, 0, s>>>(d_params, d_m, d_v, grad_partial, TCP_MLP_TRAIN_BLOCKS, 1.f, lr,
                                                       0.9f, 0.999f, 1e-8f, step, d_grad_out);
    if (d_loss_out) k_sum_losses<<<1, 32, 0, s>>>(loss_partial, TCP_MLP_TRAIN_BLOCKS, d_loss_out);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TCP_OK : cuda_fail(e, "mlp training launch");
}
