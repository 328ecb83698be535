// Internal declarations shared by the host plan builder (tcp_plan.cpp) and the
// CUDA side (tcp_mvp.cu) of libtcpmvp.so.  Not part of the public C ABI.
#pragma once

#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/tcp_mvp.h"

#include <nvtx3/nvToolsExt.h>

namespace tcp {

// NVTX range over a scope (plan building, uploads, applies), so that a
// timeline profiler shows where the host side of the library spends its
// time.  NVTX is header-only and costs a null-function call when no tool is
// attached.
struct Range {
    explicit Range(const char *name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range &) = delete;
    Range &operator=(const Range &) = delete;
};

// Thread-local last-error slot behind tcp_last_error().
void set_error(const std::string &message);
int fail(int status, const std::string &message);
// The same with the numeric fields of the PauliError variant (expected /
// actual, requested / limit, code / index, index / 0), read back through
// tcp_last_error_fields so that a binding can rebuild the variant exactly.
int fail_fields(int status, const std::string &message, uint64_t a, uint64_t b);
uint64_t clamp_u64(unsigned __int128 v);
// InvalidStructureLength {expected, actual}: "expected structure length E, got A"
int length_error(uint64_t expected, uint64_t actual);

// One compiled term: StatevectorPauliAction masks in the MSB index space and
// the weighted phase c * i^{#Y} (pauli_action.rs:58-86, hamiltonian.rs:564-571).
struct MatrixTerm {
    uint64_t x_mask;
    uint64_t z_mask;
    double w_re;
    double w_im;
};

// Tile schedule for the tiled kernels.  The 2^n rows are cut into tiles of
// 2^tile_bits consecutive rows.  Every x-mask group m splits into an outer
// pattern d = m >> tile_bits (which source tile feeds an output tile: the tile
// index XOR d) and an inner mask m & (2^tile_bits - 1) (a permutation inside
// the tile).  A "step" is one distinct outer pattern with all groups that share
// it; one tile load serves every group of a step.
//
// Inside a tile, thread t of a CTA with 2^log_threads threads owns rows
// t + j * 2^log_threads (j = 0 .. 2^(tile_bits-log_threads) - 1).  For group
// inner mask m the thread reads source rows (t ^ (m & (T-1))) + jj * T and row
// j takes source jj = j ^ (m >> log_threads).  The sign of a term at source
// column c = (tile ^ d) * 2^S + local is
//   parity(zt & tile) ^ parity(zt & d) ^ parity(zlo & t) ^ parity(zlo & m_lo) ^ parity(zj & jj)
// with zt = z >> S, zlo = z & (T-1), m_lo = m & (T-1),
// zj = (z & (2^S-1)) >> log_threads.  The schedule folds parity(zt & d) and
// parity(zlo & m_lo) into the term's weight and stores the 2^(S-logT)-bit
// pattern parity(zj & jj); the kernel applies parity(zt & tile) once per step
// and tile, and parity(zlo & t) per thread.
struct Schedule {
    uint32_t tile_bits = 0;
    uint32_t log_threads = 0;
    uint64_t distinct_outer = 0;      // distinct outer patterns d
    // step view (tiled kernels).  A step is one outer pattern d and a block of
    // its groups and terms no larger than kBlockBytesMax; a pattern with more
    // data is split over several steps (the tile is loaded once per step).
    // step_info: 4 words per step: d (lo, hi), block offset / 16,
    // group count | (block bytes / 16) << 16.
    std::vector<uint32_t> step_info;
    // Step blocks, 16-byte aligned: group records (16 B: inner mask, first
    // term, end term, 0) then term records (32 B: zlo | pattern << 32 |
    // kind << 56, zt, weight).  The weight has parity(zt & d) folded in and is
    // two doubles (complex128 blocks) or two floats + 8 pad bytes (complex64).
    std::vector<uint8_t> blocks_c128;
    std::vector<uint8_t> blocks_c64;
    // group view (row kernel, transition count, diagonal): unfolded
    std::vector<uint64_t> g_mask;     // full x mask per group (schedule order)
    std::vector<uint32_t> g_tbeg;     // terms of group g: [g_tbeg[g], g_tbeg[g+1])
    std::vector<uint64_t> t_z;        // z mask of each term, schedule order
    std::vector<double> t_w;          // weighted phase (re, im), schedule order
    std::vector<float> t_wf;          // the same rounded to FP32 (re, im)
};

// Schedule of the ring kernel (k_ring).  Same tiles and steps as Schedule
// (one step per distinct outer pattern d, split when its block outgrows
// kRingBlockBytes), but the groups of a step are arranged in cosets: groups
// whose inner masks agree on the thread bits (m & (2^log_threads - 1)) read
// the same 2^(S - log_threads) source values per thread, in a permuted order,
// so the values are loaded once per coset, in row order (fixed offsets), and
// every group of the coset applies them through a compile-time register
// permutation a = jh (its inner-mask bits above the thread bits).
// Block layout (16-byte units):
//   header    {ncosets, ngroups, terms offset / 16, 0}
//   cosets    {m_lo, 0, groups in the coset, 0} each
//   groups    u32 each: a | nterms << 4, padded to 16 bytes; a group's
//             records come in four runs (real weights with one sign for all
//             rows of a thread, real with a row pattern, then the same for
//             imaginary weights)
//   terms     16 bytes each: meta = zlo | pattern << 9 | imag << 17, zt32 =
//             z >> S (low 32 bits), then the folded weight: one f64
//             (complex128 blocks) or one f32 + 4 pad bytes (complex64 blocks).
// A weight is real (imag = 0) or imaginary (imag = 1); a term with a complex
// weight is stored as two records with the same z.  The folded sign is
// parity(zt & d) ^ parity(zlo & m_lo) ^ parity(zj & jh) as in Schedule, so the
// remaining sign of row j is parity(zlo & t) ^ parity(zt & tile) ^ bit j of
// the pattern.  Needs n - S <= 32 (zt32 holds every outer z bit).
struct RingSchedule {
    uint32_t tile_bits = 0;
    uint32_t log_threads = 0;
    uint64_t cosets = 0;               // coset loads per output tile
    uint32_t max_block_bytes = 0;      // largest step block
    std::vector<uint32_t> step_info;   // d lo, d hi, block offset / 16, block bytes / 16
    std::vector<uint8_t> blocks_c128;
    std::vector<uint8_t> blocks_c64;
};

constexpr uint32_t kRingBlockBytes = 8192;

RingSchedule build_ring_schedule(const std::vector<MatrixTerm> &terms, uint32_t nqubits, uint32_t tile_bits,
                                 uint32_t log_threads);

constexpr uint32_t kBlockBytesMax = 16384;
constexpr uint32_t kGroupRecBytes = 16;
constexpr uint32_t kTermRecBytes = 32;

// Term kinds (uniform per term): the weight is real, imaginary, or general.
enum : uint32_t { kKindReal = 0, kKindImag = 1, kKindComplex = 2 };

// Build the schedule for one tile width.  Groups are the distinct x masks
// (group_matrix_terms, hamiltonian.rs:573-582); terms keep canonical order
// inside a group so the per-group diagonal sum rounds exactly as the
// reference's eager diagonal (hamiltonian.rs:125-133).
Schedule build_schedule(const std::vector<MatrixTerm> &terms, uint32_t nqubits, uint32_t tile_bits,
                        uint32_t log_threads);

// Compile packed words into matrix terms (pauli_action.rs:24-88).
int compile_terms(uint32_t nqubits, uint64_t count, uint32_t word_count, const uint64_t *x_words,
                  const uint64_t *z_words, const double *coefficients, std::vector<MatrixTerm> &out);

uint64_t distinct_x_masks(const std::vector<MatrixTerm> &terms);

// Device allocation wrapper with host-side failure injection: when the
// environment variable TCP_FAIL_ALLOC_AFTER=N is set, the allocation after the
// first N successful ones reports failure (nothing touches the GPU).
bool injected_alloc_failure();

}  // namespace tcp
