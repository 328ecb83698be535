// Internal declarations shared by the host plan builder (tcp_plan.cpp) and the
// CUDA side (tcp_mvp.cu) of libtcpmvp.so.  Not part of the public C ABI.
#pragma once

#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/tcp_mvp.h"

namespace tcp {

// Thread-local last-error slot behind tcp_last_error().
void set_error(const std::string &message);
int fail(int status, const std::string &message);

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
struct Schedule {
    uint32_t tile_bits = 0;
    std::vector<uint64_t> step_d;     // outer pattern, as a tile-index XOR
    std::vector<uint32_t> step_gbeg;  // groups of step s: [step_gbeg[s], step_gbeg[s+1])
    std::vector<uint32_t> g_min;      // inner mask of each group
    std::vector<uint32_t> g_tbeg;     // terms of group g: [g_tbeg[g], g_tbeg[g+1])
    std::vector<uint64_t> t_z;        // z mask of each term, schedule order
    std::vector<double> t_w;          // weighted phase (re, im), schedule order
    std::vector<float> t_wf;          // the same rounded to FP32 (re, im)
};

// Build the schedule for one tile width.  Groups are the distinct x masks
// (group_matrix_terms, hamiltonian.rs:573-582); terms keep canonical order
// inside a group so the per-group diagonal sum rounds exactly as the
// reference's eager diagonal (hamiltonian.rs:125-133).
Schedule build_schedule(const std::vector<MatrixTerm> &terms, uint32_t nqubits, uint32_t tile_bits);

// Compile packed words into matrix terms (pauli_action.rs:24-88).
int compile_terms(uint32_t nqubits, uint64_t count, uint32_t word_count, const uint64_t *x_words,
                  const uint64_t *z_words, const double *coefficients, std::vector<MatrixTerm> &out);

uint64_t distinct_x_masks(const std::vector<MatrixTerm> &terms);

// Device allocation wrapper with host-side failure injection: when the
// environment variable TCP_FAIL_ALLOC_AFTER=N is set, the allocation after the
// first N successful ones reports failure (nothing touches the GPU).
bool injected_alloc_failure();

}  // namespace tcp
