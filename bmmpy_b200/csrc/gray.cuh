// Launchers for the Gray-code search kernels (gray.cu).  Device pointers,
// asynchronous on `stream`.
#pragma once

#include "common.cuh"

namespace bmm {

// Overrides used by the autotuner; -1 selects the built-in policy.
struct GrayTuning {
    int hs_blocks = -1;   // carry-save blocks per 64-word lane (0, 2-6, 8)
    int chunk_bits = -1;  // Gray-swept low bits per prefix
    int lanes = -1;       // lanes per prefix for rows of 33-64 words (1 or 2)
};
extern GrayTuning g_gray_tuning;

// Per-shape settings found by the autotuner for rows of W words searched
// against k others (bmm_gray_tune_shape); -1 fields keep the built-in policy.
int gray_tune_shape(size_t W, int k, const GrayTuning& t);
void gray_tune_reset();
// The effective tuning for a shape: the shape entry, overridden field by
// field by the process-wide g_gray_tuning where that is set.
GrayTuning gray_tuning_for(size_t W, int k);

// Low chunk width giving enough independent prefixes to fill the device.
int auto_chunk_bits(int t, int lanes_per_prefix, int sm_count, int n_items);
// The same for the per-target kernel (its occupancy and walk length).
int targets_chunk_bits(int k, int lanes_per_prefix, int sm_count, int n_targets);

// Top-kk over all nonzero masks of the t rows in d_rows (t x W words).
// d_out receives kk entries (empty ones have weight 0xffffffff).
int gray_window_launch(Workspace* ws, const uint64_t* d_rows, int t, int W, int chunk, int kk,
                       bmm_candidate* d_out, cudaStream_t stream);

// Per-target best (see bmm_gray_targets); d_keys is n_targets u64 scratch.
int gray_targets_launch(Workspace* ws, const uint64_t* d_words, int stride, int W,
                        const uint32_t* d_targets, const uint32_t* d_others, int n_targets, int k,
                        int tiebreak, int chunk, unsigned long long* d_keys, uint64_t* d_best_mask,
                        uint32_t* d_best_weight, cudaStream_t stream);

// Measures the register-only 64-bit XOR+POPC word rate of the device.
int popc_probe(double* words_per_second);

}  // namespace bmm
