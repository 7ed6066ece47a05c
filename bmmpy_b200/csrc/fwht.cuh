// Launchers for the transform and FWHT search kernels (fwht.cu).
#pragma once

#include "common.cuh"

namespace bmm {

// In-place transform of 2^t elements in device memory (wrapping arithmetic).
template <typename T>
int fwht_global_launch(Workspace* ws, T* d, int t, cudaStream_t stream);

// Per-target best for n_items (target, k others) items; k <= 16, cols <= 32767.
int fwht_targets_launch(Workspace* ws, const uint64_t* d_words, int stride, int cols,
                        const uint32_t* d_targets, const uint32_t* d_others, int n_items, int k,
                        uint64_t* d_best_mask, uint32_t* d_best_weight, cudaStream_t stream);

}  // namespace bmm
