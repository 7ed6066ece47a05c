// Launchers for the HBM-resident spectrum search (spectrum.cu).
#pragma once

#include "common.cuh"

namespace bmm {

// Top-kk (weight, mask) over all nonzero masks of the t window rows packed in
// d_rows (t x W words), t in [1, 40]; d_out receives kk entries (empty ones
// have weight 0xffffffff).  Uses workspace slots Aux, Counter, Idx, Extra0,
// Extra1, Keys, Spec, Cand and Slices.
int spectrum_topk_launch(Workspace* ws, const uint64_t* d_rows, int t, int W, long long cols,
                         int kk, bmm_candidate* d_out, cudaStream_t stream);

// In-place transform of 2^t int32 in device memory, t >= 14.
int spectrum_dense_fwht(Workspace* ws, int32_t* d, int t, cudaStream_t stream);

}  // namespace bmm
