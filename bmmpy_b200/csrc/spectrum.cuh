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

// The same restricted to a range of slices: the low `low_bits` mask bits are
// one materialised 2^low_bits spectrum per slice x (the mask bits above them),
// x in [slice_begin, slice_end).  low_bits = -1 picks the default split
// (spectrum_low_bits); 14 <= low_bits <= min(t, 33) otherwise.  A range that
// covers every slice gives spectrum_topk_launch's result; ranges that
// partition the slices give lists whose (weight, mask) merge is that result.
int spectrum_topk_slices(Workspace* ws, const uint64_t* d_rows, int t, int W, long long cols,
                         int kk, int low_bits, long long slice_begin, long long slice_end,
                         bmm_candidate* d_out, cudaStream_t stream);

// Low bits materialised per slice for a t-row window: the tuned value when
// set (bmm_spectrum_tune), else min(t, 33).
int spectrum_low_bits(int t);
extern int g_spectrum_low_bits;
// Last transform pass: 1 = one double-buffered CTA per SM, 0 = two
// single-buffered CTAs per SM.
extern int g_spectrum_last_db;
// Passes of >= 6 row bits with lists of <= 128 entries: register-resident
// (HBM straight to registers, one shared-memory exchange) with 2 = two CTAs
// per SM (default) or 1 = one CTA per SM prefetching the next tile into
// registers; 0 = the cp.async tile passes.
extern int g_spectrum_reg;
// Per-t low bits found by the autotuner (bmm_spectrum_tune_shape); -1 = none.
extern int g_spectrum_shape_low_bits[41];

// In-place transform of 2^t int32 in device memory, t >= 14.
int spectrum_dense_fwht(Workspace* ws, int32_t* d, int t, cudaStream_t stream);

}  // namespace bmm
