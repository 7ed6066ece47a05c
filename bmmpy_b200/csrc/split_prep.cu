// build_compact_split_window on the device (src/search/split_window_prep.cpp:42-137,
// include/bmmpy/search/split_window_prep.hpp:10-19): the distinct t-bit column
// patterns of a window (bit i = row i) in ascending order with their
// multiplicities, split into q = pattern >> low_bits and r = pattern & (2^low_bits
// - 1); total_weight = the number of active columns.  The reference builds it on
// the CPU with a hash map and a sort; here: one kernel extracts the patterns of
// the active columns (warp-aggregated appends), a radix sort over the t pattern
// bits orders them, a run-length encoding gives the distinct patterns and
// their counts, and one kernel splits them (CUB device primitives for the sort
// and the run-length pass; they run in the library's own workspace).
#include "common.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_run_length_encode.cuh>

#include <climits>

namespace bmm {
namespace {

// Patterns of the active columns of t packed rows (t x W words), appended in
// an unspecified order; *count receives their number.
__global__ void split_patterns_kernel(const uint64_t* __restrict__ rows, int t, int W,
                                      long long cols, uint64_t* __restrict__ pats,
                                      unsigned long long* __restrict__ count) {
    const int lane = threadIdx.x & 31;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long c0 = blockIdx.x * (long long)blockDim.x + (threadIdx.x & ~31); c0 < cols;
         c0 += stride) {
        const long long c = c0 + lane;
        uint64_t p = 0;
        if (c < cols) {
            const long long w = c >> 6;
            const int bit = (int)(c & 63);
            for (int r = 0; r < t; ++r)
                p |= ((__ldg(rows + (size_t)r * W + w) >> bit) & 1ull) << r;
        }
        const unsigned bal = __ballot_sync(kFull, p != 0);
        if (bal) {
            unsigned long long base = 0;
            if (lane == 0)
                base = atomicAdd(count, (unsigned long long)__popc(bal));
            base = __shfl_sync(kFull, base, 0);
            if (p)
                pats[base + __popc(bal & ((1u << lane) - 1))] = p;
        }
    }
}

__global__ void split_qr_kernel(const uint64_t* __restrict__ uniq, const int* __restrict__ counts,
                                const int* __restrict__ n_runs, int low_bits,
                                uint64_t* __restrict__ q, uint64_t* __restrict__ r,
                                int32_t* __restrict__ mult) {
    const int n = *n_runs;
    const uint64_t low_mask = low_bits >= 64 ? ~0ull : ((1ull << low_bits) - 1);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint64_t p = uniq[i];
        q[i] = low_bits >= 64 ? 0ull : (p >> low_bits);
        r[i] = p & low_mask;
        mult[i] = counts[i];
    }
}

}  // namespace
}  // namespace bmm

using namespace bmm;

extern "C" BMM_API int bmm_split_window_dev(const uint64_t* d_rows, size_t t, size_t W,
                                            size_t cols, size_t low_bits, uint64_t* d_q,
                                            uint64_t* d_r, int32_t* d_mult, size_t cap,
                                            size_t* n_unique, int32_t* total_weight,
                                            void* stream) {
    clear_error();
    if (!n_unique || !total_weight)
        return fail(BMM_EINVAL, "build_compact_split_window: null output count");
    *n_unique = 0;
    *total_weight = 0;
    // the reference's checks, in its order
    if (low_bits > t)
        return fail(BMM_EINVAL, "build_compact_split_window: low_bits must be <= number of rows");
    if (t > 64)
        return fail(BMM_EINVAL, "build_compact_split_window: row count must be <= 64");
    if (t == 0 || W == 0 || cols == 0)
        return BMM_OK;
    if (!d_rows || (cap && (!d_q || !d_r || !d_mult)))
        return fail(BMM_EINVAL, "build_compact_split_window: null argument");
    if (W < (cols + 63) / 64)
        return fail(BMM_EINVAL, "build_compact_split_window: W smaller than the row width");
    if (cols > (size_t)INT_MAX)
        return fail(BMM_EINVAL, "build_compact_split_window: more than 2^31 - 1 columns");
    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws)
        return st;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t n_max = cols;
    void *pats = nullptr, *sorted = nullptr, *misc = nullptr, *temp = nullptr;
    BMM_TRY(ws_buffer(ws, kSlotAux, n_max * 8, &pats));
    BMM_TRY(ws_buffer(ws, kSlotKeys, n_max * 8, &sorted));
    // misc: [count u64][n_runs int][pad] then run counts (int) and unique keys (u64)
    BMM_TRY(ws_buffer(ws, kSlotExtra0, 16 + n_max * 4 + n_max * 8 + 16, &misc));
    unsigned long long* d_count = (unsigned long long*)misc;
    int* d_runs = (int*)((char*)misc + 8);
    int* d_run_counts = (int*)((char*)misc + 16);
    uint64_t* d_uniq =
        (uint64_t*)(((uintptr_t)((char*)misc + 16 + n_max * 4) + 15) & ~(uintptr_t)15);
    BMM_CUDA_TRY(cudaMemsetAsync(d_count, 0, 8, s));
    {
        long long blocks = ((long long)cols + 255) / 256;
        if (blocks > (long long)ws->sm_count * 8)
            blocks = (long long)ws->sm_count * 8;
        split_patterns_kernel<<<(unsigned)(blocks > 0 ? blocks : 1), 256, 0, s>>>(
            d_rows, (int)t, (int)W, (long long)cols, (uint64_t*)pats, d_count);
        BMM_CUDA_TRY(cudaGetLastError());
    }
    unsigned long long n = 0;
    BMM_CUDA_TRY(cudaMemcpyAsync(&n, d_count, 8, cudaMemcpyDeviceToHost, s));
    BMM_CUDA_TRY(cudaStreamSynchronize(s));
    *total_weight = (int32_t)n;  // n <= cols <= INT_MAX
    if (n == 0)
        return BMM_OK;
    size_t sort_bytes = 0, rle_bytes = 0;
    BMM_CUDA_TRY(cub::DeviceRadixSort::SortKeys(nullptr, sort_bytes, (const uint64_t*)pats,
                                                (uint64_t*)sorted, (int)n, 0, (int)t, s));
    BMM_CUDA_TRY(cub::DeviceRunLengthEncode::Encode(nullptr, rle_bytes, (const uint64_t*)sorted,
                                                    d_uniq, d_run_counts, d_runs, (int)n, s));
    BMM_TRY(ws_buffer(ws, kSlotExtra1, sort_bytes > rle_bytes ? sort_bytes : rle_bytes, &temp));
    BMM_CUDA_TRY(cub::DeviceRadixSort::SortKeys(temp, sort_bytes, (const uint64_t*)pats,
                                                (uint64_t*)sorted, (int)n, 0, (int)t, s));
    BMM_CUDA_TRY(cub::DeviceRunLengthEncode::Encode(temp, rle_bytes, (const uint64_t*)sorted,
                                                    d_uniq, d_run_counts, d_runs, (int)n, s));
    int runs = 0;
    BMM_CUDA_TRY(cudaMemcpyAsync(&runs, d_runs, 4, cudaMemcpyDeviceToHost, s));
    BMM_CUDA_TRY(cudaStreamSynchronize(s));
    if ((size_t)runs > cap)
        return fail(BMM_EINVAL,
                    "build_compact_split_window: %d distinct patterns exceed the capacity %zu",
                    runs, cap);
    split_qr_kernel<<<(runs + 255) / 256, 256, 0, s>>>(d_uniq, d_run_counts, d_runs,
                                                       (int)low_bits, d_q, d_r, d_mult);
    BMM_CUDA_TRY(cudaGetLastError());
    BMM_CUDA_TRY(cudaStreamSynchronize(s));
    *n_unique = (size_t)runs;
    return BMM_OK;
}
