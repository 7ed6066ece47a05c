// Walsh-Hadamard transforms and FWHT spectral searches on sm_100a.
//
// Reference behaviour:
//  * fwht_inplace (src/math/fwht.cpp:28-57, src/math/fwht_scalar.cpp:19-39):
//    unnormalised transform, radix-2 stages len = 1, 2, 4, ..., wrapping
//    two's-complement add/sub.
//  * FwhtSearch::search (src/search/fwht_search.cpp:34-132): histogram of the
//    active columns' t-bit patterns, transform, weight(mask) = (N - WHT)/2,
//    exact top-k by (weight, mask) over masks >= 1.
//
// B200 design:
//  * Small transforms (and all int16 ones) move one 2^(r+b)-element tile
//    (r stage bits x 2^b consecutive low elements) through shared memory per
//    pass; int32 transforms of 2^14 elements and more use the register-round
//    passes of spectrum.cu.
//  * Per-target searches (t <= 16 others, cols <= 32767) never touch HBM: the
//    whole spectrum stays in shared memory and registers of one CTA, with two
//    int16 half-spectra packed into each int32 (h[i] + 65536*h[i + n/2]); the
//    transform is linear and the int32 sums are exact, so one add/sub does
//    two butterflies and the top bit is unpacked only at the final stage.
#include "common.cuh"
#include "fwht.cuh"
#include "target_item.cuh"

#include <type_traits>
#include "topk.cuh"

namespace bmm {
namespace {

// ---------------------------------------------------------------------------
// Global-memory transform passes.
// Tile = 2^r stage elements (stride 2^lo) x 2^b consecutive low elements.
template <typename T>
__global__ void __launch_bounds__(256)
    fwht_pass_kernel(T* __restrict__ d, int t, int lo, int r, int b) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* s = reinterpret_cast<T*>(smem_raw);
    const int tile_elems = 1 << (r + b);
    const unsigned long long lowblocks = 1ull << (lo - b);  // low positions / 2^b
    const unsigned long long ntiles = (1ull << t) >> (r + b);
    for (unsigned long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const unsigned long long lb = tile % lowblocks;
        const unsigned long long hi = tile / lowblocks;
        const unsigned long long base = (hi << (lo + r)) + (lb << b);
        for (int e = threadIdx.x; e < tile_elems; e += blockDim.x) {
            const int i = e & ((1 << b) - 1), j = e >> b;
            s[e] = d[base + ((unsigned long long)j << lo) + i];
        }
        __syncthreads();
        for (int st = 0; st < r; ++st) {
            const int half = tile_elems >> 1;
            for (int q = threadIdx.x; q < half; q += blockDim.x) {
                const int i = q & ((1 << b) - 1), jj = q >> b;
                const int j0 = ((jj >> st) << (st + 1)) | (jj & ((1 << st) - 1));
                const int a0 = (j0 << b) | i, a1 = a0 + (1 << (st + b));
                using U = typename std::conditional<sizeof(T) == 4, uint32_t, uint16_t>::type;
                const U u = (U)s[a0], v = (U)s[a1];
                s[a0] = (T)(U)(u + v);
                s[a1] = (T)(U)(u - v);
            }
            __syncthreads();
        }
        for (int e = threadIdx.x; e < tile_elems; e += blockDim.x) {
            const int i = e & ((1 << b) - 1), j = e >> b;
            d[base + ((unsigned long long)j << lo) + i] = s[e];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Per-target searches, one item per CTA iteration (persistent grid).
// Item i: target row targets[i], others others[i*k .. i*k+k).  All `cols`
// columns count (inactive ones land in bucket 0 with sign +1), so
// weight(S) = (cols - WHT[S]) / 2.  Result: argmax WHT (smallest S on ties).

struct ListOthers {
    const uint32_t* oth;
    __device__ __forceinline__ uint32_t operator()(int j) const { return oth[j]; }
};

constexpr int kT16 = item::kFwht16Threads;

__global__ void __launch_bounds__(kT16, 1)
    fwht_targets16_kernel(const uint64_t* __restrict__ words, int stride, int cols,
                          const uint32_t* __restrict__ targets, const uint32_t* __restrict__ others,
                          int n_items, uint64_t* __restrict__ best_mask,
                          uint32_t* __restrict__ best_weight) {
    extern __shared__ __align__(16) int32_t P[];  // 32768 packed entries
    __shared__ uint32_t red[kT16 / 32];
    for (int it = blockIdx.x; it < n_items; it += gridDim.x)
        item::fwht16(P, red, words, stride, cols, ListOthers{others + (size_t)it * 16}, targets[it],
                     best_mask + it, best_weight + it);
}

// k <= 15: int32 spectrum of 2^k in smem.
__global__ void __launch_bounds__(256)
    fwht_targets_small_kernel(const uint64_t* __restrict__ words, int stride, int cols,
                              const uint32_t* __restrict__ targets,
                              const uint32_t* __restrict__ others, int k, int n_items,
                              uint64_t* __restrict__ best_mask,
                              uint32_t* __restrict__ best_weight) {
    extern __shared__ __align__(16) int32_t S[];
    __shared__ unsigned long long red[8];
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        item::fwht_small(S, red, words, stride, cols, ListOthers{others + (size_t)it * k}, k,
                         targets[it], best_mask + it, best_weight + it);
        __syncthreads();
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// host
template <typename T>
int fwht_global_launch(Workspace* ws, T* d, int t, cudaStream_t stream) {
    if (t <= 0)
        return BMM_OK;
    constexpr int kTileLog = sizeof(T) == 4 ? 14 : 15;  // 64 KB of tile
    int lo = 0;
    while (lo < t) {
        const int b = lo < 3 ? lo : 3;
        int r = kTileLog - b;
        if (r > t - lo)
            r = t - lo;
        const size_t smem = ((size_t)1 << (r + b)) * sizeof(T);
        auto kern = fwht_pass_kernel<T>;
        BMM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
        const unsigned long long ntiles = (1ull << t) >> (r + b);
        unsigned long long grid = (unsigned long long)ws->sm_count * 4;
        if (ntiles < grid)
            grid = ntiles;
        kern<<<(unsigned)grid, 256, smem, stream>>>(d, t, lo, r, b);
        BMM_CUDA_TRY(cudaGetLastError());
        lo += r;
    }
    return BMM_OK;
}

template int fwht_global_launch<int32_t>(Workspace*, int32_t*, int, cudaStream_t);
template int fwht_global_launch<int16_t>(Workspace*, int16_t*, int, cudaStream_t);

int fwht_targets_launch(Workspace* ws, const uint64_t* d_words, int stride, int cols,
                        const uint32_t* d_targets, const uint32_t* d_others, int n_items, int k,
                        uint64_t* d_best_mask, uint32_t* d_best_weight, cudaStream_t stream) {
    if (n_items <= 0)
        return BMM_OK;
    if (k == 16) {
        const size_t smem = 32768 * sizeof(int32_t);
        BMM_CUDA_TRY(cudaFuncSetAttribute(fwht_targets16_kernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int grid = ws->sm_count;
        if (n_items < grid)
            grid = n_items;
        fwht_targets16_kernel<<<grid, kT16, smem, stream>>>(d_words, stride, cols, d_targets,
                                                           d_others, n_items, d_best_mask,
                                                           d_best_weight);
        BMM_CUDA_TRY(cudaGetLastError());
        return BMM_OK;
    }
    const size_t smem = ((size_t)1 << k) * sizeof(int32_t);
    BMM_CUDA_TRY(cudaFuncSetAttribute(fwht_targets_small_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int grid = ws->sm_count * 4;
    if (n_items < grid)
        grid = n_items;
    fwht_targets_small_kernel<<<grid, 256, smem, stream>>>(d_words, stride, cols, d_targets,
                                                          d_others, k, n_items, d_best_mask,
                                                          d_best_weight);
    BMM_CUDA_TRY(cudaGetLastError());
    return BMM_OK;
}

}  // namespace bmm
