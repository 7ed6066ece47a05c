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

// Pattern of column c over the k others, and the target bit.
__device__ __forceinline__ uint32_t col_pattern(const uint64_t* __restrict__ words, int stride,
                                                const uint32_t* oth, int k, uint32_t tgt, int c,
                                                int* tbit) {
    const int w = c >> 6, bit = c & 63;
    uint32_t p = 0;
    for (int j = 0; j < k; ++j)
        p |= (uint32_t)((__ldg(words + (size_t)oth[j] * stride + w) >> bit) & 1ull) << j;
    *tbit = (int)((__ldg(words + (size_t)tgt * stride + w) >> bit) & 1ull);
    return p;
}

// Packed-pair transform for k = 16: 2^15 int32 in smem, 512 threads, 64
// elements per thread held in registers for three rounds (bits 0-5, 6-11,
// 12-14).  Exact for cols <= 32767.
constexpr int kT16 = 512;

// Bank swizzle of the packed spectrum: element i lives at i ^ ((i >> 6) & 31),
// which makes all three register rounds below conflict-free.
__device__ __forceinline__ int swz(int i) { return i ^ ((i >> 6) & 31); }

__device__ __forceinline__ void bfly64(int32_t (&x)[64], int lo_bit, int nbits) {
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        if (s < nbits) {
            const int h = 1 << (s + lo_bit);
#pragma unroll
            for (int e = 0; e < 64; ++e)
                if ((e & h) == 0) {
                    const int32_t u = x[e], v = x[e | h];
                    x[e] = u + v;
                    x[e | h] = u - v;
                }
        }
    }
}

__global__ void __launch_bounds__(kT16, 1)
    fwht_targets16_kernel(const uint64_t* __restrict__ words, int stride, int cols,
                          const uint32_t* __restrict__ targets, const uint32_t* __restrict__ others,
                          int n_items, uint64_t* __restrict__ best_mask,
                          uint32_t* __restrict__ best_weight) {
    extern __shared__ __align__(16) int32_t P[];  // 32768 packed entries
    __shared__ uint32_t red[kT16 / 32];
    constexpr int k = 16;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
        const uint32_t* oth = others + (size_t)item * k;
        const uint32_t tgt = targets[item];
        int4* P4 = reinterpret_cast<int4*>(P);
        for (int i = tid; i < 32768 / 4; i += kT16)
            P4[i] = make_int4(0, 0, 0, 0);
        __syncthreads();
        // signed packed histogram
        for (int c = tid; c < cols; c += kT16) {
            int tb;
            const uint32_t p = col_pattern(words, stride, oth, k, tgt, c, &tb);
            const int32_t one = (p & 0x8000u) ? 65536 : 1;
            atomicAdd(P + swz((int)(p & 0x7fffu)), tb ? -one : one);
        }
        __syncthreads();
        int32_t x[64];
        // round 1: bits 0-5, element = tid*64 + e
        {
#pragma unroll
            for (int e = 0; e < 64; ++e)
                x[e] = P[swz((tid << 6) | e)];
            bfly64(x, 0, 6);
#pragma unroll
            for (int e = 0; e < 64; ++e)
                P[swz((tid << 6) | e)] = x[e];
        }
        __syncthreads();
        // round 2: bits 6-11, element = (tid>>6)<<12 | e<<6 | (tid&63)
        {
            const int basei = ((tid >> 6) << 12) | (tid & 63);
#pragma unroll
            for (int e = 0; e < 64; ++e)
                x[e] = P[swz(basei | (e << 6))];
            bfly64(x, 0, 6);
#pragma unroll
            for (int e = 0; e < 64; ++e)
                P[swz(basei | (e << 6))] = x[e];
        }
        __syncthreads();
        // round 3: bits 12-14; element = eh<<12 | tid<<3 | el, x[eh*8 + el]
        {
#pragma unroll
            for (int e = 0; e < 64; ++e)
                x[e] = P[swz(((e >> 3) << 12) | (tid << 3) | (e & 7))];
            bfly64(x, 3, 3);
        }
        // unpack the top bit, find max WHT with the smallest S
        int32_t best_v = INT32_MIN;
        uint32_t best_s = 0xffffffffu;
#pragma unroll
        for (int e = 0; e < 64; ++e) {
            const int32_t pk = x[e];
            const int32_t lo = (int32_t)(int16_t)(pk & 0xffff);
            const int32_t hi = (pk - lo) >> 16;
            const uint32_t s0 = (uint32_t)(((e >> 3) << 12) | (tid << 3) | (e & 7));
            const int32_t v0 = lo + hi, v1 = lo - hi;
            if (v0 > best_v || (v0 == best_v && s0 < best_s))
                best_v = v0, best_s = s0;
            if (v1 > best_v || (v1 == best_v && (s0 | 0x8000u) < best_s))
                best_v = v1, best_s = s0 | 0x8000u;
        }
        // key: larger v first, then smaller s
        uint32_t key = ((uint32_t)(best_v + 32768) << 16) | (0xffffu - best_s);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            key = max(key, __shfl_xor_sync(kFull, key, o));
        if (lane == 0)
            red[warp] = key;
        __syncthreads();
        if (warp == 0) {
            uint32_t kv = lane < kT16 / 32 ? red[lane] : 0u;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
                kv = max(kv, __shfl_xor_sync(kFull, kv, o));
            if (lane == 0) {
                const int32_t v = (int32_t)(kv >> 16) - 32768;
                best_mask[item] = 0xffffu - (kv & 0xffffu);
                best_weight[item] = (uint32_t)((cols - v) / 2);
            }
        }
        __syncthreads();
    }
}

// Generic per-target transform for k <= 15 (and any k when cols forbids
// packing is excluded by the host): int32 spectrum of 2^k in smem.
__global__ void __launch_bounds__(256)
    fwht_targets_small_kernel(const uint64_t* __restrict__ words, int stride, int cols,
                              const uint32_t* __restrict__ targets,
                              const uint32_t* __restrict__ others, int k, int n_items,
                              uint64_t* __restrict__ best_mask,
                              uint32_t* __restrict__ best_weight) {
    extern __shared__ __align__(16) int32_t S[];
    __shared__ unsigned long long red[8];
    const int n = 1 << k;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
        const uint32_t* oth = others + (size_t)item * k;
        const uint32_t tgt = targets[item];
        for (int i = tid; i < n; i += blockDim.x)
            S[i] = 0;
        __syncthreads();
        for (int c = tid; c < cols; c += blockDim.x) {
            int tb;
            const uint32_t p = col_pattern(words, stride, oth, k, tgt, c, &tb);
            atomicAdd(S + p, tb ? -1 : 1);
        }
        __syncthreads();
        for (int st = 0; st < k; ++st) {
            for (int q = tid; q < n / 2; q += blockDim.x) {
                const int j0 = ((q >> st) << (st + 1)) | (q & ((1 << st) - 1));
                const int j1 = j0 | (1 << st);
                const int32_t u = S[j0], v = S[j1];
                S[j0] = u + v;
                S[j1] = u - v;
            }
            __syncthreads();
        }
        // key: (v + 2^31) << 32 | ~s  -> max
        unsigned long long key = 0;
        for (int s = tid; s < n; s += blockDim.x) {
            const unsigned long long kk =
                ((unsigned long long)(uint32_t)(S[s] + 0x80000000u) << 32) | (0xffffffffu - (uint32_t)s);
            key = kk > key ? kk : key;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long ot = __shfl_xor_sync(kFull, key, o);
            key = ot > key ? ot : key;
        }
        if (lane == 0)
            red[warp] = key;
        __syncthreads();
        if (tid == 0) {
            unsigned long long kv = 0;
            for (int i = 0; i < (int)(blockDim.x >> 5); ++i)
                kv = red[i] > kv ? red[i] : kv;
            const int32_t v = (int32_t)((uint32_t)(kv >> 32) - 0x80000000u);
            best_mask[item] = 0xffffffffu - (uint32_t)(kv & 0xffffffffu);
            best_weight[item] = (uint32_t)(((long long)cols - v) / 2);
        }
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
