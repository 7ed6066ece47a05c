// Per-target search bodies shared by the per-target kernels (fwht.cu) and the
// batched persistent kernel (batch.cu).  One CTA solves one item: the best
// S over all subsets of k "other" rows for one target row, minimising
// popcount(target ^ XOR_{j in S} other_j), ties to the smallest S (the
// reference's mask order for the window [target, others]).
//
//  * fwht16:     k = 16, cols <= 32767.  Signed 2^16 histogram packed as 2^15
//                int32 (h[i] + 65536*h[i + 2^15]); three register rounds over a
//                bank-swizzled shared array; needs blockDim == 512 and 128 KB of
//                shared memory.
//  * fwht_small: k <= 15.  int32 spectrum of 2^k in shared memory, any blockDim.
//  * gray:       any k <= 30, rows of at most WPL words: direct reflected-Gray
//                enumeration, cost 2^k * W word operations (cheaper than the
//                transform for narrow rows).
// `others(j)` returns the row index of other j.
#pragma once

#include "common.cuh"

namespace bmm {
namespace item {

constexpr int kFwht16Threads = 512;

__device__ __forceinline__ int swz15(int i) { return i ^ ((i >> 6) & 31); }

template <typename Others>
__device__ __forceinline__ uint32_t col_pattern(const uint64_t* __restrict__ words, int stride,
                                                Others others, int k, uint32_t tgt, int c,
                                                int* tbit) {
    const int w = c >> 6, bit = c & 63;
    uint32_t p = 0;
    for (int j = 0; j < k; ++j)
        p |= (uint32_t)((__ldg(words + (size_t)others(j) * stride + w) >> bit) & 1ull) << j;
    *tbit = (int)((__ldg(words + (size_t)tgt * stride + w) >> bit) & 1ull);
    return p;
}

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

// k = 16 packed transform.  P: 32768 int32 of shared memory; red: 16 uint32.
// Thread 0 writes *out_s / *out_w.  Ends with __syncthreads().
template <typename Others>
__device__ void fwht16(int32_t* P, uint32_t* red, const uint64_t* __restrict__ words, int stride,
                       int cols, Others others, uint32_t tgt, uint64_t* out_s, uint32_t* out_w) {
    constexpr int k = 16;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int4* P4 = reinterpret_cast<int4*>(P);
    for (int i = tid; i < 32768 / 4; i += kFwht16Threads)
        P4[i] = make_int4(0, 0, 0, 0);
    __syncthreads();
    for (int c = tid; c < cols; c += kFwht16Threads) {
        int tb;
        const uint32_t p = col_pattern(words, stride, others, k, tgt, c, &tb);
        const int32_t one = (p & 0x8000u) ? 65536 : 1;
        atomicAdd(P + swz15((int)(p & 0x7fffu)), tb ? -one : one);
    }
    __syncthreads();
    int32_t x[64];
    {  // round 1: bits 0-5, element = tid*64 + e
#pragma unroll
        for (int e = 0; e < 64; ++e)
            x[e] = P[swz15((tid << 6) | e)];
        bfly64(x, 0, 6);
#pragma unroll
        for (int e = 0; e < 64; ++e)
            P[swz15((tid << 6) | e)] = x[e];
    }
    __syncthreads();
    {  // round 2: bits 6-11, element = (tid>>6)<<12 | e<<6 | (tid&63)
        const int basei = ((tid >> 6) << 12) | (tid & 63);
#pragma unroll
        for (int e = 0; e < 64; ++e)
            x[e] = P[swz15(basei | (e << 6))];
        bfly64(x, 0, 6);
#pragma unroll
        for (int e = 0; e < 64; ++e)
            P[swz15(basei | (e << 6))] = x[e];
    }
    __syncthreads();
    {  // round 3: bits 12-14; element = eh<<12 | tid<<3 | el, x[eh*8 + el]
#pragma unroll
        for (int e = 0; e < 64; ++e)
            x[e] = P[swz15(((e >> 3) << 12) | (tid << 3) | (e & 7))];
        bfly64(x, 3, 3);
    }
    // unpack the top bit; max WHT with the smallest S.  s0 grows with e, and
    // every S of the second half (bit 15 set) exceeds every S of the first,
    // so two passes with a strict '>' keep the smallest S among equal maxima.
    int32_t best_v = INT32_MIN;
    int best_e = 0;
#pragma unroll
    for (int e = 0; e < 64; ++e) {
        const int32_t lo = (int32_t)(int16_t)(x[e] & 0xffff);
        const int32_t hi = (x[e] - lo) >> 16;
        const int32_t v0 = lo + hi;
        x[e] = lo - hi;  // keep v1 for the second pass
        if (v0 > best_v)
            best_v = v0, best_e = e;
    }
#pragma unroll
    for (int e = 0; e < 64; ++e)
        if (x[e] > best_v)
            best_v = x[e], best_e = e | 64;
    const uint32_t best_s = (uint32_t)((((best_e & 63) >> 3) << 12) | (tid << 3) | (best_e & 7)) |
                            ((best_e & 64) ? 0x8000u : 0u);
    uint32_t key = ((uint32_t)(best_v + 32768) << 16) | (0xffffu - best_s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        key = max(key, __shfl_xor_sync(kFull, key, o));
    if (lane == 0)
        red[warp] = key;
    __syncthreads();
    if (warp == 0) {
        uint32_t kv = lane < kFwht16Threads / 32 ? red[lane] : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            kv = max(kv, __shfl_xor_sync(kFull, kv, o));
        if (lane == 0) {
            const int32_t v = (int32_t)(kv >> 16) - 32768;
            *out_s = 0xffffu - (kv & 0xffffu);
            *out_w = (uint32_t)((cols - v) / 2);
        }
    }
    __syncthreads();
}

// max over the CTA of a 64-bit key; red: (blockDim / 32) uint64.  Valid in
// thread 0.  Ends with __syncthreads().
__device__ __forceinline__ unsigned long long cta_max64(unsigned long long key,
                                                        unsigned long long* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long ot = __shfl_xor_sync(kFull, key, o);
        key = ot > key ? ot : key;
    }
    if (lane == 0)
        red[warp] = key;
    __syncthreads();
    unsigned long long kv = 0;
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i)
            kv = red[i] > kv ? red[i] : kv;
    __syncthreads();
    return kv;
}

// k <= 15: S has 2^k int32; red: blockDim/32 uint64.
template <typename Others>
__device__ void fwht_small(int32_t* S, unsigned long long* red, const uint64_t* __restrict__ words,
                           int stride, int cols, Others others, int k, uint32_t tgt,
                           uint64_t* out_s, uint32_t* out_w) {
    const int n = 1 << k;
    const int tid = threadIdx.x;
    for (int i = tid; i < n; i += blockDim.x)
        S[i] = 0;
    __syncthreads();
    for (int c = tid; c < cols; c += blockDim.x) {
        int tb;
        const uint32_t p = col_pattern(words, stride, others, k, tgt, c, &tb);
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
    // key: larger v, then smaller s
    unsigned long long key = 0;
    for (int s = tid; s < n; s += blockDim.x) {
        const unsigned long long kk = ((unsigned long long)(uint32_t)(S[s] + 0x80000000u) << 32) |
                                      (0xffffffffu - (uint32_t)s);
        key = kk > key ? kk : key;
    }
    const unsigned long long kv = cta_max64(key, red);
    if (tid == 0) {
        const int32_t v = (int32_t)((uint32_t)(kv >> 32) - 0x80000000u);
        *out_s = 0xffffffffu - (uint32_t)(kv & 0xffffffffu);
        *out_w = (uint32_t)(((long long)cols - v) / 2);
    }
}

// Direct Gray enumeration of the 2^k subsets; rows of W <= WPL words staged
// in srow ((k + 1) * WPL words: others then the target).  Each thread owns one
// prefix of the top min(k, log2 blockDim) bits and sweeps the rest.
// red: blockDim/32 uint64.
template <int WPL, typename Others>
__device__ void gray(uint64_t* srow, unsigned long long* red, const uint64_t* __restrict__ words,
                     int stride, int W, Others others, int k, uint32_t tgt, uint64_t* out_s,
                     uint32_t* out_w) {
    const int tid = threadIdx.x;
    for (int i = tid; i < (k + 1) * WPL; i += blockDim.x) {
        const int r = i / WPL, w = i % WPL;
        const uint32_t row = r < k ? others(r) : tgt;
        srow[i] = w < W ? words[(size_t)row * stride + w] : 0ull;
    }
    __syncthreads();
    int hb = 0;
    while (hb < k && (2 << hb) <= (int)blockDim.x)
        ++hb;
    const int chunk = k - hb;
    const unsigned p = (unsigned)tid;
    const bool valid = p < (1u << hb);
    uint64_t cur[WPL];
#pragma unroll
    for (int i = 0; i < WPL; ++i)
        cur[i] = srow[k * WPL + i];
    for (int b = 0; b < hb; ++b)
        if ((p >> b) & 1u)
#pragma unroll
            for (int i = 0; i < WPL; ++i)
                cur[i] ^= srow[(chunk + b) * WPL + i];
    uint32_t bw = 0;
#pragma unroll
    for (int i = 0; i < WPL; ++i)
        bw += __popcll(cur[i]);
    const uint64_t hi = (uint64_t)p << chunk;
    uint64_t bs = hi, low = 0;
    const uint32_t states = 1u << chunk;
    for (uint32_t s = 1; s < states; ++s) {
        const int b = __ffs(s) - 1;
        uint32_t w = 0;
#pragma unroll
        for (int i = 0; i < WPL; ++i) {
            cur[i] ^= srow[b * WPL + i];
            w += __popcll(cur[i]);
        }
        low ^= 1ull << b;
        if (w < bw || (w == bw && (hi | low) < bs)) {
            bw = w;
            bs = hi | low;
        }
    }
    // min over (w, S) == max over ~key
    const unsigned long long key = valid ? ~(((unsigned long long)bw << 40) | bs) : 0ull;
    const unsigned long long kv = ~cta_max64(key, red);
    if (tid == 0) {
        *out_s = kv & ((1ull << 40) - 1);
        *out_w = (uint32_t)(kv >> 40);
    }
}

}  // namespace item
}  // namespace bmm
