// Exact top-K of (weight, mask) pairs kept in the registers of one warp.
//
// The order is the reference's candidate_less: weight ascending, then mask
// ascending (include/bmmpy/search/cuda_launch_topk.cuh:16-19).  Lane l holds
// the sorted entries [l*E, l*E + E) of a K = 32*E list; empty slots hold
// (0xffffffff, ~0) and sort last.  Candidates arrive one warp-step at a time:
// every lane offers its own (w, mask); a ballot against the current k-th
// weight lets only the rare improving offers through, and each is inserted
// by the whole warp (position by ballots, shift by one shuffle), so the
// reference's serial lane-0 insertion sort disappears from the hot loop.
#pragma once

#include "common.cuh"

namespace bmm {

template <int E>
struct WarpTopK {
    uint32_t w[E];
    uint64_t m[E];
    uint64_t thr_m;  // mask of entry kk-1 (warp-uniform), with the caller's weight `thr`

    __device__ __forceinline__ void init() {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            w[e] = 0xffffffffu;
            m[e] = ~0ull;
        }
        thr_m = ~0ull;
    }

    // mask of entry kk-1
    __device__ __forceinline__ uint64_t threshold_mask(int kk) const {
        const int idx = kk - 1;
        const int src_lane = idx / E;
        const int src_e = idx % E;
        uint64_t mine = m[0];
#pragma unroll
        for (int e = 1; e < E; ++e)
            if (e == src_e)
                mine = m[e];
        return __shfl_sync(kFull, mine, src_lane);
    }

    // weight of entry kk-1 (the pruning threshold for a top-kk request)
    __device__ __forceinline__ uint32_t threshold(int kk) const {
        const int idx = kk - 1;
        const int src_lane = idx / E;
        const int src_e = idx % E;
        uint32_t mine = w[0];
#pragma unroll
        for (int e = 1; e < E; ++e)
            if (e == src_e)
                mine = w[e];
        return __shfl_sync(kFull, mine, src_lane);
    }

    // Insert a warp-uniform candidate; keeps the K smallest.
    __device__ __forceinline__ void insert(uint32_t wi, uint64_t mi) {
        const int lane = threadIdx.x & 31;
        int pos = 0;
#pragma unroll
        for (int e = 0; e < E; ++e)
            pos += __popc(__ballot_sync(kFull, pair_less(w[e], m[e], wi, mi)));
        if (pos >= 32 * E)
            return;
        const uint32_t pw = __shfl_up_sync(kFull, w[E - 1], 1);
        const uint64_t pm = __shfl_up_sync(kFull, m[E - 1], 1);
#pragma unroll
        for (int e = E - 1; e >= 0; --e) {
            const int j = lane * E + e;
            const uint32_t prev_w = e == 0 ? pw : w[e > 0 ? e - 1 : 0];
            const uint64_t prev_m = e == 0 ? pm : m[e > 0 ? e - 1 : 0];
            if (j > pos) {
                w[e] = prev_w;
                m[e] = prev_m;
            } else if (j == pos) {
                w[e] = wi;
                m[e] = mi;
            }
        }
    }

    // Offer one candidate per lane (ok == false lanes offer nothing).
    // `thr` caches threshold(kk) (and thr_m its mask); both are refreshed
    // after every insertion.  Only offers ordered before entry kk-1 pass the
    // ballot, so ties at the threshold weight with a larger mask -- common in
    // large spectra -- never reach the insertion.
    __device__ __forceinline__ void offer(bool ok, uint32_t wv, uint64_t mv, int kk,
                                         uint32_t& thr) {
        unsigned bal = __ballot_sync(kFull, ok && (wv < thr || (wv == thr && mv < thr_m)));
        while (bal) {
            const int src = __ffs(bal) - 1;
            const uint32_t wi = __shfl_sync(kFull, wv, src);
            const uint64_t mi = __shfl_sync(kFull, mv, src);
            insert(wi, mi);
            thr = threshold(kk);
            thr_m = threshold_mask(kk);
            bal &= ~(1u << src);
            bal &= __ballot_sync(kFull, ok && (wv < thr || (wv == thr && mv < thr_m)));
        }
    }

    // Write entries [0, kk) to out (entries past the filled part are empty).
    __device__ __forceinline__ void store(bmm_candidate* out, int kk) const {
        const int lane = threadIdx.x & 31;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int j = lane * E + e;
            if (j < kk) {
                bmm_candidate c;
                c.mask = m[e];
                c.weight = w[e];
                c.reserved = 0;
                out[j] = c;
            }
        }
    }
};

// Merge `nlists` sorted lists of kk entries into one top-kk list.  limit
// (optional): entries above *limit are known not to be among the kk best
// (some list producer held kk entries of at most that weight) and are skipped.
template <int E>
__global__ void __launch_bounds__(1024) merge_lists_kernel(const bmm_candidate* __restrict__ lists,
                                                            int nlists, int kk,
                                                            bmm_candidate* __restrict__ out,
                                                            const unsigned* __restrict__ limit) {
    extern __shared__ __align__(16) uint64_t smem_raw[];
    bmm_candidate* stage = reinterpret_cast<bmm_candidate*>(smem_raw);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint32_t lim = limit ? *limit : 0xffffffffu;
    WarpTopK<E> top;
    top.init();
    uint32_t thr = 0xffffffffu;
    for (int l = warp; l < nlists; l += nw) {
        for (int base = 0; base < kk; base += 32) {
            const int j = base + lane;
            bmm_candidate c;
            c.weight = 0xffffffffu;
            c.mask = ~0ull;
            if (j < kk)
                c = lists[(size_t)l * kk + j];
            const bool ok = c.weight != 0xffffffffu && c.weight <= lim;
            if (!__any_sync(kFull, ok && c.weight <= thr))
                break;
            top.offer(ok, c.weight, c.mask, kk, thr);
        }
    }
    top.store(stage + warp * 32 * E, 32 * E);
    __syncthreads();
    if (warp == 0) {
        for (int ow = 1; ow < nw; ++ow)
            for (int base = 0; base < 32 * E; base += 32) {
                const bmm_candidate c = stage[ow * 32 * E + base + lane];
                const bool ok = c.weight != 0xffffffffu;
                if (!__any_sync(kFull, ok && c.weight <= thr))
                    break;
                top.offer(ok, c.weight, c.mask, kk, thr);
            }
        top.store(out, kk);
    }
}

// Host: merge `nlists` sorted device lists of kk entries into d_out (kk entries).
int merge_topk_lists(const bmm_candidate* d_lists, int nlists, int kk, bmm_candidate* d_out,
                     cudaStream_t stream, const unsigned* d_limit = nullptr);

}  // namespace bmm
