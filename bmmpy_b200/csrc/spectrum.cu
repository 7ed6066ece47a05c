// Exact top-k over the full Walsh-Hadamard spectrum of a window, in HBM.
//
// Serves FwhtSearch (src/search/fwht_search.cpp:34-132) and MitmFwhtSearch
// (src/search/mitm_fwht_search.cpp:267-322): both return the k smallest
// (weight, mask) over all nonzero masks of the t window rows, with
// weight(mask) = (N - WHT[mask]) / 2, N = active columns and WHT the
// transform of the active columns' t-bit pattern histogram.
//
// B200 design.  The 2^T spectrum (T = min(t, 33); 2^33 int32 = 32 GB) lives in
// HBM and is produced in tiled passes of 2^14 int32 (64 KB of shared memory,
// 256 threads, 64 values per thread, stages applied in register rounds of up
// to six bits over a bank-swizzled tile):
//   pass A (bits 0..13): each tile is BUILT from the columns whose pattern
//       falls in it (columns bucketed by tile with a counting sort), so the
//       sparse histogram is never written; empty tiles (all-zero transforms)
//       are not written at all, and the next pass zero-fills their rows from
//       the bucket offsets instead of reading them;
//   middle passes (<= 9 bits, >= 32 consecutive elements per row so every
//       warp access is a full 128-byte line): read, transform, write;
//   the last pass keeps its values in registers and feeds the weight + top-k
//       scan instead of writing (warp-register top-k lists, merged at the end).
// For t > 33 the extra high bits are enumerated (meet-in-the-middle): slice x
// transforms the low 33 bits of the histogram signed by parity(high & x).
// Traffic for t = 32: write 16 GB x (share of nonempty pass-A tiles) + read
// the same + write 16 GB + read 16 GB (64 GB when every tile is nonempty).
// Passes of 6..9 bits (k <= 128) load HBM straight into registers and
// exchange once through shared memory (pass_reg_kernel); narrower passes and
// k > 128 move tiles with 16-byte cp.async (pass_mid_kernel), where a source
// size of 0 zero-fills without a read.
#include "common.cuh"
#include "spectrum.cuh"
#include "topk.cuh"

#include <algorithm>

namespace bmm {
namespace {

constexpr int kTileLog = 14;
constexpr int kTile = 1 << kTileLog;
constexpr int kThr = 256;
constexpr int kPer = kTile / kThr;  // 64
// Pass-A tiles with at most this many patterns are written from the closed
// form of their transform instead of being built and transformed.
constexpr unsigned kDirectMax = 4;
static_assert(kPer == 64, "register rounds assume 64 values per thread");

__device__ __forceinline__ int swz(int k) { return k ^ ((k >> 6) & 31); }

// Middle-pass tile layout: XOR with a multiple of 4 keeps every group of 4
// consecutive elements contiguous (16-byte copies), and is conflict-free for
// both register rounds used there (WL = 8: k >> 8 is the same for a warp;
// WL = 2: the warp's 8 row groups get 8 different XORs).
__device__ __forceinline__ int swzm(int k) { return k ^ (((k >> 8) & 7) << 2); }

template <bool MID>
__device__ __forceinline__ int tswz(int k) {
    return MID ? swzm(k) : swz(k);
}

// One register round: the thread holds the 64 tile elements
// k = base(tid) | (e << WL), e in [0, 64), and applies the stages on e bits
// [S0, S0 + NS).  base places tid's 8 bits outside [WL, WL + 6).
template <int WL>
__device__ __forceinline__ int round_base(int tid) {
    return ((tid >> WL) << (WL + 6)) | (tid & ((1 << WL) - 1));
}

template <int S0, int NS>
__device__ __forceinline__ void bfly(int32_t (&x)[64]) {
#pragma unroll
    for (int s = S0; s < S0 + NS; ++s) {
#pragma unroll
        for (int e = 0; e < 64; ++e)
            if ((e & (1 << s)) == 0) {
                const uint32_t u = (uint32_t)x[e], v = (uint32_t)x[e | (1 << s)];
                x[e] = (int32_t)(u + v);
                x[e | (1 << s)] = (int32_t)(u - v);
            }
    }
}

template <int WL, int S0, int NS, bool MID = false>
__device__ __forceinline__ void round_load(const int32_t* s, int32_t (&x)[64]) {
    const int base = round_base<WL>(threadIdx.x);
#pragma unroll
    for (int e = 0; e < 64; ++e)
        x[e] = s[tswz<MID>(base | (e << WL))];
    bfly<S0, NS>(x);
}

template <int WL, bool MID = false>
__device__ __forceinline__ void round_store(int32_t* s, const int32_t (&x)[64]) {
    const int base = round_base<WL>(threadIdx.x);
#pragma unroll
    for (int e = 0; e < 64; ++e)
        s[tswz<MID>(base | (e << WL))] = x[e];
}

// Offer the 64 register values of the last round to the warp's top-k.
// Global mask of element k of the tile: mask_of(k).
// A per-thread minimum over the 64 weights and one warp vote skip the offers
// whenever no lane can enter the list (the threshold only falls, so the skip
// is exact); after the first tiles that is nearly always.
template <int WL, int E, typename MaskOf>
__device__ __forceinline__ void scan_values(const int32_t (&x)[64], long long N, int kk,
                                            WarpTopK<E>& top, uint32_t& thr, MaskOf mask_of) {
    const int base = round_base<WL>(threadIdx.x);
    if (N < (1ll << 30)) {
        // Every spectrum value is a sum of N terms +-1, so N - x is even and
        // in [0, 2N]: the smallest weight of the 64 values is (N - max x) / 2,
        // one integer max per value.
        // eight independent running maxima, then a tree (no 64-long chain)
        int32_t h8[8];
#pragma unroll
        for (int j = 0; j < 8; ++j)
            h8[j] = x[j];
#pragma unroll
        for (int e = 8; e < 64; ++e)
            h8[e & 7] = max(h8[e & 7], x[e]);
        const int32_t hi = max(max(max(h8[0], h8[1]), max(h8[2], h8[3])),
                               max(max(h8[4], h8[5]), max(h8[6], h8[7])));
        const uint32_t lo2 = (uint32_t)N - (uint32_t)hi;
        if (!__any_sync(kFull, (lo2 >> 1) <= thr))
            return;
    } else {
        long long lo2 = (long long)UINT32_MAX * 2 + 2;
#pragma unroll
        for (int e = 0; e < 64; ++e) {
            const long long w2 = N - (long long)x[e];
            lo2 = (w2 >= 0 && (w2 & 1) == 0 && w2 < lo2) ? w2 : lo2;
        }
        if (!__any_sync(kFull, (lo2 >> 1) <= (long long)thr))
            return;
    }
#pragma unroll
    for (int e = 0; e < 64; ++e) {
        const uint64_t mask = mask_of(base | (e << WL));
        const long long w2 = N - (long long)x[e];
        const bool ok = mask != 0 && w2 >= 0 && (w2 & 1) == 0;
        top.offer(ok, (uint32_t)(w2 >> 1), mask, kk, thr);
    }
}

template <int E>
__device__ __forceinline__ void cta_list_out(WarpTopK<E>& top, uint32_t& thr, int kk,
                                             bmm_candidate* stage, bmm_candidate* out) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    top.store(stage + warp * 32 * E, 32 * E);
    __syncthreads();
    if (warp == 0) {
        for (int ow = 1; ow < kThr / 32; ++ow)
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

// ---------------------------------------------------------------------------
// Column patterns of the active columns (pattern != 0) of t rows (t x W words).
__global__ void patterns_kernel(const uint64_t* __restrict__ rows, int t, int W, long long cols,
                                uint64_t* __restrict__ pats, unsigned long long* __restrict__ count) {
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
        // one atomic per warp for the active columns it found
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

// Counting sort of the patterns by pass-A tile: (p & lowmask) >> 14.
__global__ void tile_count_kernel(const uint64_t* __restrict__ pats,
                                  const unsigned long long* __restrict__ count, int T,
                                  unsigned* __restrict__ counts) {
    const unsigned long long n = *count;
    const uint64_t lowmask = T >= 64 ? ~0ull : ((1ull << T) - 1);
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x)
        atomicAdd(counts + ((pats[i] & lowmask) >> kTileLog), 1u);
}

// Exclusive scan of n counts (one CTA of 1024 threads); offsets has n + 1
// entries; cursor receives a copy of the first n offsets.  Coalesced chunks of
// 1024 counts: warp-shuffle scans, one shared step, a running total.
__global__ void __launch_bounds__(1024) exclusive_scan_kernel(const unsigned* __restrict__ counts,
                                                              long long n,
                                                              unsigned* __restrict__ offsets,
                                                              unsigned* __restrict__ cursor) {
    // Each thread owns a contiguous run of ceil(n / 1024) counts: it sums its
    // run, one block-wide scan of the 1024 sums gives each run's start, and
    // the thread writes its run's offsets (two barriers in all).
    __shared__ unsigned wsum[32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long per = (n + 1023) / 1024;
    const long long b = min(n, (long long)tid * per), e = min(n, b + per);
    const bool vec = (per & 3) == 0;  // runs start on 16-byte boundaries
    unsigned sum = 0;
    if (vec) {
        const uint4* c4 = reinterpret_cast<const uint4*>(counts);
#pragma unroll 8
        for (long long i = b / 4; i < e / 4; ++i) {
            const uint4 v = c4[i];
            sum += v.x + v.y + v.z + v.w;
        }
    } else {
        for (long long i = b; i < e; ++i)
            sum += counts[i];
    }
    unsigned incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned t = __shfl_up_sync(kFull, incl, o);
        if (lane >= o)
            incl += t;
    }
    if (lane == 31)
        wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        unsigned ws = wsum[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned t = __shfl_up_sync(kFull, ws, o);
            if (lane >= o)
                ws += t;
        }
        wsum[lane] = ws;  // inclusive over warps
    }
    __syncthreads();
    unsigned run = (warp ? wsum[warp - 1] : 0u) + incl - sum;
    if (vec) {
        const uint4* c4 = reinterpret_cast<const uint4*>(counts);
        uint4* o4 = reinterpret_cast<uint4*>(offsets);
        uint4* u4 = reinterpret_cast<uint4*>(cursor);
#pragma unroll 4
        for (long long i = b / 4; i < e / 4; ++i) {
            const uint4 v = c4[i];
            uint4 o;
            o.x = run;
            o.y = o.x + v.x;
            o.z = o.y + v.y;
            o.w = o.z + v.z;
            run = o.w + v.w;
            o4[i] = o;
            u4[i] = o;
        }
    } else {
        for (long long i = b; i < e; ++i) {
            const unsigned v = counts[i];
            offsets[i] = run;
            cursor[i] = run;
            run += v;
        }
    }
    if (tid == 0)
        offsets[n] = wsum[31];
}

__global__ void tile_scatter_kernel(const uint64_t* __restrict__ pats,
                                    const unsigned long long* __restrict__ count, int T,
                                    unsigned* __restrict__ cursor, uint64_t* __restrict__ sorted) {
    const unsigned long long n = *count;
    const uint64_t lowmask = T >= 64 ? ~0ull : ((1ull << T) - 1);
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const uint64_t p = pats[i];
        const unsigned pos = atomicAdd(cursor + ((p & lowmask) >> kTileLog), 1u);
        sorted[pos] = p;
    }
}

// ---------------------------------------------------------------------------
// Pass A: bits 0..13.  SPARSE: tile built from its bucketed patterns (value
// (-1)^parity(p >> T & xhi) each); DENSE: tile loaded from d.  LAST: scan
// instead of writing (single-pass spectra, T == 14).
template <bool SPARSE, bool LAST, int E>
__global__ void __launch_bounds__(kThr, LAST ? 1 : 2)
    pass_a_kernel(int32_t* __restrict__ d, int T, long long ntiles,
                  const uint64_t* __restrict__ sorted, const unsigned* __restrict__ offsets,
                  unsigned long long xhi, const unsigned long long* __restrict__ total, int kk,
                  bmm_candidate* __restrict__ cta_out) {
    extern __shared__ __align__(16) int32_t s[];
    const int tid = threadIdx.x;
    WarpTopK<E> top;
    uint32_t thr = 0xffffffffu;
    long long N = 0;
    if (LAST) {
        top.init();
        N = (long long)*total;
    }
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int32_t* gt = d + (size_t)tile * kTile;
        if (SPARSE) {
            const unsigned b0 = offsets[tile], b1 = offsets[tile + 1];
            // An empty tile's transform is zero and is never written: the
            // next pass (bits 14.., the only reader) zero-fills its rows from
            // the same offsets instead of reading them.
            if (b0 == b1 && !LAST)
                continue;
            if (!LAST && b1 - b0 <= kDirectMax) {
                // A tile with few patterns: its transform in closed form,
                // out[k] = sum_j v_j (-1)^popc(p_j & k), k = (e << 8) | tid,
                // with no shared memory; the sign of element e is bit e of a
                // 64-bit parity mask built from the pattern's bits 8..13.
                int32_t x[64];
#pragma unroll
                for (int e = 0; e < 64; ++e)
                    x[e] = 0;
                for (unsigned i = b0; i < b1; ++i) {
                    const uint64_t p = sorted[i];
                    const int32_t v = (T < 64 && (__popcll((p >> T) & xhi) & 1)) ? -1 : 1;
                    const uint32_t ph = (uint32_t)(p >> 8) & 63u;
                    uint64_t m = 0;  // bit e = parity(ph & e) ^ parity(p & tid)
                    if (ph & 1u) m ^= 0xAAAAAAAAAAAAAAAAull;
                    if (ph & 2u) m ^= 0xCCCCCCCCCCCCCCCCull;
                    if (ph & 4u) m ^= 0xF0F0F0F0F0F0F0F0ull;
                    if (ph & 8u) m ^= 0xFF00FF00FF00FF00ull;
                    if (ph & 16u) m ^= 0xFFFF0000FFFF0000ull;
                    if (ph & 32u) m ^= 0xFFFFFFFF00000000ull;
                    if (__popc((uint32_t)p & 255u & (uint32_t)tid) & 1)
                        m = ~m;
                    const uint32_t mlo = (uint32_t)m, mhi = (uint32_t)(m >> 32);
#pragma unroll
                    for (int e = 0; e < 64; ++e) {
                        const uint32_t bit = ((e < 32 ? mlo : mhi) >> (e & 31)) & 1u;
                        x[e] += bit ? -v : v;
                    }
                }
#pragma unroll
                for (int e = 0; e < 64; ++e)
                    gt[(e << 8) | tid] = x[e];  // coalesced: consecutive tid
                continue;
            }
            int4* s4 = reinterpret_cast<int4*>(s);
            for (int i = tid; i < kTile / 4; i += kThr)
                s4[i] = make_int4(0, 0, 0, 0);
            __syncthreads();
            for (unsigned i = b0 + tid; i < b1; i += kThr) {
                const uint64_t p = sorted[i];
                const int v = (T < 64 && (__popcll((p >> T) & xhi) & 1)) ? -1 : 1;
                atomicAdd(s + swz((int)(p & (kTile - 1))), v);
            }
        } else {
            int32_t v[64];
#pragma unroll
            for (int u = 0; u < 64; ++u)
                v[u] = gt[u * kThr + tid];
#pragma unroll
            for (int u = 0; u < 64; ++u)
                s[swz(u * kThr + tid)] = v[u];
        }
        __syncthreads();
        int32_t x[64];
        round_load<0, 0, 6>(s, x);
        round_store<0>(s, x);
        __syncthreads();
        round_load<6, 0, 6>(s, x);
        round_store<6>(s, x);
        __syncthreads();
        round_load<8, 4, 2>(s, x);  // element k = (e << 8) | tid
        if (LAST) {
            const uint64_t tbase = (uint64_t)tile << kTileLog;
            scan_values<8, E>(x, N, kk, top, thr,
                              [&](int k) { return (xhi << T) | tbase | (uint64_t)k; });
        } else {
#pragma unroll
            for (int e = 0; e < 64; ++e)
                gt[(e << 8) | tid] = x[e];  // coalesced: consecutive tid
        }
        __syncthreads();
    }
    if (LAST)
        cta_list_out<E>(top, thr, kk, reinterpret_cast<bmm_candidate*>(s),
                        cta_out + (size_t)blockIdx.x * kk);
}

// Middle / last pass over bits [lo, lo + R), R <= 9: tile = 2^R rows
// (stride 2^lo) x 2^B consecutive elements, B = 14 - R >= 5.  Tiles move
// from HBM straight into the swizzled shared tile with 4-byte cp.async (a
// warp copies 32 consecutive elements of one row: full lines), so no register
// holds a loaded value or its address.  The last pass (one CTA per SM, its
// scan is the longer phase) double-buffers: tile n+1 is in flight while
// tile n is transformed and scanned.
template <int R, bool LAST, int E, bool DB = true>
__global__ void __launch_bounds__(kThr, (LAST && DB) ? 1 : 2)
    pass_mid_kernel(int32_t* __restrict__ d, int T, int lo, unsigned long long xhi,
                    const unsigned long long* __restrict__ total, int kk,
                    bmm_candidate* __restrict__ cta_out,
                    const unsigned* __restrict__ empty_offsets) {
    static_assert(R >= 1 && R <= 9, "R in [1, 9]");
    constexpr int B = kTileLog - R;
    extern __shared__ __align__(16) int32_t s[];
    const int tid = threadIdx.x;
    const long long lowblocks = 1ll << (lo - B);
    const long long ntiles = (1ll << T) >> kTileLog;
    WarpTopK<E> top;
    uint32_t thr = 0xffffffffu;
    long long N = 0;
    if (LAST) {
        top.init();
        N = (long long)*total;
    }
    auto tile_base = [&](long long tl) -> uint64_t {
        return ((uint64_t)(tl / lowblocks) << (lo + R)) | ((uint64_t)(tl % lowblocks) << B);
    };
    // 16-byte copies: chunk c = 4 consecutive elements k = 4c .. 4c+3 of one row
    auto issue = [&](long long tl, int32_t* buf) {
        const uint64_t gb = tile_base(tl);
        const uint32_t sb = (uint32_t)__cvta_generic_to_shared(buf);
#pragma unroll 4
        for (int u = 0; u < kTile / 4 / kThr; ++u) {
            const int k = (u * kThr + tid) * 4;
            const uint64_t gi = gb | ((uint64_t)(k >> B) << lo) | (uint64_t)(k & ((1 << B) - 1));
            // rows of pass-A tiles that were empty (never written) are
            // zero-filled: 0 source bytes, nothing is read
            uint32_t src_bytes = 16;
            if (empty_offsets) {
                const uint64_t at = gi >> kTileLog;
                src_bytes = empty_offsets[at] == empty_offsets[at + 1] ? 0u : 16u;
            }
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(
                             sb + 4u * (uint32_t)swzm(k)),
                         "l"(d + gi), "r"(src_bytes)
                         : "memory");
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    long long tile = blockIdx.x;
    if (LAST && DB && tile < ntiles)
        issue(tile, s);
    for (int it = 0; tile < ntiles; ++it, tile += gridDim.x) {
        int32_t* cur = (LAST && DB) ? s + (it & 1) * kTile : s;
        if (LAST && DB) {
            const long long nxt = tile + gridDim.x;
            if (nxt < ntiles) {
                issue(nxt, s + ((it + 1) & 1) * kTile);
                asm volatile("cp.async.wait_group 1;" ::: "memory");
            } else {
                asm volatile("cp.async.wait_group 0;" ::: "memory");
            }
        } else {
            issue(tile, s);
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        __syncthreads();
        const uint64_t gbase = tile_base(tile);
        auto gidx = [&](int k) -> uint64_t {
            return gbase | ((uint64_t)(k >> B) << lo) | (uint64_t)(k & ((1 << B) - 1));
        };
        int32_t x[64];
        if constexpr (R > 6) {
            round_load<8, 0, 6, true>(cur, x);  // k bits 8..13 = the top six stage bits
            round_store<8, true>(cur, x);
            __syncthreads();
            round_load<2, B - 2, R - 6, true>(cur, x);
            if (LAST) {
                scan_values<2, E>(x, N, kk, top, thr,
                                  [&](int k) { return (xhi << T) | gidx(k); });
            } else {
                round_store<2, true>(cur, x);
                __syncthreads();
#pragma unroll 4
                for (int u = 0; u < kTile / 4 / kThr; ++u) {
                    const int k = (u * kThr + tid) * 4;
                    *reinterpret_cast<int4*>(d + gidx(k)) =
                        *reinterpret_cast<const int4*>(cur + swzm(k));
                }
            }
        } else {
            round_load<8, B - 8, R, true>(cur, x);  // stage bits [B, 14) all inside k bits 8..13
            if (LAST) {
                scan_values<8, E>(x, N, kk, top, thr,
                                  [&](int k) { return (xhi << T) | gidx(k); });
            } else {
#pragma unroll
                for (int e = 0; e < 64; ++e)
                    d[gidx((e << 8) | tid)] = x[e];
            }
        }
        __syncthreads();
    }
    if (LAST)
        cta_list_out<E>(top, thr, kk, reinterpret_cast<bmm_candidate*>(s),
                        cta_out + (size_t)blockIdx.x * kk);
}

// ---------------------------------------------------------------------------
// Register-resident passes (6 <= R <= 9 row bits, tiles of 2^R rows x 2^B
// consecutive entries, B = 14 - R >= 5).  Lane = column within a 32-column
// block, so every warp load or store of one row is one full 128-byte line,
// and values go from HBM straight into registers:
//   round 1: element e of a thread is row e | rw << 6 (the six low row bits
//            in registers, six stages with no shared memory);
//   round 2 (R > 6): one exchange through shared memory, laid out row-major
//            (lane = column: conflict-free without a swizzle), then the R - 6
//            high row stages in registers.
// 8 bytes per value cross shared memory (the cp.async passes move 16-20).
// Two CTAs per SM (one 64-value register tile per thread, <= 128 registers):
// while one CTA waits on its loads the other transforms (measured faster than
// one CTA per SM that prefetches the next tile into a second register set,
// the PF variant).  Each
// add of a butterfly is an IMAD (x * one + y, `one` == 1 at run time) on the
// FMA pipe and each subtract an IADD on the ALU pipe.
template <int R>
struct RegTile {
    static constexpr int B = kTileLog - R;  // log2 columns per row, 5..8
    static constexpr int CWB = B - 5;       // warp bits choosing the 32-column block
    static constexpr int RWB = R - 6;       // warp bits choosing row bits (both rounds)
    static_assert(R >= 6 && R <= 9, "register passes take 6..9 row bits");
    // row of element e = the e part | the warp part
    __device__ static __forceinline__ int row1_e(int e) { return e; }
    __device__ static __forceinline__ int row1_w(int rw) { return rw << 6; }
    __device__ static __forceinline__ int row2_e(int e) {
        return (e >> RWB) | ((e & ((1 << RWB) - 1)) << 6);
    }
    __device__ static __forceinline__ int row2_w(int rw) { return rw << (12 - R); }
    __device__ static __forceinline__ int row1(int e, int rw) { return row1_e(e) | row1_w(rw); }
    __device__ static __forceinline__ int row2(int e, int rw) { return row2_e(e) | row2_w(rw); }
    __device__ static __forceinline__ int last_e(int e) { return R > 6 ? row2_e(e) : row1_e(e); }
    __device__ static __forceinline__ int last_w(int rw) { return R > 6 ? row2_w(rw) : row1_w(rw); }
    __device__ static __forceinline__ int row_last(int e, int rw) { return last_e(e) | last_w(rw); }
};

// Byte stride between rows, 4 << lo < 2^32 (lo <= 27), read through an asm
// move so that the compiler forms each address in the tile loop (one wide
// IMAD) instead of keeping 64 loop-invariant 64-bit offsets in registers.
__device__ __forceinline__ uint32_t row_stride_bytes(int lo) {
    uint32_t sb;
    asm volatile("mov.b32 %0, %1;" : "=r"(sb) : "r"(4u << lo));
    return sb;
}

__device__ __forceinline__ uint32_t mad_one(uint32_t a, uint32_t one, uint32_t c) {
    uint32_t d;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(one), "r"(c));
    return d;
}

template <int S0, int NS>
__device__ __forceinline__ void bfly_split(int32_t (&x)[64], uint32_t one) {
#pragma unroll
    for (int s = S0; s < S0 + NS; ++s) {
#pragma unroll
        for (int e = 0; e < 64; ++e)
            if ((e & (1 << s)) == 0) {
                const uint32_t u = (uint32_t)x[e], v = (uint32_t)x[e | (1 << s)];
                x[e] = (int32_t)mad_one(v, one, u);
                x[e | (1 << s)] = (int32_t)(u - v);
            }
    }
}

// Offer a tile's 64 register values (rows row_last(e), column col) to the
// warp top-k.  Values above `lim` = min(own threshold, *gthr) are dropped:
// *gthr is the smallest threshold weight any warp of the launch has published,
// i.e. some warp holds k candidates of at most that weight, so a value above
// it is not among the k best of the window (values at or below it are always
// offered, and each warp's list keeps the k best it was offered, so the merged
// lists stay exact).  The prefilter is one integer max per value (N - WHT is
// even and in [0, 2N]); when some lane may pass it, the thread parks its
// values at its own shared-memory positions (no other thread touches them
// before the next barrier) and walks them in a rolled loop, one warp vote per
// value, offering only where a lane is at or below the limit.
template <int R, int E>
__device__ __forceinline__ void reg_offer(const int32_t (&x)[64], int rw, int col, uint64_t mbase,
                                          int lo, long long N, int kk, WarpTopK<E>& top,
                                          uint32_t& thr, int32_t* s, unsigned* gthr) {
    using M = RegTile<R>;
    uint32_t g;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(g) : "l"(gthr) : "memory");
    uint32_t lim = min(thr, g);
    if (N < (1ll << 30)) {
        int32_t h8[8];
#pragma unroll
        for (int j = 0; j < 8; ++j)
            h8[j] = x[j];
#pragma unroll
        for (int e = 8; e < 64; ++e)
            h8[e & 7] = max(h8[e & 7], x[e]);
        const int32_t hi = max(max(max(h8[0], h8[1]), max(h8[2], h8[3])),
                               max(max(h8[4], h8[5]), max(h8[6], h8[7])));
        const uint32_t lo2 = (uint32_t)N - (uint32_t)hi;
        if (!__any_sync(kFull, (lo2 >> 1) <= lim))
            return;
    }
#pragma unroll
    for (int e = 0; e < 64; ++e)
        s[(M::row_last(e, rw) << M::B) | col] = x[e];
    const uint32_t thr0 = thr;
    long long vmin = N - 2 * (long long)lim;  // weight <= lim  <=>  value >= vmin
#pragma unroll 1
    for (int e = 0; e < 64; ++e) {
        const int row = M::row_last(e, rw);
        const int32_t v = s[(row << M::B) | col];
        if (!__any_sync(kFull, (long long)v >= vmin))
            continue;
        const uint64_t mask = mbase | ((uint64_t)row << lo);
        const long long w2 = N - (long long)v;
        const bool ok = mask != 0 && w2 >= 0 && (w2 & 1) == 0;
        top.offer(ok, (uint32_t)(w2 >> 1), mask, kk, thr);
        lim = min(thr, g);
        vmin = N - 2 * (long long)lim;
    }
    if (thr < thr0 && (threadIdx.x & 31) == 0)
        atomicMin(gthr, thr);
}

// One pass over the row bits [lo, lo + R).  empty_bits (first pass after
// pass A only, lo == 14): bit i of word j set = pass-A tile 64 j + i was
// never written; its rows are zeros and are not read.
// LO > 0: the pass's low bit is the compile-time LO (the first pass after
// pass A has lo = 14): row addresses are then a base plus immediate offsets.
template <int R, bool LAST, int E, bool PF = true, int LO = 0>
__global__ void __launch_bounds__(kThr, PF ? 1 : 2)
    pass_reg_kernel(int32_t* __restrict__ d, int T, int lo, unsigned long long xhi,
                    const unsigned long long* __restrict__ total, int kk,
                    bmm_candidate* __restrict__ cta_out, const uint64_t* __restrict__ empty_bits,
                    unsigned* __restrict__ gthr, uint32_t one) {
    using M = RegTile<R>;
    if constexpr (LO > 0)
        lo = LO;
    constexpr int B = M::B;
    extern __shared__ __align__(16) int32_t s[];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int cw = w & ((1 << M::CWB) - 1), rw = w >> M::CWB;
    const int col = lane | (cw << 5);
    const long long lowblocks = 1ll << (lo - B);
    const long long ntiles = (1ll << T) >> kTileLog;
    WarpTopK<E> top;
    uint32_t thr = 0xffffffffu;
    long long N = 0;
    if (LAST) {
        top.init();
        N = (long long)*total;
    }
    auto tile_base = [&](long long tl) -> uint64_t {
        return ((uint64_t)(tl / lowblocks) << (lo + R)) | ((uint64_t)(tl % lowblocks) << B);
    };
    auto load = [&](long long tl, int32_t (&x)[64]) {
        const uint64_t gb = tile_base(tl);
        uint64_t eb = 0;
        if (empty_bits)
            eb = __ldg(empty_bits + ((gb >> 20) | (uint64_t)rw));
        const char* p = reinterpret_cast<const char*>(
            d + (gb | ((uint64_t)M::row1_w(rw) << lo) | (uint64_t)col));
        const uint32_t sb = LO > 0 ? (4u << LO) : row_stride_bytes(lo);
        if (eb == 0) {  // warp-uniform: rw is one per warp
#pragma unroll
            for (int e = 0; e < 64; ++e)
                x[e] = __ldcs(reinterpret_cast<const int32_t*>(
                    p + (uint64_t)sb * (uint32_t)M::row1_e(e)));
        } else {
#pragma unroll
            for (int e = 0; e < 64; ++e)
                x[e] = ((eb >> e) & 1ull)
                           ? 0
                           : __ldcs(reinterpret_cast<const int32_t*>(
                                 p + (uint64_t)sb * (uint32_t)M::row1_e(e)));
        }
    };
    auto process = [&](long long tl, int32_t (&x)[64]) {
        bfly_split<0, 6>(x, one);
        if constexpr (R > 6) {
            __syncthreads();  // the previous tile's round-2 reads are done
#pragma unroll
            for (int e = 0; e < 64; ++e)
                s[(M::row1(e, rw) << B) | col] = x[e];
            __syncthreads();
#pragma unroll
            for (int e = 0; e < 64; ++e)
                x[e] = s[(M::row2(e, rw) << B) | col];
            bfly_split<0, R - 6>(x, one);
        }
        const uint64_t gb = tile_base(tl);
        if constexpr (LAST) {
            reg_offer<R, E>(x, rw, col, (xhi << T) | gb | (uint64_t)col, lo, N, kk, top, thr,
                            s, gthr);
        } else {
            char* p = reinterpret_cast<char*>(
                d + (gb | ((uint64_t)M::last_w(rw) << lo) | (uint64_t)col));
            const uint32_t sb = LO > 0 ? (4u << LO) : row_stride_bytes(lo);
#pragma unroll
            for (int e = 0; e < 64; ++e)
                __stcs(reinterpret_cast<int32_t*>(p + (uint64_t)sb * (uint32_t)M::last_e(e)),
                       x[e]);
        }
    };
    const long long G = gridDim.x;
    if constexpr (!PF) {
        // two CTAs per SM, one register tile each: the other CTA hides the loads
        for (long long tile = blockIdx.x; tile < ntiles; tile += G) {
            int32_t x[64];
            load(tile, x);
            process(tile, x);
        }
        if (LAST)
            cta_list_out<E>(top, thr, kk, reinterpret_cast<bmm_candidate*>(s),
                            cta_out + (size_t)blockIdx.x * kk);
        return;
    }
    int32_t xa[64], xb[64];
    long long tile = blockIdx.x;
    if (tile < ntiles)
        load(tile, xa);
    while (tile < ntiles) {
        const long long t1 = tile + G;
        if (t1 < ntiles)
            load(t1, xb);
        process(tile, xa);
        if (t1 >= ntiles)
            break;
        const long long t2 = t1 + G;
        if (t2 < ntiles)
            load(t2, xa);
        process(t1, xb);
        tile = t2;
    }
    if (LAST)
        cta_list_out<E>(top, thr, kk, reinterpret_cast<bmm_candidate*>(s),
                        cta_out + (size_t)blockIdx.x * kk);
}

// empty_bits[j] bit i = pass-A tile 64 j + i holds no pattern.
__global__ void empty_bits_kernel(const unsigned* __restrict__ offsets, long long ntiles,
                                  uint64_t* __restrict__ bits) {
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j * 64 >= ntiles)
        return;
    uint64_t b = 0;
    for (int i = 0; i < 64 && j * 64 + i < ntiles; ++i)
        b |= (uint64_t)(offsets[j * 64 + i] == offsets[j * 64 + i + 1]) << i;
    bits[j] = b;
}

// Small spectra (T < 14): one CTA, everything in shared memory.
template <int E>
__global__ void __launch_bounds__(kThr)
    small_spectrum_kernel(const uint64_t* __restrict__ pats,
                          const unsigned long long* __restrict__ count, int t, int kk,
                          bmm_candidate* __restrict__ out) {
    extern __shared__ __align__(16) int32_t s[];
    const int n = 1 << t;
    const int tid = threadIdx.x;
    for (int i = tid; i < n; i += kThr)
        s[i] = 0;
    __syncthreads();
    const unsigned long long cnt = *count;
    for (unsigned long long i = tid; i < cnt; i += kThr)
        atomicAdd(s + pats[i], 1);
    __syncthreads();
    for (int st = 0; st < t; ++st) {
        for (int q = tid; q < n / 2; q += kThr) {
            const int j0 = ((q >> st) << (st + 1)) | (q & ((1 << st) - 1));
            const int j1 = j0 | (1 << st);
            const int32_t u = s[j0], v = s[j1];
            s[j0] = u + v;
            s[j1] = u - v;
        }
        __syncthreads();
    }
    WarpTopK<E> top;
    top.init();
    uint32_t thr = 0xffffffffu;
    const long long N = (long long)cnt;
    for (int b0 = tid & ~31; b0 < n; b0 += kThr) {
        const int m = b0 + (tid & 31);
        bool ok = m >= 1 && m < n;
        uint32_t w = 0xffffffffu;
        if (ok) {
            const long long w2 = N - (long long)s[m];
            ok = w2 >= 0 && (w2 & 1) == 0;
            w = (uint32_t)(w2 >> 1);
        }
        top.offer(ok, w, (uint64_t)m, kk, thr);
    }
    __syncthreads();
    cta_list_out<E>(top, thr, kk, reinterpret_cast<bmm_candidate*>(s), out);
}

template <typename F>
int dispatch_e(int kk, F&& f) {
    if (kk <= 32)
        return f(std::integral_constant<int, 1>{});
    if (kk <= 128)
        return f(std::integral_constant<int, 4>{});
    if (kk <= 1024)
        return f(std::integral_constant<int, 32>{});
    return fail(BMM_EINVAL, "spectrum search: k must be <= 1024");
}

// Dynamic shared memory of a pass kernel: the 64 KB tile, or for the last
// pass the larger of the tile and the staging of 8 warp lists of 32*E.
constexpr size_t pass_smem(bool last, int E) {
    return last && (size_t)(kThr / 32) * 32 * E * sizeof(bmm_candidate) > kTile * sizeof(int32_t)
               ? (size_t)(kThr / 32) * 32 * E * sizeof(bmm_candidate)
               : kTile * sizeof(int32_t);
}

// The last middle pass double-buffers its tiles (one CTA per SM), or runs two
// single-buffered CTAs per SM within 128 registers (g_spectrum_last_db = 0).
constexpr size_t mid_smem(bool last, int E, bool db = true) {
    return last ? (pass_smem(true, E) > (db ? 2 : 1) * kTile * sizeof(int32_t)
                       ? pass_smem(true, E)
                       : (db ? 2 : 1) * kTile * sizeof(int32_t))
                : kTile * sizeof(int32_t);
}

// Register-resident passes for R >= 6 row bits and lists of <= 128 entries
// (WarpTopK<32> does not fit beside two register tiles).
bool use_reg_pass(int R, int kk) { return g_spectrum_reg != 0 && R >= 6 && kk <= 128; }

template <int E>
int launch_reg(int R, bool last, int32_t* d, int T, int lo, unsigned long long xhi,
               const unsigned long long* total, int kk, bmm_candidate* lists, int grid,
               cudaStream_t st, const uint64_t* empty_bits, unsigned* gthr) {
    const size_t smem = pass_smem(last, E);
#define BMM_REG(RR)                                                                               \
    case RR: {                                                                                    \
        auto k = g_spectrum_reg == 2                                                              \
                     ? (last ? pass_reg_kernel<RR, true, E, false>                                \
                             : (lo == kTileLog ? pass_reg_kernel<RR, false, E, false, kTileLog>   \
                                               : pass_reg_kernel<RR, false, E, false>))           \
                     : (last ? pass_reg_kernel<RR, true, E> : pass_reg_kernel<RR, false, E>);    \
        BMM_CUDA_TRY(                                                                             \
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));     \
        k<<<grid, kThr, smem, st>>>(d, T, lo, xhi, total, kk, lists, empty_bits, gthr, 1u);       \
        BMM_CUDA_TRY(cudaGetLastError());                                                         \
        return BMM_OK;                                                                            \
    }
    switch (R) {
        BMM_REG(6)
        BMM_REG(7)
        BMM_REG(8)
        BMM_REG(9)
    }
#undef BMM_REG
    return fail(BMM_EINVAL, "spectrum: bad pass width");
}

template <int E>
int launch_mid(int R, bool last, int32_t* d, int T, int lo, unsigned long long xhi,
               const unsigned long long* total, int kk, bmm_candidate* lists, int grid,
               cudaStream_t st, const unsigned* empty_offsets = nullptr,
               const uint64_t* empty_bits = nullptr, unsigned* gthr = nullptr) {
    if constexpr (E <= 4) {
        if (use_reg_pass(R, kk))
            return launch_reg<E>(R, last, d, T, lo, xhi, total, kk, lists, grid, st, empty_bits,
                                 gthr);
    }
    const bool db = g_spectrum_last_db != 0 || E > 4;  // E = 32 lists need the registers
    const size_t smem = mid_smem(last, E, db);
#define BMM_MID(RR)                                                                               \
    case RR: {                                                                                    \
        auto k = last ? (db ? pass_mid_kernel<RR, true, E, true>                                  \
                            : pass_mid_kernel<RR, true, E, false>)                                \
                      : pass_mid_kernel<RR, false, E>;                                            \
        BMM_CUDA_TRY(                                                                             \
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));     \
        k<<<grid, kThr, smem, st>>>(d, T, lo, xhi, total, kk, lists, empty_offsets);              \
        BMM_CUDA_TRY(cudaGetLastError());                                                         \
        return BMM_OK;                                                                            \
    }
    switch (R) {
        BMM_MID(1)
        BMM_MID(2)
        BMM_MID(3)
        BMM_MID(4)
        BMM_MID(5)
        BMM_MID(6)
        BMM_MID(7)
        BMM_MID(8)
        BMM_MID(9)
    }
#undef BMM_MID
    return fail(BMM_EINVAL, "spectrum: bad pass width");
}

// Split the bits above the first 14 into passes of at most 9, as even as possible.
void plan_mid(int T, int* widths, int* n) {
    const int rest = T - kTileLog;
    const int passes = (rest + 8) / 9;
    *n = passes;
    for (int i = 0; i < passes; ++i)
        widths[i] = rest / passes + (i < rest % passes ? 1 : 0);
}

int grid_for(Workspace* ws, long long ntiles) {
    long long g = (long long)ws->sm_count * 2;  // 2 x 64 KB tiles per SM
    return (int)(ntiles < g ? ntiles : g);
}

// Grid of a pass of width R after pass A: register passes and the
// double-buffered last pass run one CTA per SM.
int grid_mid(Workspace* ws, long long ntiles, int R, bool last, int kk) {
    int per_sm = 2;
    if (use_reg_pass(R, kk))
        per_sm = g_spectrum_reg == 2 ? 2 : 1;
    else if (last && (g_spectrum_last_db != 0 || kk > 128))
        per_sm = 1;
    const long long g = (long long)ws->sm_count * per_sm;
    return (int)(ntiles < g ? ntiles : g);
}

}  // namespace

int g_spectrum_low_bits = -1;
int g_spectrum_last_db = 1;
int g_spectrum_reg = 2;
int g_spectrum_shape_low_bits[41] = {-1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1,
                                     -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1,
                                     -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1};

int spectrum_low_bits(int t) {
    const int top = t < 33 ? t : 33;
    if (t <= kTileLog || t > 40)
        return top;
    int want = g_spectrum_low_bits > 0 ? g_spectrum_low_bits : g_spectrum_shape_low_bits[t];
    if (want <= 0)
        return top;
    return want < kTileLog ? kTileLog : (want > top ? top : want);
}

int spectrum_topk_launch(Workspace* ws, const uint64_t* d_rows, int t, int W, long long cols,
                         int kk, bmm_candidate* d_out, cudaStream_t stream) {
    return spectrum_topk_slices(ws, d_rows, t, W, cols, kk, -1, 0, -1, d_out, stream);
}

int spectrum_topk_slices(Workspace* ws, const uint64_t* d_rows, int t, int W, long long cols,
                         int kk, int low_bits, long long slice_begin, long long slice_end,
                         bmm_candidate* d_out, cudaStream_t stream) {
    if (t < 1 || t > 40)
        return fail(BMM_EINVAL, "spectrum search: t must be in [1, 40]");
    const int T = low_bits < 0 ? spectrum_low_bits(t) : low_bits;
    if (T > (t < 33 ? t : 33) || (T < kTileLog && T != t))
        return fail(BMM_EINVAL, "spectrum search: low_bits must be in [14, min(t, 33)]");
    const int H = t - T;
    const long long all_slices = 1ll << H;
    if (slice_end < 0)
        slice_end = all_slices;
    if (slice_begin < 0 || slice_begin >= slice_end || slice_end > all_slices)
        return fail(BMM_EINVAL, "spectrum search: slice range [%lld, %lld) outside [0, %lld)",
                    slice_begin, slice_end, all_slices);
    void *pats = nullptr, *cnt = nullptr;
    BMM_TRY(ws_buffer(ws, kSlotAux, (size_t)(cols > 0 ? cols : 1) * 8, &pats));
    BMM_TRY(ws_buffer(ws, kSlotCounter, 16, &cnt));
    BMM_CUDA_TRY(cudaMemsetAsync(cnt, 0, 8, stream));
    // bytes 8..11: the smallest threshold weight published by the last pass
    unsigned* gthr = reinterpret_cast<unsigned*>(static_cast<char*>(cnt) + 8);
    BMM_CUDA_TRY(cudaMemsetAsync(gthr, 0xff, 4, stream));
    {
        long long blocks = (cols + 255) / 256;
        if (blocks > (long long)ws->sm_count * 8)
            blocks = (long long)ws->sm_count * 8;
        patterns_kernel<<<(unsigned)(blocks > 0 ? blocks : 1), 256, 0, stream>>>(
            d_rows, t, W, cols, (uint64_t*)pats, (unsigned long long*)cnt);
        BMM_CUDA_TRY(cudaGetLastError());
    }
    const unsigned long long* total = (const unsigned long long*)cnt;
    if (T < kTileLog) {
        return dispatch_e(kk, [&](auto Ec) -> int {
            constexpr int E = decltype(Ec)::value;
            const size_t smem0 = ((size_t)1 << T) * 4;
            const size_t smem1 = (size_t)8 * 32 * E * sizeof(bmm_candidate);
            const size_t smem = smem0 > smem1 ? smem0 : smem1;
            auto k = small_spectrum_kernel<E>;
            BMM_CUDA_TRY(
                cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k<<<1, kThr, smem, stream>>>((const uint64_t*)pats, total, t, kk, d_out);
            BMM_CUDA_TRY(cudaGetLastError());
            return BMM_OK;
        });
    }
    // bucket the patterns by pass-A tile
    const long long ntiles = 1ll << (T - kTileLog);
    void *counts = nullptr, *offsets = nullptr, *cursor = nullptr, *sorted = nullptr;
    BMM_TRY(ws_buffer(ws, kSlotIdx, (size_t)ntiles * 4, &counts));
    BMM_TRY(ws_buffer(ws, kSlotExtra0, (size_t)(ntiles + 1) * 4, &offsets));
    BMM_TRY(ws_buffer(ws, kSlotExtra1, (size_t)ntiles * 4, &cursor));
    BMM_TRY(ws_buffer(ws, kSlotKeys, (size_t)(cols > 0 ? cols : 1) * 8, &sorted));
    BMM_CUDA_TRY(cudaMemsetAsync(counts, 0, (size_t)ntiles * 4, stream));
    const int pblocks = ws->sm_count * 4;
    tile_count_kernel<<<pblocks, 256, 0, stream>>>((const uint64_t*)pats, total, T,
                                                   (unsigned*)counts);
    exclusive_scan_kernel<<<1, 1024, 0, stream>>>((const unsigned*)counts, ntiles,
                                                  (unsigned*)offsets, (unsigned*)cursor);
    tile_scatter_kernel<<<pblocks, 256, 0, stream>>>((const uint64_t*)pats, total, T,
                                                     (unsigned*)cursor, (uint64_t*)sorted);
    BMM_CUDA_TRY(cudaGetLastError());

    void* spec = nullptr;
    if (T > kTileLog)
        BMM_TRY(ws_buffer(ws, kSlotSpec, ((size_t)1 << T) * 4, &spec));
    int widths[4], nmid = 0;
    plan_mid(T, widths, &nmid);
    const int grid_a = grid_for(ws, ntiles);  // every pass has 2^(T-14) tiles
    const int grid_last = nmid ? grid_mid(ws, ntiles, widths[nmid - 1], true, kk) : grid_a;
    // pass-A tiles that hold no pattern, one bit each, for a register first pass
    uint64_t* empty_bits = nullptr;
    if (nmid && use_reg_pass(widths[0], kk)) {
        const long long words = (ntiles + 63) / 64;
        BMM_TRY(ws_buffer(ws, kSlotEmptyBits, (size_t)words * 8, (void**)&empty_bits));
        empty_bits_kernel<<<(unsigned)((words + 255) / 256), 256, 0, stream>>>(
            (const unsigned*)offsets, ntiles, empty_bits);
        BMM_CUDA_TRY(cudaGetLastError());
    }
    const long long slices = slice_end - slice_begin;
    bmm_candidate *lists = nullptr, *slice_lists = nullptr;
    BMM_TRY(ws_buffer(ws, kSlotCand, (size_t)grid_last * kk * sizeof(bmm_candidate),
                      (void**)&lists));
    if (slices > 1)
        BMM_TRY(ws_buffer(ws, kSlotSlices, (size_t)slices * kk * sizeof(bmm_candidate),
                          (void**)&slice_lists));
    const size_t smem = kTile * sizeof(int32_t);
    return dispatch_e(kk, [&](auto Ec) -> int {
        constexpr int E = decltype(Ec)::value;
        for (long long x = slice_begin; x < slice_end; ++x) {
            bmm_candidate* dst =
                slices > 1 ? slice_lists + (size_t)(x - slice_begin) * kk : d_out;
            if (nmid == 0) {
                auto k = pass_a_kernel<true, true, E>;
                const size_t lsmem = pass_smem(true, E);
                BMM_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)lsmem));
                k<<<grid_a, kThr, lsmem, stream>>>((int32_t*)spec, T, ntiles,
                                                  (const uint64_t*)sorted,
                                                  (const unsigned*)offsets, (unsigned long long)x,
                                                  total, kk, lists);
                BMM_CUDA_TRY(cudaGetLastError());
            } else {
                auto k = pass_a_kernel<true, false, E>;
                BMM_CUDA_TRY(
                    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                k<<<grid_a, kThr, smem, stream>>>((int32_t*)spec, T, ntiles,
                                                  (const uint64_t*)sorted,
                                                  (const unsigned*)offsets, (unsigned long long)x,
                                                  total, kk, lists);
                BMM_CUDA_TRY(cudaGetLastError());
                int lo = kTileLog;
                for (int i = 0; i < nmid; ++i) {
                    const bool last = i == nmid - 1;
                    BMM_TRY(launch_mid<E>(widths[i], last, (int32_t*)spec, T, lo,
                                          (unsigned long long)x, total, kk, lists,
                                          last ? grid_last
                                               : grid_mid(ws, ntiles, widths[i], false, kk),
                                          stream, i == 0 ? (const unsigned*)offsets : nullptr,
                                          i == 0 ? empty_bits : nullptr, gthr));
                    lo += widths[i];
                }
            }
            BMM_TRY(merge_topk_lists(lists, grid_last, kk, dst, stream, gthr));
        }
        if (slices > 1)
            BMM_TRY(merge_topk_lists(slice_lists, (int)slices, kk, d_out, stream, gthr));
        return BMM_OK;
    });
}

// Dense in-place transform of 2^t int32 (t >= 14) with the same passes.
int spectrum_dense_fwht(Workspace* ws, int32_t* d, int t, cudaStream_t stream) {
    const long long ntiles = 1ll << (t - kTileLog);
    const size_t smem = kTile * sizeof(int32_t);
    auto ka = pass_a_kernel<false, false, 1>;
    BMM_CUDA_TRY(cudaFuncSetAttribute(ka, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    ka<<<grid_for(ws, ntiles), kThr, smem, stream>>>(d, t, ntiles, nullptr, nullptr, 0, nullptr, 0,
                                                     nullptr);
    BMM_CUDA_TRY(cudaGetLastError());
    int widths[4], nmid = 0;
    plan_mid(t, widths, &nmid);
    int lo = kTileLog;
    for (int i = 0; i < nmid; ++i) {
        BMM_TRY(launch_mid<1>(widths[i], false, d, t, lo, 0, nullptr, 1, nullptr,
                              grid_mid(ws, ntiles, widths[i], false, 1), stream));
        lo += widths[i];
    }
    return BMM_OK;
}

}  // namespace bmm
