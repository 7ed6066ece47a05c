// Gray-code exhaustive search on sm_100a.
//
// Reference behaviour: BruteforceSearch::search / sweep_prefix
// (src/search/bruteforce_search.cpp:126-170,300-329) and the CUDA twin
// bruteforce_persistent_kernel (src/search/cuda_bruteforce_launch.cu:131-296):
// split the t-bit mask into a high prefix and a low chunk, start each prefix
// from the XOR of its high rows, then walk the 2^chunk low states in
// reflected-Gray order (one row XOR + full popcount per step).
//
// B200 design (not the reference's): one LANE owns one prefix and keeps the
// whole current row (WPL words) in registers, so a step is WPL XOR+POPC with
// no shuffle; every lane of a warp flips the same row at the same step, so
// the row words come from shared memory as broadcast 128-bit loads.  Rows
// wider than 64 words are split over G lanes (words [g*WPL, (g+1)*WPL) in
// lane g of the group) with a log2(G) shuffle reduction per step.  Top-k
// lives in the warp's registers (WarpTopK); top-1 per target is a register
// min folded with one 64-bit atomicMin per warp.
#include "common.cuh"
#include "gray.cuh"
#include "popc.cuh"
#include "topk.cuh"

#include <cmath>
#include <mutex>
#include <vector>

namespace bmm {
namespace {

constexpr int kThreads = 128;

template <int WPL>
__device__ __forceinline__ uint32_t xor_row_popc(uint64_t (&cur)[WPL], const uint64_t* srow) {
    const ulonglong2* p = reinterpret_cast<const ulonglong2*>(srow);
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < WPL / 2; ++i) {
        const ulonglong2 v = p[i];
        cur[2 * i] ^= v.x;
        cur[2 * i + 1] ^= v.y;
        s += __popcll(cur[2 * i]) + __popcll(cur[2 * i + 1]);
    }
    return s;
}

template <int WPL>
__device__ __forceinline__ void xor_row(uint64_t (&cur)[WPL], const uint64_t* srow) {
    const ulonglong2* p = reinterpret_cast<const ulonglong2*>(srow);
#pragma unroll
    for (int i = 0; i < WPL / 2; ++i) {
        const ulonglong2 v = p[i];
        cur[2 * i] ^= v.x;
        cur[2 * i + 1] ^= v.y;
    }
}

template <int WPL>
__device__ __forceinline__ uint32_t popc_row(const uint64_t (&cur)[WPL]) {
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < WPL; ++i)
        s += __popcll(cur[i]);
    return s;
}

template <int G>
__device__ __forceinline__ uint32_t group_sum(uint32_t v) {
#pragma unroll
    for (int o = 1; o < G; o <<= 1)
        v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// Shared-memory row layout: a row is G lane slices of WPL words; with G > 1
// each slice is followed by 2 pad words (16 bytes), so the G lanes of a group
// read their slices' 16-byte chunks from different banks in one request.
__host__ __device__ constexpr int lane_stride(int wpl, int g) { return wpl + (g > 1 ? 2 : 0); }
__host__ __device__ constexpr int row_stride(int wpl, int g) { return g * lane_stride(wpl, g); }

// Stage `nrows` rows (row r from row_of(r), W words) into shared memory in
// that layout (row stride row_stride(WPL, G) words), zero padded past W.
template <int WPL, int G, typename RowOf>
__device__ __forceinline__ void stage_rows(uint64_t* srow, int nrows, int W, RowOf row_of) {
    constexpr int RW = WPL * G, LS = lane_stride(WPL, G), SW = row_stride(WPL, G);
    for (int i = threadIdx.x; i < nrows * RW; i += blockDim.x) {
        const int r = i / RW, w = i % RW;
        srow[r * SW + (w / WPL) * LS + w % WPL] = w < W ? row_of(r)[w] : 0ull;
    }
}

// ---------------------------------------------------------------------------
// Window search: top-kk over all nonzero masks of t rows.
// rows: t x W words (device, packed in window order).
template <int WPL, int G, int E, int NHB>
__global__ void __launch_bounds__(kThreads)
    gray_window_kernel(const uint64_t* __restrict__ rows, int t, int W, int chunk,
                       unsigned long long n_prefix, int kk, bmm_candidate* __restrict__ cta_out) {
    extern __shared__ __align__(16) uint64_t srow[];
    constexpr int SW = row_stride(WPL, G);
    stage_rows<WPL, G>(srow, t, W, [&](int r) { return rows + (size_t)r * W; });
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const int gl = lane % G;  // lane within the group
    const unsigned long long groups_per_cta = kThreads / G;
    const unsigned long long stride_groups = groups_per_cta * gridDim.x;
    unsigned long long p = blockIdx.x * groups_per_cta + threadIdx.x / G;
    const int hb = t - chunk;
    const uint32_t states = 1u << chunk;

    WarpTopK<E> top;
    top.init();
    uint32_t thr = 0xffffffffu;

    const uint64_t* my = srow + gl * lane_stride(WPL, G);
    while (__any_sync(kFull, p < n_prefix)) {
        const bool valid = p < n_prefix && gl == 0;
        uint64_t cur[WPL];
#pragma unroll
        for (int i = 0; i < WPL; ++i)
            cur[i] = 0;
        for (int b = 0; b < hb; ++b)
            if ((p >> b) & 1ull)
                xor_row<WPL>(cur, my + (size_t)(chunk + b) * SW);
        uint64_t mask = (uint64_t)p << chunk;
        uint32_t w = group_sum<G>(popc_row<WPL>(cur));
        top.offer(valid && mask != 0, w, mask, kk, thr);
        for (uint32_t s = 1; s < states; ++s) {
            const int b = __ffs(s) - 1;
            w = group_sum<G>(xor_row_popc_hs<WPL, NHB>(cur, my + (size_t)b * SW));
            mask ^= 1ull << b;
            top.offer(valid, w, mask, kk, thr);
        }
        p += stride_groups;
    }

    // merge the CTA's warps: warps 1.. offer their lists to warp 0 via smem
    __syncthreads();
    bmm_candidate* stage = reinterpret_cast<bmm_candidate*>(srow);
    const int warp = threadIdx.x >> 5;
    top.store(stage + warp * 32 * E, 32 * E);
    __syncthreads();
    if (warp == 0) {
        for (int ow = 1; ow < kThreads / 32; ++ow) {
            for (int base = 0; base < 32 * E; base += 32) {
                const bmm_candidate c = stage[ow * 32 * E + base + lane];
                const bool ok = c.weight != 0xffffffffu;
                if (!__any_sync(kFull, ok && c.weight <= thr))
                    break;  // lists are sorted: nothing further can enter
                top.offer(ok, c.weight, c.mask, kk, thr);
            }
        }
        top.store(cta_out + (size_t)blockIdx.x * kk, kk);
    }
}

// ---------------------------------------------------------------------------
// Per-target top-1.  CTA b serves target b / ctas_per_target.
// key = (weight << 40) | tie, tie = S (TB 0) or inverse-Gray(S) (TB 1).
// Within a lane's walk the prefix part of the tie is fixed, so the running
// best is one 32-bit key (weight << chunk) | low tie bits, built by an IMAD
// (weight * wmul + tie, wmul = one << chunk) and kept by one integer min;
// the host keeps chunk + bits(max weight) <= 32.  `one` is 1 at run time.
// Carry-save blocks per step of the per-target kernel.  With its popcount
// sums on the FMA pipe, 4 of the 8 blocks of a 64-word lane balance the ALU
// (XOR + carry-save LOP3) and XU (POPC) pipes best: 40 x 4096, k = 24 on
// B200 takes 13.5 ms with 4 blocks, 14.0 ms with 5, 14.7 ms with 3.
constexpr int targets_nhb(int wpl) { return wpl >= 64 ? 4 : default_nhb(wpl); }

// CTAs per SM the register budget is set for.  64-word lanes: no minimum;
// the compiler's 234-register schedule (2 CTAs per SM) ran 8 % faster than a
// 3-CTA budget (168 registers) and 28 % faster than an unrolled pair of steps.
// 32-word lane pairs fit 6 CTAs in 80 registers without spills.
constexpr int targets_min_ctas(int wpl) { return wpl == 32 ? 6 : 1; }

template <int WPL, int G, int NHB, int TB>
__global__ void __launch_bounds__(kThreads, targets_min_ctas(WPL))
    gray_targets_kernel(const uint64_t* __restrict__ words, int stride, int W,
                        const uint32_t* __restrict__ targets, const uint32_t* __restrict__ others,
                        int k, int chunk, int ctas_per_target, uint32_t one,
                        unsigned long long* __restrict__ best_keys) {
    extern __shared__ __align__(16) uint64_t srow[];
    constexpr int SW = row_stride(WPL, G);
    const int ti = blockIdx.x / ctas_per_target;
    const int part = blockIdx.x % ctas_per_target;
    const uint32_t* oth = others + (size_t)ti * k;
    const uint32_t tgt = targets[ti];
    // rows 0..k-1: others, row k: the target
    stage_rows<WPL, G>(srow, k + 1, W, [&](int r) {
        return words + (size_t)(r < k ? oth[r] : tgt) * stride;
    });
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const int gl = lane % G;
    const int hb = k - chunk;
    const unsigned long long n_prefix = 1ull << hb;
    const unsigned long long p = (unsigned long long)part * (kThreads / G) + threadIdx.x / G;
    const bool valid = p < n_prefix && gl == 0;
    const uint64_t* my = srow + gl * lane_stride(WPL, G);

    uint64_t cur[WPL];
    {
        const ulonglong2* tp = reinterpret_cast<const ulonglong2*>(my + (size_t)k * SW);
#pragma unroll
        for (int i = 0; i < WPL / 2; ++i) {
            const ulonglong2 v = tp[i];
            cur[2 * i] = v.x;
            cur[2 * i + 1] = v.y;
        }
    }
    for (int b = 0; b < hb; ++b)
        if ((p >> b) & 1ull)
            xor_row<WPL>(cur, my + (size_t)(chunk + b) * SW);

    const uint32_t lowmask = (uint32_t)((1ull << chunk) - 1);
    // tie key in the Gray order: inverse-Gray(S) = (ig(p) << chunk) | (s ^ flip)
    const uint32_t flip = (TB && (__popcll(p) & 1)) ? lowmask : 0u;
    const uint32_t wmul = one << chunk;
    const uint32_t states = 1u << chunk;

    uint32_t low = 0;  // low chunk bits of S (the Gray code of s)
    uint32_t best = mad_u32(group_sum<G>(popc_row<WPL>(cur)), wmul, TB ? flip : 0u);
    for (uint32_t s = 1; s < states; ++s) {
        const int b = __ffs(s) - 1;
        const uint32_t w =
            group_sum<G>(xor_row_popc_hs_fma<WPL, NHB>(cur, my + (size_t)b * SW, one));
        low ^= 1u << b;
        best = min(best, mad_u32(w, wmul, TB ? (s ^ flip) : low));
    }
    const uint64_t hi_tie = TB ? (inverse_gray64(p) << chunk) : (p << chunk);
    const uint64_t best_w = chunk < 32 ? (best >> chunk) : 0;
    unsigned long long key =
        valid ? ((best_w << 40) | hi_tie | (uint64_t)(best & lowmask)) : ~0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(kFull, key, o);
        key = other < key ? other : key;
    }
    if (lane == 0 && key != ~0ull)
        atomicMin(best_keys + ti, key);
}

// Decode keys into (mask, weight).
__global__ void decode_keys_kernel(const unsigned long long* __restrict__ keys, int n, int tiebreak,
                                   uint64_t* __restrict__ best_mask,
                                   uint32_t* __restrict__ best_weight) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const unsigned long long key = keys[i];
    const uint64_t tie = key & ((1ull << 40) - 1);
    // S = gray(tie) when the tie key is the Gray index
    best_mask[i] = tiebreak ? (tie ^ (tie >> 1)) : tie;
    best_weight[i] = (uint32_t)(key >> 40);
}

// ---------------------------------------------------------------------------
// host side

// Carry-save blocks (of 8 words) per Gray step of the window kernel, by lane
// width (default_nhb): without them the XU pipe (POPC) saturates while ALU
// idles at ~36 %; 5 of the 8 blocks of a 64-word lane balanced the pipes when
// the popcount sums were ALU adds (the per-target kernel, whose sums are
// IMADs, uses 4: targets_nhb).

int group_shape(size_t W, int* wpl, int* g) {
    if (W <= 2) {
        *wpl = 2, *g = 1;
    } else if (W <= 4) {
        *wpl = 4, *g = 1;
    } else if (W <= 8) {
        *wpl = 8, *g = 1;
    } else if (W <= 16) {
        *wpl = 16, *g = 1;
    } else if (W <= 32) {
        *wpl = 32, *g = 1;
    } else if (W <= 64) {
        *wpl = 64, *g = 1;
    } else {
        int G = 2;
        while ((size_t)G * 64 < W)
            G *= 2;
        if (G > 32)
            return fail(BMM_EINVAL, "gray search: rows wider than 2048 words are not supported");
        *wpl = 64, *g = G;
    }
    return BMM_OK;
}

// The per-target kernel may split a 33-64-word row over a lane pair (32 words
// each): half the registers per lane, so more warps fit per SM, for one
// shuffle-add per step.
int targets_shape(size_t W, int lanes, int* wpl, int* g) {
    BMM_TRY(group_shape(W, wpl, g));
    if (*wpl == 64 && *g == 1 && W > 32 && lanes == 2)
        *wpl = 32, *g = 2;
    return BMM_OK;
}

template <typename F>
int dispatch_wg(int wpl, int g, F&& f) {
#define BMM_WG(A, B)                                                                              \
    if (wpl == A && g == B)                                                                       \
        return f(std::integral_constant<int, A>{}, std::integral_constant<int, B>{});
    BMM_WG(2, 1)
    BMM_WG(4, 1)
    BMM_WG(8, 1)
    BMM_WG(16, 1)
    BMM_WG(32, 1)
    BMM_WG(32, 2)
    BMM_WG(64, 1)
    BMM_WG(64, 2)
    BMM_WG(64, 4)
    BMM_WG(64, 8)
    BMM_WG(64, 16)
    BMM_WG(64, 32)
#undef BMM_WG
    return fail(BMM_EINVAL, "gray search: unsupported row shape");
}

template <typename F>
int dispatch_e(int kk, F&& f) {
    if (kk <= 32)
        return f(std::integral_constant<int, 1>{});
    if (kk <= 128)
        return f(std::integral_constant<int, 4>{});
    if (kk <= 1024)
        return f(std::integral_constant<int, 32>{});
    return fail(BMM_EINVAL, "gray search: k must be <= 1024");
}

}  // namespace

GrayTuning g_gray_tuning;

namespace {
struct GrayShapeEntry {
    size_t W;
    int k;
    GrayTuning t;
};
std::mutex g_shape_mu;
std::vector<GrayShapeEntry> g_shapes;
}  // namespace

int gray_tune_shape(size_t W, int k, const GrayTuning& t) {
    std::lock_guard<std::mutex> lock(g_shape_mu);
    for (auto& e : g_shapes)
        if (e.W == W && e.k == k) {
            e.t = t;
            return BMM_OK;
        }
    if (g_shapes.size() >= 4096)
        return fail(BMM_EINVAL, "gray tuning: at most 4096 shapes");
    g_shapes.push_back({W, k, t});
    return BMM_OK;
}

void gray_tune_reset() {
    std::lock_guard<std::mutex> lock(g_shape_mu);
    g_shapes.clear();
    g_gray_tuning = GrayTuning{};
}

GrayTuning gray_tuning_for(size_t W, int k) {
    GrayTuning t;
    {
        std::lock_guard<std::mutex> lock(g_shape_mu);
        for (const auto& e : g_shapes)
            if (e.W == W && e.k == k)
                t = e.t;
    }
    if (g_gray_tuning.hs_blocks != -1)
        t.hs_blocks = g_gray_tuning.hs_blocks;
    if (g_gray_tuning.chunk_bits != -1)
        t.chunk_bits = g_gray_tuning.chunk_bits;
    if (g_gray_tuning.lanes != -1)
        t.lanes = g_gray_tuning.lanes;
    return t;
}

int auto_chunk_bits(int t, int lanes_per_prefix, int sm_count, int n_items) {
    // Enough independent prefixes for ~32 waves of 128-thread CTAs at 3 CTAs
    // per SM (so the last wave's tail is small), but keep at least 2^8 Gray
    // steps per prefix so the prefix set-up (up to t - chunk row XORs) stays
    // cheap.  Measured on 40 x 4096, k = 24: chunk 10 beats 12 by 9 %.
    const double want =
        (double)sm_count * 3 * 32 * kThreads / lanes_per_prefix / (n_items ? n_items : 1);
    int hb = 0;
    while (hb < t && (double)(1ull << hb) < want)
        ++hb;
    int chunk = t - hb;
    if (chunk < 8)
        chunk = t < 8 ? t : 8;
    if (chunk > 20)
        chunk = 20;
    if (chunk > t)
        chunk = t;
    return chunk;
}

int targets_chunk_bits(int k, int lanes_per_prefix, int sm_count, int n_targets) {
    // Waves of 128-thread CTAs the launch fills at 2 CTAs per SM (the
    // kernel's 234-register schedule) when each prefix walks 2^chunk states.
    auto waves = [&](int chunk) {
        return std::ldexp((double)(n_targets > 0 ? n_targets : 1) * lanes_per_prefix, k - chunk) /
               ((double)sm_count * 2 * kThreads);
    };
    // Long walks keep the prefix set-up (up to k - chunk row XORs) near 1 %;
    // many waves keep the last wave's tail small.  Large jobs: the longest
    // walk (>= 2^10) that still fills 16 waves; small jobs: the longest walk
    // (>= 2^8) that fills 4 waves, else 2^8.  Measured optima on B200: 40 x
    // 4096, k = 24 -> 10 (13.49 ms); 40 x 2048, k = 20 -> 8 (0.52 ms vs 0.84
    // at 10); 64 x 256, k = 16 -> 8 (0.035 ms vs 0.112 at 10).
    const int top = k < 20 ? k : 20;
    for (int c = top; c >= 10; --c)
        if (waves(c) >= 16)
            return c;
    for (int c = top; c >= 8; --c)
        if (waves(c) >= 4)
            return c;
    return k < 8 ? k : 8;
}

int gray_window_launch(Workspace* ws, const uint64_t* d_rows, int t, int W, int chunk, int kk,
                       bmm_candidate* d_out, cudaStream_t stream) {
    int wpl = 0, g = 0;
    BMM_TRY(group_shape((size_t)W, &wpl, &g));
    const size_t srow_bytes = (size_t)t * row_stride(wpl, g) * 8;
    const unsigned long long n_prefix = 1ull << (t - chunk);
    return dispatch_wg(wpl, g, [&](auto WPLc, auto Gc) -> int {
        constexpr int WPL = decltype(WPLc)::value, G = decltype(Gc)::value;
        return dispatch_e(kk, [&](auto Ec) -> int {
            constexpr int E = decltype(Ec)::value;
            auto kern = gray_window_kernel<WPL, G, E, default_nhb(WPL)>;
            const size_t merge_bytes = (size_t)(kThreads / 32) * 32 * E * sizeof(bmm_candidate);
            const size_t smem = srow_bytes > merge_bytes ? srow_bytes : merge_bytes;
            if (smem > (size_t)ws->smem_optin)
                return fail(BMM_EINVAL, "gray search: %zu bytes of rows exceed shared memory",
                            srow_bytes);
            BMM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)smem));
            int occ = 0;
            BMM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kThreads, smem));
            if (occ < 1)
                occ = 1;
            unsigned long long need = (n_prefix * G + kThreads - 1) / kThreads;
            unsigned long long grid = (unsigned long long)ws->sm_count * occ;
            if (need < grid)
                grid = need;
            if (grid < 1)
                grid = 1;
            bmm_candidate* lists = nullptr;
            BMM_TRY(ws_buffer(ws, kSlotCand, grid * kk * sizeof(bmm_candidate), (void**)&lists));
            kern<<<(unsigned)grid, kThreads, smem, stream>>>(d_rows, t, W, chunk, n_prefix, kk,
                                                            lists);
            BMM_CUDA_TRY(cudaGetLastError());
            return merge_topk_lists(lists, (int)grid, kk, d_out, stream);
        });
    });
}

int gray_targets_launch(Workspace* ws, const uint64_t* d_words, int stride, int W,
                        const uint32_t* d_targets, const uint32_t* d_others, int n_targets, int k,
                        int tiebreak, int chunk, unsigned long long* d_keys, uint64_t* d_best_mask,
                        uint32_t* d_best_weight, cudaStream_t stream) {
    int wpl = 0, g = 0;
    const GrayTuning tune = gray_tuning_for((size_t)W, k);
    BMM_TRY(targets_shape((size_t)W, tune.lanes, &wpl, &g));
    const size_t smem = (size_t)(k + 1) * row_stride(wpl, g) * 8;
    if (smem > (size_t)ws->smem_optin)
        return fail(BMM_EINVAL, "gray targets: %zu bytes of rows exceed shared memory", smem);
    // the kernel's running key is (weight << chunk) | low tie in 32 bits:
    // chunk + bits(largest weight of a wpl * g-word row) <= 32 (speed only)
    {
        int wbits = 0;
        while ((1ull << wbits) <= (unsigned long long)wpl * g * 64)
            ++wbits;
        if (chunk > 32 - wbits)
            chunk = 32 - wbits;
    }
    const unsigned long long n_prefix = 1ull << (k - chunk);
    const unsigned long long per_cta = kThreads / g;
    const unsigned long long ctas = (n_prefix + per_cta - 1) / per_cta;
    if (ctas * (unsigned long long)n_targets > 0x7fffffffull)
        return fail(BMM_EINVAL, "gray targets: grid too large (raise chunk_bits)");
    BMM_CUDA_TRY(cudaMemsetAsync(d_keys, 0xff, sizeof(unsigned long long) * n_targets, stream));
    const uint32_t one = 1;
    BMM_TRY(dispatch_wg(wpl, g, [&](auto WPLc, auto Gc) -> int {
        constexpr int WPL = decltype(WPLc)::value, G = decltype(Gc)::value;
        auto go = [&](auto kern) -> int {
            BMM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)smem));
            kern<<<(unsigned)(ctas * n_targets), kThreads, smem, stream>>>(
                d_words, stride, W, d_targets, d_others, k, chunk, (int)ctas, one, d_keys);
            BMM_CUDA_TRY(cudaGetLastError());
            return BMM_OK;
        };
        auto by_tb = [&](auto NHBc) -> int {
            constexpr int NHB = decltype(NHBc)::value;
            return tiebreak ? go(gray_targets_kernel<WPL, G, NHB, 1>)
                            : go(gray_targets_kernel<WPL, G, NHB, 0>);
        };
        const int hs = tune.hs_blocks;
        if constexpr (WPL == 64 && G == 1) {
            switch (hs) {
            case -1: break;
            case 0: return by_tb(std::integral_constant<int, 0>{});
            case 2: return by_tb(std::integral_constant<int, 2>{});
            case 3: return by_tb(std::integral_constant<int, 3>{});
            case 4: return by_tb(std::integral_constant<int, 4>{});
            case 5: return by_tb(std::integral_constant<int, 5>{});
            case 6: return by_tb(std::integral_constant<int, 6>{});
            case 8: return by_tb(std::integral_constant<int, 8>{});
            default: return fail(BMM_EINVAL, "gray tuning: hs_blocks must be 0, 2-6 or 8");
            }
        }
        if constexpr (WPL == 32) {
            switch (hs) {
            case -1: break;
            case 0: return by_tb(std::integral_constant<int, 0>{});
            case 2: return by_tb(std::integral_constant<int, 2>{});
            case 3: return by_tb(std::integral_constant<int, 3>{});
            case 4: return by_tb(std::integral_constant<int, 4>{});
            default: return fail(BMM_EINVAL, "gray tuning: hs_blocks must be 0, 2-4 for 32-word lanes");
            }
        }
        (void)hs;
        return by_tb(std::integral_constant<int, targets_nhb(WPL)>{});
    }));
    decode_keys_kernel<<<(n_targets + 127) / 128, 128, 0, stream>>>(d_keys, n_targets, tiebreak,
                                                                    d_best_mask, d_best_weight);
    BMM_CUDA_TRY(cudaGetLastError());
    return BMM_OK;
}

}  // namespace bmm

// ---------------------------------------------------------------------------
// Throughput probe for the roofline denominator of the Gray-code kernels:
// the same per-word work as a Gray step (64-bit XOR + 64-bit POPC + add)
// with everything in registers (no shared-memory loads, no top-k), so its
// rate is the device's ceiling for that instruction mix.
namespace bmm {
namespace {
__global__ void __launch_bounds__(256) popc_probe_kernel(int iters, unsigned long long* sink) {
    uint64_t x[64];
#pragma unroll
    for (int i = 0; i < 64; ++i)
        x[i] = (uint64_t)(threadIdx.x + 1) * 0x9E3779B97F4A7C15ull + (uint64_t)i * 0x632BE59BD9B4E019ull;
    uint32_t acc = 0;
    uint64_t c = blockIdx.x;
    for (int it = 0; it < iters; ++it) {
        c = c * 6364136223846793005ull + 1442695040888963407ull;
#pragma unroll
        for (int i = 0; i < 64; ++i) {
            x[i] ^= c;
            acc += __popcll(x[i]);
        }
    }
    if (acc == 0x7fffffffu)  // never true in practice; keeps the work alive
        sink[blockIdx.x] = acc;
}
}  // namespace

int popc_probe(double* words_per_second) {
    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws)
        return st;
    void* sink = nullptr;
    BMM_TRY(ws_buffer(ws, kSlotExtra1, 8 * 4096, &sink));
    const int blocks = ws->sm_count * 4, iters = 4096;
    cudaEvent_t a, b;
    BMM_CUDA_TRY(cudaEventCreate(&a));
    BMM_CUDA_TRY(cudaEventCreate(&b));
    popc_probe_kernel<<<blocks, 256, 0, ws->stream>>>(64, (unsigned long long*)sink);  // warm
    BMM_CUDA_TRY(cudaEventRecord(a, ws->stream));
    popc_probe_kernel<<<blocks, 256, 0, ws->stream>>>(iters, (unsigned long long*)sink);
    BMM_CUDA_TRY(cudaEventRecord(b, ws->stream));
    BMM_CUDA_TRY(cudaEventSynchronize(b));
    float ms = 0;
    BMM_CUDA_TRY(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *words_per_second = (double)blocks * 256 * iters * 64 / (ms * 1e-3);
    return BMM_OK;
}
}  // namespace bmm

// ---------------------------------------------------------------------------
// Allocation-free variant of the per-target Gray-code search.
//
// Who needs it: callers that are not allowed to allocate device memory --
// code running inside another framework's memory pool or arena (which must
// see every byte it hands out), plug-ins loaded into a host that forbids
// cudaMalloc/cudaFree on its threads, or real-time loops where an allocation
// can stall.  They pass device inputs and outputs they already own; the only
// other device memory this call touches is the fixed per-target key array
// below, which the CUDA runtime reserves when the library's kernels are
// loaded on a device and keeps until the process exits.
namespace bmm {

// Largest n_targets one call accepts: 16384 keys x 8 bytes = 128 KiB per device.
constexpr size_t kNoAllocMaxTargets = 16384;

static __device__ __align__(256) unsigned long long g_noalloc_keys[kNoAllocMaxTargets];

namespace {
struct NoAllocDevice {
    bool ready = false;
    unsigned long long* keys = nullptr;  // device address of g_noalloc_keys
    int sm_count = 0;
    int smem_optin = 0;
};
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];

// Once per device, with that device current: resolve the array's device
// address (a host-side reference to g_noalloc_keys is only a stand-in, never
// a device address) and read the launch limits.  Allocates nothing.
int noalloc_setup(NoAllocDevice** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return fail(BMM_ENODEV, "no CUDA device is available: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kNoAllocMaxDevices)
        return fail(BMM_EINVAL, "gray targets (no-alloc): device %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    NoAllocDevice& d = g_noalloc_dev[dev];
    if (!d.ready) {
        void* addr = nullptr;
        e = cudaGetSymbolAddress(&addr, g_noalloc_keys);
        if (e != cudaSuccess)
            return fail(BMM_ECUDA, "cudaGetSymbolAddress(g_noalloc_keys) failed: %s",
                        cudaGetErrorString(e));
        int sms = 0, optin = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess)
            e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (e != cudaSuccess)
            return fail(BMM_ECUDA, "device query failed: %s", cudaGetErrorString(e));
        d.keys = static_cast<unsigned long long*>(addr);
        d.sm_count = sms;
        d.smem_optin = optin;
        d.ready = true;
    }
    *out = &d;
    return BMM_OK;
}
}  // namespace
}  // namespace bmm

extern "C" BMM_API int bmm_gray_targets_noalloc(const uint64_t* d_words, size_t rows, size_t stride,
                                                size_t cols, const uint32_t* d_targets,
                                                const uint32_t* d_others, size_t n_targets,
                                                size_t k, int tiebreak, uint64_t* d_best_mask,
                                                uint32_t* d_best_weight, void* stream) {
    using namespace bmm;
    clear_error();
    (void)rows;
    if (n_targets == 0)
        return BMM_OK;
    if (n_targets > kNoAllocMaxTargets)
        return fail(BMM_EINVAL,
                    "gray targets (no-alloc): %zu targets exceed the fixed scratch of %zu; split "
                    "the call or use bmm_gray_targets_dev",
                    n_targets, kNoAllocMaxTargets);
    if (k < 1 || k > 40)
        return fail(BMM_EINVAL, "gray targets (no-alloc): k must be in [1, 40]");
    if (cols >= (1ull << 24))
        return fail(BMM_EINVAL, "gray targets (no-alloc): cols must be < 2^24");
    if ((cols + 63) / 64 > stride)
        return fail(BMM_EINVAL, "gray targets (no-alloc): stride smaller than the row width");
    if (!d_words || !d_targets || !d_others || !d_best_mask || !d_best_weight)
        return fail(BMM_EINVAL, "gray targets (no-alloc): null argument");
    NoAllocDevice* d = nullptr;
    BMM_TRY(noalloc_setup(&d));
    // Launch limits only; this Workspace owns no buffers and no stream.
    Workspace limits;
    limits.sm_count = d->sm_count;
    limits.smem_optin = d->smem_optin;
    const size_t W = (cols + 63) / 64;
    int lanes = 1;
    while ((size_t)lanes * 64 < W)
        lanes *= 2;
    int chunk = targets_chunk_bits((int)k, lanes, d->sm_count, (int)n_targets);
    const GrayTuning tune = gray_tuning_for(W, (int)k);  // as bmm_gray_targets_dev
    if (tune.chunk_bits > 0)
        chunk = tune.chunk_bits;
    if (chunk > (int)k)
        chunk = (int)k;
    // gray_targets_launch clears the keys it uses to ~0 before the search, so
    // whatever the previous call left in the array does not leak into this one.
    return gray_targets_launch(&limits, d_words, (int)stride, (int)W, d_targets, d_others,
                               (int)n_targets, (int)k, tiebreak, chunk, d->keys, d_best_mask,
                               d_best_weight, (cudaStream_t)stream);
}
