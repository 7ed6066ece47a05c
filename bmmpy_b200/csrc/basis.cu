// Exact minimum-weight basis of a window (ExactBasisSolver::solve,
// src/solver/exact_basis_solver.cpp:58-157).
//
// The reference walks all 2^t - 1 nonzero row combinations of a window
// (t <= 32) in reflected-Gray order (index 1..2^t-1, mask = index ^ index>>1),
// buckets them by weight (a counting sort, enumeration order inside a bucket)
// and inserts them weight by weight into a GF(2) basis until the window's
// rank r is reached.  The accepted set of such a greedy insertion depends
// only on the order in which candidates are offered, so this version keeps
// the order and changes everything else:
//
//  * enumeration on the device, in the reference's own Gray walk: state k
//    (1 <= k < 2^t) is mask k ^ (k >> 1), reached from k - 1 by toggling row
//    ctz(k).  One wave of CTAs (one per resident slot) cuts the walk into
//    equal contiguous slices, one per group of G lanes; each lane holds WPL
//    words of the running XOR in registers, the window rows sit in shared
//    memory.  Pass 0 builds the weight histogram (per-CTA shared bins), pass
//    1 collects the states whose weight lies in [lo, hi] as keys
//    (weight << 32) | k, which sorted ascending are the reference's bucket
//    order.  Windows wider than 64 words per lane x 32 lanes accumulate
//    per-mask weights slab by slab instead.
//  * the greedy on r-bit coordinates.  Projecting the row space onto the
//    pivot columns of an echelon form of the window is an isomorphism, so a
//    combination's coordinate is the XOR of its rows' coordinates (four byte
//    tables) and independence is tested in a 32-slot XOR basis.
//  * only as many candidates as the greedy consumes: the weight cut starts
//    where the histogram holds 4r nonzero candidates and grows 4x per pass.
#include "common.cuh"
#include "popc.cuh"

#include <algorithm>
#include <type_traits>
#include <vector>

namespace bmm {
namespace basis {

constexpr int kThreads = 128;
constexpr int kHistSmem = 16384;  // weight bins held in shared memory (64 KB)
constexpr int kMaxWpl = 64;       // words per lane in registers
constexpr int kMaxGroup = 32;     // lanes per prefix (one warp)

enum Mode : int { kHist = 0, kCollect = 1, kAccumulate = 2 };

// Histogram increments as fire-and-forget reductions.  The asm carries no
// memory clobber on purpose: the bins never alias the window rows in shared
// memory, and without a clobber the compiler may issue the next step's row
// loads ahead of this update instead of serialising every step behind it.
__device__ __forceinline__ void red_shared_add(unsigned* p, unsigned v) {
    asm volatile("red.shared.add.u32 [%0], %1;" ::"r"((unsigned)__cvta_generic_to_shared(p)),
                 "r"(v));
}

struct Launch {
    const uint64_t* rows;  // t rows of W words, `pitch` words apart (a column slab)
    size_t pitch;
    int t, W, cols, mode;
    uint32_t L;                     // states per lane group (a multiple of 32)
    uint32_t lo, hi;                // kCollect: weight range
    unsigned long long* counts;     // kHist: cols + 1 bins
    unsigned long long* keys;       // kCollect
    unsigned long long* nkeys;      // kCollect
    unsigned long long cap;         // kCollect
    uint32_t* weights;              // kAccumulate: indexed by mask
    int first;                      // kAccumulate: first slab stores, later slabs add
};

// Shared layout of the window rows: lane gl of a group owns words
// [gl * WPL, (gl + 1) * WPL) of every row, stored in VEC-word chunks
// interleaved across the group -- chunk q of lane gl of row b at
// ((b * Q + q) * G + gl) -- so the G lanes of a group read adjacent chunks
// (the groups of a warp read the same row at the same step, a broadcast,
// except where their slices' counters differ in a bit >= 5).
template <int WPL, int G, int NHB>
__global__ void __launch_bounds__(kThreads) enum_kernel(const Launch a) {
    constexpr int VEC = WPL >= 2 ? 2 : 1;  // words per shared load
    constexpr int Q = WPL / VEC;
    using Vec = typename std::conditional<VEC == 2, ulonglong2, unsigned long long>::type;
    extern __shared__ __align__(16) unsigned char smem[];
    Vec* srow = reinterpret_cast<Vec*>(smem);  // t x Q x G chunks
    const int SW = G * WPL;
    unsigned* hist = reinterpret_cast<unsigned*>(smem + (size_t)a.t * SW * 8);
    const bool shared_hist = a.mode == kHist && a.cols + 1 <= kHistSmem;
    uint64_t* sw = reinterpret_cast<uint64_t*>(smem);
    for (int i = threadIdx.x; i < a.t * SW; i += blockDim.x) {
        const int r = i / SW, w = i % SW;  // word w of row r
        const int gl = w / WPL, k = w % WPL, q = k / VEC, v = k % VEC;
        sw[(((size_t)r * Q + q) * G + gl) * VEC + v] =
            w < a.W ? a.rows[(size_t)r * a.pitch + w] : 0ull;
    }
    if (shared_hist)
        for (int i = threadIdx.x; i <= a.cols; i += blockDim.x)
            hist[i] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int gl = lane % G;  // lane within the group
    uint64_t cur[WPL];
#pragma unroll
    for (int i = 0; i < WPL; ++i)
        cur[i] = 0;
    auto toggle = [&](int b) {
        const Vec* src = srow + (size_t)b * Q * G + gl;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const Vec x = src[q * G];
            if constexpr (VEC == 2) {
                cur[2 * q] ^= x.x;
                cur[2 * q + 1] ^= x.y;
            } else {
                cur[q] ^= x;
            }
        }
    };
    // this group's slice [k0, k0 + n) of the Gray walk k -> mask k ^ (k >> 1);
    // only the last groups have n < L (n = 0 past the end)
    const unsigned long long total = 1ull << a.t;
    const unsigned long long k0 =
        ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) / G * a.L;
    const uint32_t n = k0 < total ? (uint32_t)min((unsigned long long)a.L, total - k0) : 0u;
    const unsigned gmask = G == 32 ? kFull : ((1u << G) - 1) << (lane & ~(G - 1));
    auto emit = [&](unsigned long long k, uint32_t w) {
        if (gl != 0 || k == 0)
            return;
        if (a.mode == kHist) {
            if (shared_hist)
                red_shared_add(hist + w, 1u);
            else
                atomicAdd(a.counts + w, 1ull);
        } else if (a.mode == kCollect) {
            if (w >= a.lo && w <= a.hi) {
                const unsigned long long pos = atomicAdd(a.nkeys, 1ull);
                if (pos < a.cap)
                    a.keys[pos] = ((unsigned long long)w << 32) | (uint32_t)k;
            }
        } else {
            const uint32_t mask = (uint32_t)(k ^ (k >> 1));
            if (a.first)
                a.weights[mask] = w;
            else
                a.weights[mask] += w;
        }
    };
    if (n) {
        uint32_t g0 = (uint32_t)(k0 ^ (k0 >> 1));
        while (g0) {
            toggle(__ffs(g0) - 1);
            g0 &= g0 - 1;
        }
        uint32_t w = 0;
#pragma unroll
        for (int i = 0; i < WPL; ++i)
            w += __popcll(cur[i]);
        for (int o = G >> 1; o > 0; o >>= 1)
            w += __shfl_xor_sync(gmask, w, o);
        emit(k0, w);
    }
    for (uint32_t j = 1; j < n; ++j) {
        // k0 and L are multiples of 32: the toggled row is ctz(j) unless j is
        // a multiple of 32 too, so it is warp-uniform 31 steps in 32
        const unsigned long long k = k0 + j;
        const int b = (j & 31) ? __ffs(j) - 1 : __ffsll((long long)k) - 1;
        uint32_t w;
        if constexpr (VEC == 2) {
            w = xor_row_popc_hs<WPL, NHB>(cur, sw + ((size_t)b * Q * G + gl) * 2, G);
        } else {
            toggle(b);
            w = __popcll(cur[0]);
        }
        for (int o = G >> 1; o > 0; o >>= 1)
            w += __shfl_xor_sync(gmask, w, o);
        emit(k, w);
    }
    if (shared_hist) {
        __syncthreads();
        for (int i = threadIdx.x; i <= a.cols; i += blockDim.x)
            if (hist[i])
                atomicAdd(a.counts + i, (unsigned long long)hist[i]);
    }
}

// Histogram / collection over per-mask weights (wide windows).
__global__ void weights_hist_kernel(const uint32_t* __restrict__ weights, unsigned long long n,
                                    unsigned long long* __restrict__ counts) {
    for (unsigned long long m = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x + 1;
         m <= n; m += (unsigned long long)gridDim.x * blockDim.x)
        atomicAdd(counts + weights[m], 1ull);
}

__global__ void weights_collect_kernel(const uint32_t* __restrict__ weights,
                                       unsigned long long n, uint32_t lo, uint32_t hi,
                                       unsigned long long* __restrict__ keys,
                                       unsigned long long* __restrict__ nkeys,
                                       unsigned long long cap) {
    const int lane = threadIdx.x & 31;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long base_m = blockIdx.x * (unsigned long long)blockDim.x; base_m <= n;
         base_m += stride) {
        const unsigned long long m = base_m + threadIdx.x;
        const uint32_t w = (m >= 1 && m <= n) ? weights[m] : 0u;
        const bool hit = m >= 1 && m <= n && w >= lo && w <= hi;
        const unsigned bal = __ballot_sync(kFull, hit);
        if (!bal)
            continue;
        unsigned long long base = 0;
        if (lane == __ffs(bal) - 1)
            base = atomicAdd(nkeys, (unsigned long long)__popc(bal));
        base = __shfl_sync(kFull, base, __ffs(bal) - 1);
        if (hit) {
            const unsigned long long pos = base + __popc(bal & ((1u << lane) - 1));
            if (pos < cap)
                keys[pos] = ((unsigned long long)w << 32) | (uint32_t)inverse_gray64(m);
        }
    }
}

struct Plan {
    int G, wpl;
    size_t smem;
};

// W: words per row handled by one launch (the whole row, or one slab).
Plan plan_for(int t, int W, int cols) {
    Plan p{};
    p.G = 1;
    while ((W + p.G - 1) / p.G > kMaxWpl)
        p.G <<= 1;
    const int need = (W + p.G - 1) / p.G;
    p.wpl = 1;
    while (p.wpl < need)
        p.wpl <<= 1;
    // G * WPL is the power of two at or above W, and W <= slab_words(t)
    p.smem = (size_t)t * p.G * p.wpl * 8 + (size_t)(cols + 1 <= kHistSmem ? (cols + 1) * 4 : 0);
    return p;
}

// One CTA per resident slot (a single wave); the 2^t states are cut into
// equal contiguous slices of the Gray walk, one per lane group, each a
// multiple of 32 states long.
template <typename K>
int launch_kernel(K kernel, const Plan& pl, Launch a, int sm_count, cudaStream_t s) {
    BMM_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)pl.smem));
    int per_sm = 0;
    BMM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads,
                                                               pl.smem));
    if (per_sm < 1)
        return fail(BMM_EINVAL, "exact basis: kernel does not fit on an SM");
    const unsigned long long total = 1ull << a.t;
    const unsigned long long groups = (unsigned long long)per_sm * sm_count * kThreads / pl.G;
    unsigned long long L = (total + groups - 1) / groups;
    L = std::max<unsigned long long>(32, (L + 31) / 32 * 32);
    const unsigned long long used = (total + L - 1) / L;  // groups with work
    const unsigned blocks = (unsigned)((used * pl.G + kThreads - 1) / kThreads);
    a.L = (uint32_t)L;
    kernel<<<blocks, kThreads, pl.smem, s>>>(a);
    BMM_CUDA_TRY(cudaGetLastError());
    return BMM_OK;
}

int g_basis_nhb = -1;  // carry-save blocks per 64-word lane; -1 = default_nhb

template <int WPL, int G>
int launch_g(const Plan& pl, const Launch& a, int sm_count, cudaStream_t s) {
    if constexpr (WPL == 64) {
        switch (g_basis_nhb) {
        case 0: return launch_kernel(enum_kernel<64, G, 0>, pl, a, sm_count, s);
        case 2: return launch_kernel(enum_kernel<64, G, 2>, pl, a, sm_count, s);
        case 8: return launch_kernel(enum_kernel<64, G, 8>, pl, a, sm_count, s);
        default: break;
        }
    }
    // rows of 8+ lanes per group favour the full carry-save tree (measured)
    constexpr int nhb = (WPL == 64 && G >= 8) ? 8 : default_nhb(WPL);
    return launch_kernel(enum_kernel<WPL, G, nhb>, pl, a, sm_count, s);
}

// G > 1 only when one lane's share is above 32 words, i.e. WPL == 64.
int launch(const Plan& pl, Launch a, int sm_count, cudaStream_t s) {
    if (pl.wpl == 64) {
        switch (pl.G) {
        case 1: return launch_g<64, 1>(pl, a, sm_count, s);
        case 2: return launch_g<64, 2>(pl, a, sm_count, s);
        case 4: return launch_g<64, 4>(pl, a, sm_count, s);
        case 8: return launch_g<64, 8>(pl, a, sm_count, s);
        case 16: return launch_g<64, 16>(pl, a, sm_count, s);
        case 32: return launch_g<64, 32>(pl, a, sm_count, s);
        }
    } else if (pl.G == 1) {
        switch (pl.wpl) {
        case 1: return launch_g<1, 1>(pl, a, sm_count, s);
        case 2: return launch_g<2, 1>(pl, a, sm_count, s);
        case 4: return launch_g<4, 1>(pl, a, sm_count, s);
        case 8: return launch_g<8, 1>(pl, a, sm_count, s);
        case 16: return launch_g<16, 1>(pl, a, sm_count, s);
        case 32: return launch_g<32, 1>(pl, a, sm_count, s);
        }
    }
    return fail(BMM_EINVAL, "exact basis: unsupported row width");
}

// Widest row slab one launch handles: G * WPL words per row for all t rows
// in shared memory (at most 192 KB; cols < 16384 also keeps a 64 KB histogram,
// and those rows are at most 256 words).  Wider windows run one launch per
// slab, adding each slab's popcounts into a per-mask weight array.
size_t slab_words(int t) {
    size_t s = (size_t)kMaxWpl * kMaxGroup;
    while (s > 1 && (size_t)t * s * 8 > 196608)
        s >>= 1;
    return s;
}

// Device-side enumeration of one window: rows compacted on the device,
// per-mask weights for wide windows, histogram and ranged collection.
struct Enumerator {
    Workspace* ws = nullptr;
    cudaStream_t stream = nullptr;
    int t = 0, cols = 0;
    size_t W = 0, slab = 0;
    const uint64_t* d_rows = nullptr;
    uint32_t* d_weights = nullptr;  // wide windows only
    unsigned long long states = 0;

    bool wide() const { return W > slab; }

    // Window rows (t x W words, row-major, tail bits clear) already on the device.
    int init_dev(Workspace* w, const uint64_t* rows_dev, size_t ncols, size_t nt,
                 cudaStream_t st) {
        ws = w;
        stream = st;
        t = (int)nt;
        cols = (int)ncols;
        W = (ncols + 63) / 64;
        slab = slab_words(t);
        states = (1ull << nt) - 1;
        d_rows = rows_dev;
        if (wide()) {
            void* q = nullptr;
            BMM_TRY(ws_buffer(ws, kSlotExtra0, (size_t)(states + 1) * 4, &q));
            d_weights = (uint32_t*)q;
            const Plan pl = plan_for(t, (int)slab, cols);
            for (size_t j = 0; j * slab < W; ++j) {
                Launch a{};
                a.rows = d_rows + j * slab;
                a.pitch = W;
                a.t = t;
                a.W = (int)std::min(slab, W - j * slab);
                a.cols = cols;
                a.mode = kAccumulate;
                a.weights = d_weights;
                a.first = j == 0;
                BMM_TRY(launch(pl, a, ws->sm_count, stream));
            }
        }
        return BMM_OK;
    }

    // Window rows gathered from a host matrix.
    int init(Workspace* w, const uint64_t* words, size_t stride, size_t ncols,
             const uint32_t* win, size_t nt) {
        const size_t nw = (ncols + 63) / 64;
        std::vector<uint64_t> h(nt * std::max<size_t>(nw, 1), 0ull);
        const uint64_t tail = (ncols & 63) ? ((1ull << (ncols & 63)) - 1) : ~0ull;
        for (size_t r = 0; r < nt; ++r)
            for (size_t c = 0; c < nw; ++c)
                h[r * nw + c] = words[(size_t)win[r] * stride + c] & (c == nw - 1 ? tail : ~0ull);
        void* p = nullptr;
        BMM_TRY(ws_buffer(w, kSlotRows, h.size() * 8, &p));
        BMM_CUDA_TRY(cudaMemcpyAsync(p, h.data(), h.size() * 8, cudaMemcpyHostToDevice,
                                     w->stream));
        return init_dev(w, (const uint64_t*)p, ncols, nt, w->stream);
    }

    int hist(unsigned long long* d_counts) {
        BMM_CUDA_TRY(cudaMemsetAsync(d_counts, 0, ((size_t)cols + 1) * 8, stream));
        if (wide()) {
            const unsigned blocks = (unsigned)std::min<unsigned long long>(
                (states + 255) / 256, (unsigned long long)ws->sm_count * 16);
            weights_hist_kernel<<<blocks, 256, 0, stream>>>(d_weights, states, d_counts);
            BMM_CUDA_TRY(cudaGetLastError());
            return BMM_OK;
        }
        Launch a{};
        a.rows = d_rows;
        a.pitch = W;
        a.t = t;
        a.W = (int)W;
        a.cols = cols;
        a.mode = kHist;
        a.counts = d_counts;
        return launch(plan_for(t, (int)W, cols), a, ws->sm_count, stream);
    }

    int collect(uint32_t lo, uint32_t hi, unsigned long long* d_keys, unsigned long long cap,
                unsigned long long* d_n) {
        BMM_CUDA_TRY(cudaMemsetAsync(d_n, 0, 8, stream));
        if (wide()) {
            const unsigned blocks = (unsigned)std::min<unsigned long long>(
                (states + 256) / 256, (unsigned long long)ws->sm_count * 16);
            weights_collect_kernel<<<blocks, 256, 0, stream>>>(d_weights, states, lo, hi, d_keys,
                                                               d_n, cap);
            BMM_CUDA_TRY(cudaGetLastError());
            return BMM_OK;
        }
        Launch a{};
        a.rows = d_rows;
        a.pitch = W;
        a.t = t;
        a.W = (int)W;
        a.cols = cols;
        a.mode = kCollect;
        a.lo = lo;
        a.hi = hi;
        a.keys = d_keys;
        a.nkeys = d_n;
        a.cap = cap;
        return launch(plan_for(t, (int)W, cols), a, ws->sm_count, stream);
    }
};

// Pivot columns of an echelon form of the window rows and each row's
// coordinate (its bits at those columns); returns the rank.
int coordinates(const uint64_t* words, size_t stride, size_t cols, const uint32_t* win, size_t t,
                std::vector<uint32_t>& coord) {
    const size_t W = (cols + 63) / 64;
    const uint64_t tail = (cols & 63) ? ((1ull << (cols & 63)) - 1) : ~0ull;
    std::vector<std::vector<uint64_t>> basis;
    std::vector<size_t> pivots;
    std::vector<uint64_t> v(W);
    for (size_t r = 0; r < t; ++r) {
        for (size_t c = 0; c < W; ++c)
            v[c] = words[(size_t)win[r] * stride + c] & (c == W - 1 ? tail : ~0ull);
        for (size_t k = 0; k < basis.size(); ++k)
            if ((v[pivots[k] >> 6] >> (pivots[k] & 63)) & 1)
                for (size_t c = 0; c < W; ++c)
                    v[c] ^= basis[k][c];
        for (size_t c = 0; c < W; ++c)
            if (v[c]) {
                pivots.push_back(c * 64 + __builtin_ctzll(v[c]));
                basis.push_back(v);
                break;
            }
    }
    coord.assign(t, 0u);
    for (size_t r = 0; r < t; ++r)
        for (size_t k = 0; k < pivots.size(); ++k)
            if ((words[(size_t)win[r] * stride + (pivots[k] >> 6)] >> (pivots[k] & 63)) & 1)
                coord[r] |= 1u << k;
    return (int)pivots.size();
}

}  // namespace basis
}  // namespace bmm

using namespace bmm;

namespace {

int check_window(const uint64_t* words, size_t stride, size_t cols, const uint32_t* win,
                 size_t t) {
    if (!words || !win)
        return fail(BMM_EINVAL, "exact basis: null window");
    if (stride < (cols + 63) / 64)
        return fail(BMM_EINVAL, "exact basis: stride is smaller than the row width");
    if (cols >= (1ull << 31))
        return fail(BMM_EINVAL, "exact basis: too many columns");
    for (size_t i = 0; i < t; ++i)
        for (size_t j = 0; j < i; ++j)
            if (win[i] == win[j])
                return fail(BMM_EINVAL, "exact basis: window rows must be unique");
    return BMM_OK;
}

}  // namespace

extern "C" {

BMM_API int bmm_basis_weight_counts(const uint64_t* words, size_t stride, size_t cols,
                                    const uint32_t* win, size_t t, uint64_t* counts) {
    clear_error();
    if (!counts)
        return fail(BMM_EINVAL, "exact basis: null counts");
    if (t > 32)
        return fail(BMM_EINVAL, "ExactBasisSolver: this implementation supports at most 32 rows");
    if (t)
        BMM_TRY(check_window(words, stride, cols, win, t));
    std::fill(counts, counts + cols + 1, 0ull);
    if (t == 0)
        return BMM_OK;
    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws)
        return st;
    basis::Enumerator en;
    BMM_TRY(en.init(ws, words, stride, cols, win, t));
    void* d_counts = nullptr;
    BMM_TRY(ws_buffer(ws, kSlotAux, (cols + 1) * 8, &d_counts));
    BMM_TRY(en.hist((unsigned long long*)d_counts));
    BMM_CUDA_TRY(cudaMemcpyAsync(counts, d_counts, (cols + 1) * 8, cudaMemcpyDeviceToHost,
                                 ws->stream));
    BMM_CUDA_TRY(cudaStreamSynchronize(ws->stream));
    return BMM_OK;
}

BMM_API int bmm_basis_tune(int hs_blocks) {
    clear_error();
    if (hs_blocks != -1 && hs_blocks != 0 && hs_blocks != 2 && hs_blocks != 5 && hs_blocks != 8)
        return fail(BMM_EINVAL, "basis tuning: hs_blocks must be -1, 0, 2, 5 or 8");
    basis::g_basis_nhb = hs_blocks == 5 ? -1 : hs_blocks;
    return BMM_OK;
}

BMM_API int bmm_basis_weight_counts_dev(const uint64_t* rows, size_t t, size_t cols,
                                        uint64_t* counts, void* stream) {
    clear_error();
    if (!rows || !counts)
        return fail(BMM_EINVAL, "exact basis: null device pointer");
    if (t == 0 || t > 32)
        return fail(BMM_EINVAL, "exact basis: window rows must be in [1, 32]");
    if (cols >= (1ull << 31))
        return fail(BMM_EINVAL, "exact basis: too many columns");
    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws)
        return st;
    basis::Enumerator en;
    BMM_TRY(en.init_dev(ws, rows, cols, t, (cudaStream_t)stream));
    return en.hist((unsigned long long*)counts);
}

BMM_API int bmm_exact_basis(const uint64_t* words, size_t stride, size_t cols,
                            const uint32_t* win, size_t t, const bmm_exact_basis_config* cfg,
                            bmm_exact_basis_result* res, uint32_t* basis_masks,
                            uint32_t* basis_weights) {
    clear_error();
    if (!cfg || !res)
        return fail(BMM_EINVAL, "exact basis: null config or result");
    *res = bmm_exact_basis_result{};
    res->input_rows = t;
    res->cols = cols;
    if (t == 0)
        return BMM_OK;
    // the reference's checks, in its order
    if (t > cfg->max_rows)
        return fail(BMM_EINVAL,
                    "ExactBasisSolver: window has more rows than the configured max_rows cap");
    if (t > 32)
        return fail(BMM_EINVAL, "ExactBasisSolver: this implementation supports at most 32 rows");
    const uint64_t states = (1ull << t) - 1;
    if (states > cfg->max_states)
        return fail(BMM_EINVAL,
                    "ExactBasisSolver: state count exceeds the configured max_states cap");
    if (states * 4ull > cfg->max_storage_bytes)
        return fail(BMM_EINVAL,
                    "ExactBasisSolver: required packed-mask storage exceeds max_storage_bytes");
    BMM_TRY(check_window(words, stride, cols, win, t));
    if (!basis_masks || !basis_weights)
        return fail(BMM_EINVAL, "exact basis: null output arrays");

    std::vector<uint32_t> coord;
    const int rank = basis::coordinates(words, stride, cols, win, t, coord);
    res->rank = (size_t)rank;
    res->enumerated_states = states;
    if (rank == 0)
        return BMM_OK;

    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws)
        return st;
    basis::Enumerator en;
    BMM_TRY(en.init(ws, words, stride, cols, win, t));
    void* d_counts = nullptr;
    BMM_TRY(ws_buffer(ws, kSlotAux, (cols + 1) * 8, &d_counts));
    BMM_TRY(en.hist((unsigned long long*)d_counts));
    std::vector<unsigned long long> counts(cols + 1);
    BMM_CUDA_TRY(cudaMemcpyAsync(counts.data(), d_counts, (cols + 1) * 8,
                                 cudaMemcpyDeviceToHost, ws->stream));
    BMM_CUDA_TRY(cudaStreamSynchronize(ws->stream));

    // coordinate of a mask = XOR of its rows' coordinates, by bytes
    uint32_t table[4][256];
    for (int b = 0; b < 4; ++b)
        for (int v = 0; v < 256; ++v) {
            uint32_t c = 0;
            for (int i = 0; i < 8; ++i)
                if (((v >> i) & 1) && (size_t)(b * 8 + i) < t)
                    c ^= coord[b * 8 + i];
            table[b][v] = c;
        }
    uint32_t slot[32] = {};  // XOR basis by highest set bit
    size_t accepted = 0;
    std::vector<unsigned long long> keys;
    size_t lo = 1;
    unsigned long long want = 4ull * (unsigned long long)rank;
    while (accepted < (size_t)rank && lo <= cols) {
        size_t hi = lo;
        unsigned long long n = counts[lo];
        while (hi < cols && n < want)
            n += counts[++hi];
        if (n) {
            void *d_keys = nullptr, *d_n = nullptr;
            BMM_TRY(ws_buffer(ws, kSlotKeys, (size_t)n * 8, &d_keys));
            BMM_TRY(ws_buffer(ws, kSlotCounter, 8, &d_n));
            BMM_TRY(en.collect((uint32_t)lo, (uint32_t)hi, (unsigned long long*)d_keys, n,
                               (unsigned long long*)d_n));
            unsigned long long got = 0;
            keys.resize((size_t)n);
            BMM_CUDA_TRY(cudaMemcpyAsync(&got, d_n, 8, cudaMemcpyDeviceToHost, ws->stream));
            BMM_CUDA_TRY(cudaMemcpyAsync(keys.data(), d_keys, (size_t)n * 8,
                                         cudaMemcpyDeviceToHost, ws->stream));
            BMM_CUDA_TRY(cudaStreamSynchronize(ws->stream));
            if (got != n)
                return fail(BMM_ECUDA, "exact basis: collected %llu combinations, expected %llu",
                            got, n);
            std::sort(keys.begin(), keys.end());
            for (size_t i = 0; i < keys.size() && accepted < (size_t)rank; ++i) {
                const uint32_t idx = (uint32_t)keys[i];
                const uint32_t mask = idx ^ (idx >> 1);
                uint32_t c = table[0][mask & 255] ^ table[1][(mask >> 8) & 255] ^
                             table[2][(mask >> 16) & 255] ^ table[3][mask >> 24];
                while (c) {
                    const int h = 31 - __builtin_clz(c);
                    if (!slot[h]) {
                        slot[h] = c;
                        const uint32_t w = (uint32_t)(keys[i] >> 32);
                        basis_masks[accepted] = mask;
                        basis_weights[accepted] = w;
                        res->total_weight += w;
                        ++accepted;
                        break;
                    }
                    c ^= slot[h];
                }
            }
        }
        lo = hi + 1;
        want *= 4;
    }
    if (accepted != (size_t)rank)
        return fail(BMM_ERUNTIME,
                    "ExactBasisSolver: failed to assemble a full basis from enumerated candidates");
    return BMM_OK;
}

}  // extern "C"
