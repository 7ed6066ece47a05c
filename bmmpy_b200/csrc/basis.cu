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
//  * enumeration on the device.  G lanes share one prefix of the high `hb`
//    mask bits, each holding WPL words of the running XOR in registers (the
//    window rows staged in shared memory); a prefix sweeps its 2^chunk low
//    bits in Gray order.  Pass 0 builds the weight histogram (per-CTA shared
//    bins), pass 1 collects the combinations whose weight lies in [lo, hi]
//    as keys (weight << 32) | enumeration index, which sorted ascending are
//    the reference's bucket order.  Windows wider than 64 words per lane x 32
//    lanes accumulate per-mask weights slab by slab instead.
//  * the greedy on r-bit coordinates.  Projecting the row space onto the
//    pivot columns of an echelon form of the window is an isomorphism, so a
//    combination's coordinate is the XOR of its rows' coordinates (four byte
//    tables) and independence is tested in a 32-slot XOR basis.
//  * only as many candidates as the greedy consumes: the weight cut starts
//    where the histogram holds 4r nonzero candidates and grows 4x per pass.
#include "common.cuh"

#include <algorithm>
#include <vector>

namespace bmm {
namespace basis {

constexpr int kThreads = 128;
constexpr int kHistSmem = 16384;  // weight bins held in shared memory (64 KB)
constexpr int kMaxWpl = 64;       // words per lane in registers
constexpr int kMaxGroup = 32;     // lanes per prefix (one warp)

enum Mode : int { kHist = 0, kCollect = 1, kAccumulate = 2 };

struct Launch {
    const uint64_t* rows;  // t x W words (one column slab in kAccumulate)
    int t, W, cols, G, hb, chunk, mode;
    uint32_t lo, hi;                // kCollect: weight range
    unsigned long long* counts;     // kHist: cols + 1 bins
    unsigned long long* keys;       // kCollect
    unsigned long long* nkeys;      // kCollect
    unsigned long long cap;         // kCollect
    uint32_t* weights;              // kAccumulate: indexed by mask
    int first;                      // kAccumulate: first slab stores, later slabs add
};

template <int WPL>
__global__ void __launch_bounds__(kThreads) enum_kernel(const Launch a) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t* srow = reinterpret_cast<uint64_t*>(smem);  // t x (G * WPL) words
    const int SW = a.G * WPL;
    unsigned* hist = reinterpret_cast<unsigned*>(srow + (size_t)a.t * SW);
    const bool shared_hist = a.mode == kHist && a.cols + 1 <= kHistSmem;
    for (int i = threadIdx.x; i < a.t * SW; i += blockDim.x) {
        const int r = i / SW, w = i % SW;
        srow[i] = w < a.W ? a.rows[(size_t)r * a.W + w] : 0ull;
    }
    if (shared_hist)
        for (int i = threadIdx.x; i <= a.cols; i += blockDim.x)
            hist[i] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int gl = lane % a.G;  // lane within the group
    const unsigned long long p =
        ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) / a.G;
    const bool valid = p < (1ull << a.hb);
    uint64_t cur[WPL];
#pragma unroll
    for (int i = 0; i < WPL; ++i)
        cur[i] = 0;
    if (valid)
        for (int b = 0; b < a.hb; ++b)
            if ((p >> b) & 1ull)
#pragma unroll
                for (int i = 0; i < WPL; ++i)
                    cur[i] ^= srow[(size_t)(a.chunk + b) * SW + gl * WPL + i];
    const uint32_t hi_bits = (uint32_t)(p << a.chunk);
    // enumeration index of mask hi|gray(s): inverse Gray of the high part on
    // top, and s itself, complemented when the high part has odd parity
    const uint32_t idx_hi = (uint32_t)(inverse_gray64(p) << a.chunk);
    const uint32_t low_flip = (__popcll(p) & 1) ? ((1u << a.chunk) - 1) : 0u;
    uint32_t low = 0;
    const uint32_t states = 1u << a.chunk;
    for (uint32_t s = 0; s < states; ++s) {
        if (s) {
            const int b = __ffs(s) - 1;
#pragma unroll
            for (int i = 0; i < WPL; ++i)
                cur[i] ^= srow[(size_t)b * SW + gl * WPL + i];
            low ^= 1u << b;
        }
        uint32_t w = 0;
#pragma unroll
        for (int i = 0; i < WPL; ++i)
            w += __popcll(cur[i]);
        for (int o = a.G >> 1; o > 0; o >>= 1)
            w += __shfl_xor_sync(kFull, w, o);
        const uint32_t mask = hi_bits | low;
        const bool lead = valid && gl == 0;
        if (a.mode == kHist) {
            if (lead && mask != 0) {
                if (shared_hist)
                    atomicAdd(hist + w, 1u);
                else
                    atomicAdd(a.counts + w, 1ull);
            }
        } else if (a.mode == kCollect) {
            const bool hit = lead && mask != 0 && w >= a.lo && w <= a.hi;
            const unsigned bal = __ballot_sync(kFull, hit);
            if (bal) {
                unsigned long long base = 0;
                if (lane == __ffs(bal) - 1)
                    base = atomicAdd(a.nkeys, (unsigned long long)__popc(bal));
                base = __shfl_sync(kFull, base, __ffs(bal) - 1);
                if (hit) {
                    const unsigned long long pos = base + __popc(bal & ((1u << lane) - 1));
                    if (pos < a.cap)
                        a.keys[pos] =
                            ((unsigned long long)w << 32) | (idx_hi | (s ^ low_flip));
                }
            }
        } else if (lead) {
            if (a.first)
                a.weights[mask] = w;
            else
                a.weights[mask] += w;
        }
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
    int G, wpl, hb, chunk;
    long long blocks;
    size_t smem;
};

// W: words per row handled by one launch (the whole row, or one slab).
Plan plan_for(int t, int W, int cols, int sm_count) {
    Plan p{};
    p.G = 1;
    while ((W + p.G - 1) / p.G > kMaxWpl)
        p.G <<= 1;
    const int need = (W + p.G - 1) / p.G;
    p.wpl = 1;
    while (p.wpl < need)
        p.wpl <<= 1;
    // prefixes for about 8 CTAs of 128 threads per SM, each sweeping at least
    // 2^min(6, t) states, and chunk <= 31 so a sweep counts in 32 bits
    const long long want = (long long)sm_count * 8 * kThreads / p.G;
    int hb = 0;
    while (hb < t && (2ll << hb) <= want && t - (hb + 1) >= std::min(6, t))
        ++hb;
    if (t - hb > 31)
        hb = t - 31;
    p.hb = hb;
    p.chunk = t - hb;
    const long long threads = (1ll << hb) * p.G;
    p.blocks = (threads + kThreads - 1) / kThreads;
    p.smem = (size_t)t * p.G * p.wpl * 8 + (size_t)(cols + 1 <= kHistSmem ? (cols + 1) * 4 : 0);
    // G * WPL is the power of two at or above W, and W <= slab_words(t)
    return p;
}

int launch(const Plan& pl, Launch a, cudaStream_t s) {
    a.G = pl.G;
    a.hb = pl.hb;
    a.chunk = pl.chunk;
#define BMM_ENUM(N)                                                                               \
    case N: {                                                                                     \
        auto k = enum_kernel<N>;                                                                  \
        BMM_CUDA_TRY(                                                                             \
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl.smem));  \
        k<<<(unsigned)pl.blocks, kThreads, pl.smem, s>>>(a);                                      \
        BMM_CUDA_TRY(cudaGetLastError());                                                         \
        return BMM_OK;                                                                            \
    }
    switch (pl.wpl) {
        BMM_ENUM(1)
        BMM_ENUM(2)
        BMM_ENUM(4)
        BMM_ENUM(8)
        BMM_ENUM(16)
        BMM_ENUM(32)
        BMM_ENUM(64)
    }
#undef BMM_ENUM
    return fail(BMM_EINVAL, "exact basis: unsupported row width");
}

// Widest row slab one launch handles: G * WPL words per row for all t rows
// in shared memory (at most 192 KB; cols < 16384 also keeps a 64 KB histogram,
// and those rows are at most 256 words).
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
    int t = 0, cols = 0;
    size_t W = 0, slab = 0;
    uint64_t* d_rows = nullptr;
    uint32_t* d_weights = nullptr;  // wide windows only
    unsigned long long states = 0;

    bool wide() const { return W > slab; }

    int init(Workspace* w, const uint64_t* words, size_t stride, size_t ncols,
             const uint32_t* win, size_t nt) {
        ws = w;
        t = (int)nt;
        cols = (int)ncols;
        W = (ncols + 63) / 64;
        slab = slab_words(t);
        states = (1ull << nt) - 1;
        const size_t slabs = (W + slab - 1) / slab;
        // narrow: row r at r * W; wide: slab j of row r at (j * t + r) * slab
        std::vector<uint64_t> h(wide() ? slabs * nt * slab : nt * std::max<size_t>(W, 1), 0ull);
        const uint64_t tail = (ncols & 63) ? ((1ull << (ncols & 63)) - 1) : ~0ull;
        for (size_t r = 0; r < nt; ++r)
            for (size_t c = 0; c < W; ++c) {
                const uint64_t v = words[(size_t)win[r] * stride + c] & (c == W - 1 ? tail : ~0ull);
                if (wide())
                    h[((c / slab) * nt + r) * slab + c % slab] = v;
                else
                    h[r * W + c] = v;
            }
        void* p = nullptr;
        BMM_TRY(ws_buffer(ws, kSlotRows, h.size() * 8, &p));
        BMM_CUDA_TRY(cudaMemcpyAsync(p, h.data(), h.size() * 8, cudaMemcpyHostToDevice,
                                     ws->stream));
        d_rows = (uint64_t*)p;
        if (wide()) {
            void* q = nullptr;
            BMM_TRY(ws_buffer(ws, kSlotExtra0, (size_t)(states + 1) * 4, &q));
            d_weights = (uint32_t*)q;
            const Plan pl = plan_for(t, (int)slab, cols, ws->sm_count);
            for (size_t j = 0; j < slabs; ++j) {
                Launch a{};
                a.rows = d_rows + j * nt * slab;
                a.t = t;
                a.W = (int)slab;
                a.cols = cols;
                a.mode = kAccumulate;
                a.weights = d_weights;
                a.first = j == 0;
                BMM_TRY(launch(pl, a, ws->stream));
            }
        }
        return BMM_OK;
    }

    int hist(unsigned long long* d_counts) {
        BMM_CUDA_TRY(cudaMemsetAsync(d_counts, 0, ((size_t)cols + 1) * 8, ws->stream));
        if (wide()) {
            const unsigned blocks = (unsigned)std::min<unsigned long long>(
                (states + 255) / 256, (unsigned long long)ws->sm_count * 16);
            weights_hist_kernel<<<blocks, 256, 0, ws->stream>>>(d_weights, states, d_counts);
            BMM_CUDA_TRY(cudaGetLastError());
            return BMM_OK;
        }
        Launch a{};
        a.rows = d_rows;
        a.t = t;
        a.W = (int)W;
        a.cols = cols;
        a.mode = kHist;
        a.counts = d_counts;
        return launch(plan_for(t, (int)W, cols, ws->sm_count), a, ws->stream);
    }

    int collect(uint32_t lo, uint32_t hi, unsigned long long* d_keys, unsigned long long cap,
                unsigned long long* d_n) {
        BMM_CUDA_TRY(cudaMemsetAsync(d_n, 0, 8, ws->stream));
        if (wide()) {
            const unsigned blocks = (unsigned)std::min<unsigned long long>(
                (states + 256) / 256, (unsigned long long)ws->sm_count * 16);
            weights_collect_kernel<<<blocks, 256, 0, ws->stream>>>(d_weights, states, lo, hi,
                                                                   d_keys, d_n, cap);
            BMM_CUDA_TRY(cudaGetLastError());
            return BMM_OK;
        }
        Launch a{};
        a.rows = d_rows;
        a.t = t;
        a.W = (int)W;
        a.cols = cols;
        a.mode = kCollect;
        a.lo = lo;
        a.hi = hi;
        a.keys = d_keys;
        a.nkeys = d_n;
        a.cap = cap;
        return launch(plan_for(t, (int)W, cols, ws->sm_count), a, ws->stream);
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
