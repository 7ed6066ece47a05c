// Simulated-annealing window selector (SASelector::select,
// src/search/sa_selector.cpp:10-75, sa_selector_pairwise.cpp:21-172,
// sa_selector_higher_order.cpp:11-227).
//
// The selection is a Markov chain: every iteration draws two indices from one
// xorshift64 stream and, only when the swap does not improve the score, a
// third value for the Metropolis test; the restarts continue the same stream.
// The draw count is data-dependent, so no restart or iteration can start
// before the previous one has finished, and the chain itself is a few table
// lookups per step -- host work.  The O(rows^2 * words) part is the pairwise
// synergy table 2 * popc(r_i & r_j), which the reference rebuilds for every
// restart: here it is built once on the device (AND + POPC tiles in shared
// memory) and read back, and the chain runs on the host with the same
// generator, the same libm exp/log and the same operation order as the
// reference, so its trajectory is the reference's.
#include "common.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>
#include <vector>

namespace bmm {
namespace sa {

constexpr int kTile = 64;    // output tile (rows x rows)
constexpr int kKc = 32;      // words per K step
constexpr int kPad = kKc + 1;

// table[i][j] = 2 * popc(r_i & r_j) for i != j, 0 on the diagonal.  One CTA
// per 64 x 64 tile of the upper triangle (mirrored into the lower one) and
// per slice of `kslice` words, adding its partial counts into the zeroed table
// (integer atomics: the sum does not depend on their order); thread (ty, tx)
// owns rows 4ty.. and columns 4tx.. of the tile.
__global__ void __launch_bounds__(256)
    pairwise_table_kernel(const uint64_t* __restrict__ words, size_t stride, int rows, int W,
                          uint64_t tail, int kslice, uint32_t* __restrict__ table) {
    const int bi = blockIdx.y, bj = blockIdx.x;
    if (bi > bj)
        return;
    const int kbeg = blockIdx.z * kslice, kend = min(W, kbeg + kslice);
    __shared__ uint64_t As[kTile][kPad];
    __shared__ uint64_t Bs[kTile][kPad];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    uint32_t acc[4][4] = {};
    for (int k0 = kbeg; k0 < kend; k0 += kKc) {
        for (int i = threadIdx.x; i < kTile * kKc; i += blockDim.x) {
            const int r = i / kKc, k = i % kKc;
            const int ra = bi * kTile + r, rb = bj * kTile + r, w = k0 + k;
            uint64_t a = 0, b = 0;
            if (w < kend) {
                const uint64_t m = w == W - 1 ? tail : ~0ull;
                if (ra < rows)
                    a = words[(size_t)ra * stride + w] & m;
                if (rb < rows)
                    b = words[(size_t)rb * stride + w] & m;
            }
            As[r][k] = a;
            Bs[r][k] = b;
        }
        __syncthreads();
#pragma unroll 4
        for (int k = 0; k < kKc; ++k) {
            uint64_t a[4], b[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                a[q] = As[ty * 4 + q][k];
                b[q] = Bs[tx * 4 + q][k];
            }
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int c = 0; c < 4; ++c)
                    acc[q][c] += __popcll(a[q] & b[c]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int i = bi * kTile + ty * 4 + q, j = bj * kTile + tx * 4 + c;
            if (i < j && j < rows && acc[q][c]) {
                atomicAdd(table + (size_t)i * rows + j, 2u * acc[q][c]);
                atomicAdd(table + (size_t)j * rows + i, 2u * acc[q][c]);
            }
        }
}

int pairwise_table_launch(const uint64_t* d_words, size_t stride, size_t rows, size_t cols,
                          uint32_t* d_table, cudaStream_t s) {
    if (rows == 0)
        return BMM_OK;
    const int W = (int)((cols + 63) / 64);
    const uint64_t tail = (cols & 63) ? ((1ull << (cols & 63)) - 1) : ~0ull;
    const unsigned tiles = (unsigned)((rows + kTile - 1) / kTile);
    BMM_CUDA_TRY(cudaMemsetAsync(d_table, 0, rows * rows * 4, s));
    if (W == 0)
        return BMM_OK;
    // enough slices of the word range for about four CTAs per SM
    int dev = 0, sms = 148;
    BMM_CUDA_TRY(cudaGetDevice(&dev));
    BMM_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const long long upper = (long long)tiles * (tiles + 1) / 2;
    const int ksteps = (W + kKc - 1) / kKc;
    const int split = (int)std::max(1LL, std::min<long long>(ksteps, (4LL * sms + upper - 1) / upper));
    const int kslice = (ksteps + split - 1) / split * kKc;
    const unsigned zs = (unsigned)((W + kslice - 1) / kslice);
    pairwise_table_kernel<<<dim3(tiles, tiles, zs), 256, 0, s>>>(d_words, stride, (int)rows, W,
                                                                tail, kslice, d_table);
    BMM_CUDA_TRY(cudaGetLastError());
    return BMM_OK;
}

// detail::XorShift64 (include/bmmpy/core/detail/xorshift64.hpp:10-40).
struct Rng {
    uint64_t s;
    uint64_t next() {
        s ^= s << 13;
        s ^= s >> 7;
        s ^= s << 17;
        return s;
    }
    size_t index(size_t n) { return n == 0 ? 0 : (size_t)(next() % n); }
    double unit() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

struct Restart {
    std::vector<size_t> rows;
    int64_t score = std::numeric_limits<int64_t>::min();
    size_t accepted = 0, iterations_run = 0, best_iteration = 0;
};

// Higher score wins; equal scores prefer the lexicographically smaller sorted
// row list (sa_selector_internal.hpp:26-33).
bool better(int64_t ls, const std::vector<size_t>& lr, int64_t rs, const std::vector<size_t>& rr) {
    return ls != rs ? ls > rs : lr < rr;
}

std::vector<size_t> sorted(const std::vector<size_t>& v) {
    std::vector<size_t> o = v;
    std::sort(o.begin(), o.end());
    return o;
}

// A random t-subset by a partial Fisher-Yates shuffle; the rest is the pool.
void partition(size_t n, size_t t, Rng& rng, std::vector<size_t>& win, std::vector<size_t>& pool) {
    pool.resize(n);
    std::iota(pool.begin(), pool.end(), (size_t)0);
    for (size_t i = 0; i < t; ++i)
        std::swap(pool[i], pool[i + rng.index(n - i)]);
    win.assign(pool.begin(), pool.begin() + (ptrdiff_t)t);
    pool.erase(pool.begin(), pool.begin() + (ptrdiff_t)t);
}

// Score policies: score of a window, change of score for one swap, and the
// bookkeeping after an accepted swap.
struct Pairwise {
    const uint32_t* T;
    size_t n;
    int64_t score(const std::vector<size_t>& w) {
        int64_t s = 0;
        for (size_t i = 0; i < w.size(); ++i)
            for (size_t j = i + 1; j < w.size(); ++j)
                s += (int64_t)T[w[i] * n + w[j]];
        return s;
    }
    int64_t delta(const std::vector<size_t>& w, size_t out_idx, size_t in_row) const {
        const uint32_t* ti = T + in_row * n;
        const uint32_t* to = T + w[out_idx] * n;
        int64_t d = 0;
        for (size_t i = 0; i < w.size(); ++i)
            if (i != out_idx)
                d += (int64_t)ti[w[i]] - (int64_t)to[w[i]];
        return d;
    }
    void moved(size_t, size_t) {}
};

inline int64_t ho_term(uint32_t c) {
    const int64_t n = c;
    return n * (n - 1) * (n - 1);
}

// Column-count score sum_c n_c (n_c - 1)^2 over the window's rows.
struct HigherOrder {
    const uint64_t* words;
    size_t stride, cols, W;
    uint64_t tail;
    std::vector<uint32_t> count;
    uint64_t word(size_t r, size_t w) const {
        const uint64_t v = words[r * stride + w];
        return w + 1 == W ? v & tail : v;
    }
    int64_t score(const std::vector<size_t>& win) {
        count.assign(cols, 0u);
        for (size_t r : win)
            for (size_t w = 0; w < W; ++w)
                for (uint64_t b = word(r, w); b; b &= b - 1)
                    ++count[w * 64 + __builtin_ctzll(b)];
        int64_t s = 0;
        for (uint32_t c : count)
            s += ho_term(c);
        return s;
    }
    int64_t delta(const std::vector<size_t>& win, size_t out_idx, size_t in_row) const {
        const size_t out_row = win[out_idx];
        int64_t d = 0;
        for (size_t w = 0; w < W; ++w) {
            const uint64_t o = word(out_row, w), i = word(in_row, w);
            for (uint64_t b = o & ~i; b; b &= b - 1) {
                const uint32_t c = count[w * 64 + __builtin_ctzll(b)];
                d += ho_term(c - 1) - ho_term(c);
            }
            for (uint64_t b = i & ~o; b; b &= b - 1) {
                const uint32_t c = count[w * 64 + __builtin_ctzll(b)];
                d += ho_term(c + 1) - ho_term(c);
            }
        }
        return d;
    }
    void moved(size_t out_row, size_t in_row) {
        for (size_t w = 0; w < W; ++w) {
            const uint64_t o = word(out_row, w), i = word(in_row, w);
            for (uint64_t b = o & ~i; b; b &= b - 1)
                --count[w * 64 + __builtin_ctzll(b)];
            for (uint64_t b = i & ~o; b; b &= b - 1)
                ++count[w * 64 + __builtin_ctzll(b)];
        }
    }
};

// One restart of the annealing chain (run_pairwise_restart,
// sa_selector_pairwise.cpp:118-170; run_higher_order_restart,
// sa_selector_higher_order.cpp:171-225: same chain, different score).
template <typename Policy>
Restart run_restart(Policy& P, size_t n, size_t t, const bmm_sa_config& c, Rng& rng) {
    std::vector<size_t> win, pool;
    partition(n, t, rng, win, pool);
    int64_t score = P.score(win);
    Restart best;
    best.rows = sorted(win);
    best.score = score;
    best.iterations_run = pool.empty() ? 0 : (size_t)c.iterations;
    if (pool.empty() || c.iterations == 0)
        return best;

    // initial temperature from sampled worsening swaps
    double temp = 1.0;
    {
        const size_t samples = std::max<size_t>((size_t)c.temperature_probe_samples, 1);
        double neg_sum = 0.0;
        size_t neg = 0;
        for (size_t k = 0; k < samples; ++k) {
            const size_t iw = rng.index(win.size());
            const size_t ip = rng.index(pool.size());
            const int64_t d = P.delta(win, iw, pool[ip]);
            if (d < 0) {
                neg_sum += (double)(-d);
                ++neg;
            }
        }
        if (neg != 0) {
            const double avg = neg_sum / (double)neg;
            const double t0 = -avg / std::log(c.initial_acceptance_probability);
            temp = std::max(t0, c.min_temperature);
        }
    }

    size_t accepted = 0;
    for (size_t it = 0; it < (size_t)c.iterations; ++it) {
        const size_t iw = rng.index(win.size());
        const size_t ip = rng.index(pool.size());
        const size_t in_row = pool[ip];
        const int64_t d = P.delta(win, iw, in_row);
        bool accept = d > 0;
        if (!accept && temp > c.min_temperature) {
            const double p = std::exp((double)d / temp);
            accept = rng.unit() < p;
        }
        if (accept) {
            P.moved(win[iw], in_row);
            std::swap(win[iw], pool[ip]);
            score += d;
            ++accepted;
            std::vector<size_t> s = sorted(win);
            if (better(score, s, best.score, best.rows)) {
                best.rows = std::move(s);
                best.score = score;
                best.accepted = accepted;
                best.best_iteration = it + 1;
            }
        }
        temp = std::max(c.min_temperature, temp * c.cooling_rate);
    }
    return best;
}

}  // namespace sa
}  // namespace bmm

using namespace bmm;

extern "C" {

BMM_API int bmm_sa_pairwise_table_dev(const uint64_t* words, size_t stride, size_t rows,
                                      size_t cols, uint32_t* table, void* stream) {
    clear_error();
    if (rows && (!words || !table))
        return fail(BMM_EINVAL, "sa: null device pointer");
    if (stride < (cols + 63) / 64)
        return fail(BMM_EINVAL, "sa: stride is smaller than the row width");
    if (rows > 0x7fffffffull || cols >= (1ull << 31))
        return fail(BMM_EINVAL, "sa: matrix too large");
    return sa::pairwise_table_launch(words, stride, rows, cols, table, (cudaStream_t)stream);
}

BMM_API int bmm_sa_pairwise_table(const uint64_t* words, size_t stride, size_t rows, size_t cols,
                                  uint32_t* table) {
    clear_error();
    if (rows == 0)
        return BMM_OK;
    if (!words || !table)
        return fail(BMM_EINVAL, "sa: null pointer");
    if (stride < (cols + 63) / 64)
        return fail(BMM_EINVAL, "sa: stride is smaller than the row width");
    if (rows > 0x7fffffffull || cols >= (1ull << 31))
        return fail(BMM_EINVAL, "sa: matrix too large");
    if (rows > std::numeric_limits<size_t>::max() / rows / 4)
        return fail(BMM_EOVERFLOW, "SASelector: synergy matrix size overflow");
    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws)
        return st;
    void *d_words = nullptr, *d_table = nullptr;
    const size_t nw = std::max<size_t>(stride, 1) * rows;
    BMM_TRY(ws_buffer(ws, kSlotRows, nw * 8, &d_words));
    BMM_TRY(ws_buffer(ws, kSlotAux, rows * rows * 4, &d_table));
    BMM_CUDA_TRY(cudaMemcpyAsync(d_words, words, nw * 8, cudaMemcpyHostToDevice, ws->stream));
    BMM_TRY(sa::pairwise_table_launch((const uint64_t*)d_words, stride, rows, cols,
                                      (uint32_t*)d_table, ws->stream));
    BMM_CUDA_TRY(cudaMemcpyAsync(table, d_table, rows * rows * 4, cudaMemcpyDeviceToHost,
                                 ws->stream));
    BMM_CUDA_TRY(cudaStreamSynchronize(ws->stream));
    return BMM_OK;
}

BMM_API int bmm_sa_select(const uint64_t* words, size_t stride, size_t rows, size_t cols,
                          size_t window_size, const bmm_sa_config* cfg, bmm_sa_result* res,
                          size_t* out_rows) {
    clear_error();
    if (!cfg || !res)
        return fail(BMM_EINVAL, "sa: null config or result");
    const bmm_sa_config c = *cfg;
    // the reference's checks, in its order (sa_selector.cpp:11-29)
    if (c.restarts == 0)
        return fail(BMM_EINVAL, "SASelector: restarts must be >= 1");
    if (!(c.initial_acceptance_probability > 0.0 && c.initial_acceptance_probability < 1.0))
        return fail(BMM_EINVAL, "SASelector: initial_acceptance_probability must be in (0, 1)");
    if (c.cooling_rate <= 0.0 || c.cooling_rate > 1.0)
        return fail(BMM_EINVAL, "SASelector: cooling_rate must be in (0, 1]");
    if (c.min_temperature <= 0.0)
        return fail(BMM_EINVAL, "SASelector: min_temperature must be > 0");
    if (window_size > rows)
        return fail(BMM_EINVAL, "SASelector: window_size exceeds matrix row count");
    std::memset(res, 0, sizeof(*res));
    res->seed = c.seed == 0 ? 0x9E3779B97F4A7C15ull : c.seed;
    if (window_size == 0)
        return BMM_OK;
    if (c.cooling_policy != 0)
        return fail(BMM_EINVAL, "SASelector: unsupported cooling policy");
    if (c.score_policy > 1)
        return fail(BMM_EINVAL, "SASelector: unsupported score policy");
    if (!words || !out_rows)
        return fail(BMM_EINVAL, "sa: null matrix or output");
    if (stride < (cols + 63) / 64)
        return fail(BMM_EINVAL, "sa: stride is smaller than the row width");

    sa::Rng rng{res->seed};
    sa::Restart out;
    bool have = false;
    size_t out_restart = 0;
    auto consider = [&](sa::Restart&& r, size_t restart) {
        if (!have || sa::better(r.score, r.rows, out.score, out.rows)) {
            out = std::move(r);
            out_restart = restart;
            have = true;
        }
    };
    if (c.score_policy == 0) {
        std::vector<uint32_t> table(rows * rows);
        BMM_TRY(bmm_sa_pairwise_table(words, stride, rows, cols, table.data()));
        sa::Pairwise P{table.data(), rows};
        for (size_t r = 0; r < (size_t)c.restarts; ++r)
            consider(sa::run_restart(P, rows, window_size, c, rng), r);
    } else {
        sa::HigherOrder P{words, stride, cols, (cols + 63) / 64,
                          (cols & 63) ? ((1ull << (cols & 63)) - 1) : ~0ull, {}};
        for (size_t r = 0; r < (size_t)c.restarts; ++r)
            consider(sa::run_restart(P, rows, window_size, c, rng), r);
    }
    res->score = out.score;
    res->accepted_moves = out.accepted;
    res->iterations_run = out.iterations_run;
    res->best_iteration = out.best_iteration;
    res->restart_index = out_restart;
    res->n_rows = out.rows.size();
    std::copy(out.rows.begin(), out.rows.end(), out_rows);
    return BMM_OK;
}

}  // extern "C"
