// Device-resident search -> apply over a list of windows of one matrix
// (bmmpy/workflows.py:45-90 search_apply with MitmFwhtSearch / FwhtSearch and
// GreedyApplier, src/apply/greedy_applier.cpp:13-109, or GlobalGreedyApplier,
// src/apply/global_greedy_applier.cpp:59-105), without host round trips: per
// window, on one stream,
//   gather    the window's rows from the device matrix (and their weights),
//   search    the exact top-k spectrum search of the window searchers,
//   decide    the applier's bookkeeping in one thread: which candidates apply
//             and to which row -- decisions depend only on candidate masks and
//             weights, the row weights and the row-space basis c[], never on
//             row contents -- summarised as the window transform T (new row i
//             = XOR of the old rows in T[i]),
//   apply     new rows = T x old rows, written back to the matrix.
// The greedy applier XORs rows one candidate at a time; composing those XORs
// into T first and applying T once gives the same rows.  The global applier
// computes the new rows' exact total weight before committing, as the
// reference does.
#include "common.cuh"
#include "spectrum.cuh"

#include <algorithm>
#include <cstring>
#include <vector>

namespace bmm {
namespace sweep {

constexpr int kMaxT = 64;

struct WinState {
    unsigned long long rowpop[kMaxT];  // weights of the window rows
    unsigned long long T[kMaxT];       // transform masks
    unsigned long long old_weight, new_weight;
    unsigned long long applied, improvement;  // ApplyResult of the window
    int changed;                              // T != identity
    int error;                                // global applier: no full transform
    int skipped;                              // not searched: an earlier window failed
};

// Window rows into a packed t x W block; row weights into the state.
__global__ void gather_kernel(const uint64_t* __restrict__ words, size_t stride, int W,
                              const uint32_t* __restrict__ win, int t,
                              uint64_t* __restrict__ packed, WinState* __restrict__ st) {
    const int r = blockIdx.y;
    const uint64_t* src = words + (size_t)win[r] * stride;
    unsigned long long pop = 0;
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < W; w += gridDim.x * blockDim.x) {
        const uint64_t v = src[w];
        packed[(size_t)r * W + w] = v;
        pop += __popcll(v);
    }
    for (int o = 16; o > 0; o >>= 1)
        pop += __shfl_xor_sync(kFull, pop, o);
    if ((threadIdx.x & 31) == 0 && pop)
        atomicAdd(&st->rowpop[r], pop);
}

struct Rng {
    unsigned long long s;
    __device__ unsigned long long next() {
        s ^= s << 13;
        s ^= s >> 7;
        s ^= s << 17;
        return s;
    }
};

// GreedyApplier::apply (src/apply/greedy_applier.cpp:13-109) on the candidate
// list of one window, in one thread.  order[] is scratch for kk indices.
__global__ void greedy_decide_kernel(const bmm_candidate* __restrict__ cands, int kk, int t,
                                     unsigned long long min_gain, int stochastic,
                                     unsigned long long* __restrict__ rng_state,
                                     int* __restrict__ order, const int* __restrict__ abort_flag,
                                     WinState* __restrict__ st) {
    if (threadIdx.x != 0 || blockIdx.x != 0)
        return;
    if (*abort_flag) {  // an earlier window failed: the sweep stops there
        st->skipped = 1;
        st->changed = 0;
        return;
    }
    int n = 0;
    for (int i = 0; i < kk; ++i)
        if (cands[i].weight != 0xffffffffu)
            order[n++] = i;
    Rng rng{*rng_state};
    if (stochastic) {
        for (int i = n; i > 1; --i) {
            const int j = (int)(rng.next() % (unsigned long long)i);
            const int x = order[i - 1];
            order[i - 1] = order[j];
            order[j] = x;
        }
        // stable sort by weight (insertion sort keeps equal weights in order)
        for (int i = 1; i < n; ++i) {
            const int x = order[i];
            const uint32_t wx = cands[x].weight;
            int j = i - 1;
            while (j >= 0 && cands[order[j]].weight > wx) {
                order[j + 1] = order[j];
                --j;
            }
            order[j + 1] = x;
        }
    }
    unsigned long long c[kMaxT], cur[kMaxT];
    for (int i = 0; i < t; ++i) {
        c[i] = 1ull << i;
        cur[i] = st->rowpop[i];
        st->T[i] = 1ull << i;
    }
    unsigned long long applied = 0, gain_sum = 0;
    int changed = 0;
    for (int q = 0; q < n; ++q) {
        const bmm_candidate cd = cands[order[q]];
        unsigned long long a = 0;
        for (int i = 0; i < t; ++i)
            a |= (unsigned long long)(__popcll(cd.mask & c[i]) & 1) << i;
        if (a == 0)
            continue;
        int best[kMaxT];
        int nb = 0;
        unsigned long long best_gain = 0;
        for (int r = 0; r < t; ++r) {
            if (!((a >> r) & 1ull))
                continue;
            const unsigned long long old_w = cur[r], cw = cd.weight;
            if (old_w <= cw)
                continue;
            const unsigned long long gain = old_w - cw;
            if (gain < min_gain)
                continue;
            if (gain > best_gain) {
                best_gain = gain;
                best[0] = r;
                nb = 1;
            } else if (gain == best_gain) {
                best[nb++] = r;
            }
        }
        if (nb == 0)
            continue;
        const int ch = stochastic ? best[rng.next() % (unsigned long long)nb] : best[0];
        unsigned long long acc = 0;
        for (int i = 0; i < t; ++i)
            if ((a >> i) & 1ull)
                acc ^= st->T[i];
        st->T[ch] = acc;
        cur[ch] = cd.weight;
        for (int j = 0; j < t; ++j)
            if (j != ch && ((a >> j) & 1ull))
                c[j] ^= c[ch];
        ++applied;
        gain_sum += best_gain;
        changed = 1;
    }
    *rng_state = rng.s;
    st->applied = applied;
    st->improvement = gain_sum;
    st->changed = changed;
}

// GlobalGreedyApplier (src/apply/global_greedy_applier.cpp:30-91): candidates
// and unit rows in one pool, stable-sorted by weight, inserted into a pivot
// basis (pivot = highest set bit) until t are independent; T = the chosen
// masks.  One thread; order[] is scratch for kk + t entries.  A window that
// cannot assemble t independent masks sets *abort_flag, and every later window
// of the call becomes a no-op, as the reference loop stops at the exception
// (with the unit rows in the pool this cannot happen for valid candidates).
__global__ void global_decide_kernel(const bmm_candidate* __restrict__ cands, int kk, int t,
                                     int* __restrict__ order, int* __restrict__ abort_flag,
                                     WinState* __restrict__ st) {
    if (threadIdx.x != 0 || blockIdx.x != 0)
        return;
    if (*abort_flag) {
        st->skipped = 1;
        st->changed = 0;
        return;
    }
    int n = 0;
    for (int i = 0; i < kk; ++i)
        if (cands[i].weight != 0xffffffffu)
            order[n++] = i;
    for (int r = 0; r < t; ++r)
        order[n++] = kk + r;  // unit row r
    auto weight_of = [&](int e) -> unsigned long long {
        return e < kk ? (unsigned long long)cands[e].weight : st->rowpop[e - kk];
    };
    auto mask_of = [&](int e) -> unsigned long long {
        return e < kk ? cands[e].mask : (1ull << (e - kk));
    };
    for (int i = 1; i < n; ++i) {
        const int x = order[i];
        const unsigned long long wx = weight_of(x);
        int j = i - 1;
        while (j >= 0 && weight_of(order[j]) > wx) {
            order[j + 1] = order[j];
            --j;
        }
        order[j + 1] = x;
    }
    unsigned long long basis[kMaxT] = {};
    int chosen = 0;
    for (int q = 0; q < n && chosen < t; ++q) {
        const unsigned long long m0 = mask_of(order[q]);
        unsigned long long v = m0;
        while (v) {
            const int h = 63 - __clzll(v);
            if (!basis[h]) {
                basis[h] = v;
                st->T[chosen++] = m0;
                break;
            }
            v ^= basis[h];
        }
    }
    st->error = chosen != t;
    st->changed = chosen == t;
    if (chosen != t)
        *abort_flag = 1;
}

// rows_out[i] = XOR of rows_in[j] for j in T[i] (t x W, word-parallel).
__global__ void transform_kernel(const uint64_t* __restrict__ rows_in, int t, int W,
                                 const WinState* __restrict__ st, uint64_t* __restrict__ rows_out,
                                 unsigned long long* __restrict__ weight) {
    if (!st->changed)
        return;
    unsigned long long pop = 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)t * W;
         e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e / W), w = (int)(e % W);
        uint64_t v = 0;
        for (unsigned long long m = st->T[i]; m; m &= m - 1)
            v ^= rows_in[(size_t)(__ffsll((long long)m) - 1) * W + w];
        rows_out[e] = v;
        pop += __popcll(v);
    }
    if (weight) {
        for (int o = 16; o > 0; o >>= 1)
            pop += __shfl_xor_sync(kFull, pop, o);
        if ((threadIdx.x & 31) == 0 && pop)
            atomicAdd(weight, pop);
    }
}

// Rows back into the matrix.  Greedy: whenever T changed.  Global: only when
// the new weight does not exceed the old (and is smaller, when improvement is
// required); records the ApplyResult.
__global__ void scatter_kernel(const uint64_t* __restrict__ rows, int t, int W,
                               const uint32_t* __restrict__ win, uint64_t* __restrict__ words,
                               size_t stride, WinState* __restrict__ st, int global,
                               int require_improvement) {
    if (!st->changed)
        return;
    if (global) {
        unsigned long long old_w = 0;
        for (int r = 0; r < t; ++r)
            old_w += st->rowpop[r];
        const unsigned long long new_w = st->new_weight;
        const bool ok = new_w < old_w || (new_w == old_w && !require_improvement);
        if (!ok)
            return;
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            st->applied = 1;
            st->improvement = old_w - new_w;
        }
    }
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)t * W;
         e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e / W), w = (int)(e % W);
        words[(size_t)win[i] * stride + w] = rows[e];
    }
}

}  // namespace sweep
}  // namespace bmm

using namespace bmm;

extern "C" {

BMM_API int bmm_search_apply_dev(uint64_t* words, size_t rows, size_t stride, size_t cols,
                                 const uint32_t* windows, size_t t, size_t n_windows,
                                 const bmm_sweep_config* cfg, bmm_apply_result* results,
                                 uint64_t* final_state, void* stream) {
    clear_error();
    if (!cfg || !results || (n_windows && (!windows || !words)))
        return fail(BMM_EINVAL, "search_apply: null argument");
    if (n_windows == 0)
        return BMM_OK;
    if (t == 0 || t > (size_t)sweep::kMaxT)
        return fail(BMM_EINVAL, "search_apply: window rows must be in [1, 64]");
    if (t > 40)
        return fail(BMM_EINVAL, "search_apply: 2^%zu combinations cannot be enumerated", t);
    if (cfg->applier > 1)
        return fail(BMM_EINVAL, "search_apply: unknown applier");
    const size_t W = (cols + 63) / 64;
    if (stride < W)
        return fail(BMM_EINVAL, "search_apply: stride is smaller than the row width");
    if (cols > 0x7fffffffull)
        return fail(BMM_EOVERFLOW, "search_apply: total weight exceeds int32 range");
    const size_t states = ((size_t)1 << t) - 1;
    const size_t kk = std::min<size_t>(cfg->max_candidates, states);
    if (kk > 1024)
        return fail(BMM_EINVAL, "search_apply: max_candidates above 1024 is not supported");
    // every row index is checked here, before anything is launched: the
    // kernels index the matrix with them unchecked
    for (size_t i = 0; i < n_windows * t; ++i)
        if ((size_t)windows[i] >= rows)
            return fail(BMM_EINVAL, "search_apply: row index %u out of range (rows = %zu)",
                        windows[i], rows);
    for (size_t q = 0; q < n_windows; ++q)
        for (size_t i = 0; i < t; ++i)
            for (size_t j = 0; j < i; ++j)
                if (windows[q * t + i] == windows[q * t + j])
                    return fail(BMM_EINVAL, "search_apply: window rows must be unique");
    std::memset(results, 0, n_windows * sizeof(bmm_apply_result));
    const unsigned long long seed = cfg->seed == 0 ? 0xDEADBull : cfg->seed;
    if (final_state)
        *final_state = seed;
    if (W == 0 || kk == 0)
        return BMM_OK;
    int st_ = 0;
    Workspace* ws = workspace(&st_);
    if (!ws)
        return st_;
    cudaStream_t s = (cudaStream_t)stream;
    // scratch: window lists, packed rows (old, new), candidates, states, rng,
    // the sticky abort flag
    void *d_win = nullptr, *d_rows = nullptr, *d_new = nullptr, *d_cand = nullptr,
         *d_state = nullptr, *d_order = nullptr, *d_rng = nullptr;
    // (the spectrum search allocates its own slots; these are not among them)
    BMM_TRY(ws_buffer(ws, kSlotSweepWin, n_windows * t * 4, &d_win));
    BMM_TRY(ws_buffer(ws, kSlotRows, t * W * 8, &d_rows));
    BMM_TRY(ws_buffer(ws, kSlotSweepNew, t * W * 8, &d_new));
    BMM_TRY(ws_buffer(ws, kSlotOut, kk * sizeof(bmm_candidate), &d_cand));
    BMM_TRY(ws_buffer(ws, kSlotSweepState, n_windows * sizeof(sweep::WinState), &d_state));
    BMM_TRY(ws_buffer(ws, kSlotSweepOrder, (kk + t) * sizeof(int) + 32, &d_order));
    d_rng = (char*)d_order + (kk + t) * sizeof(int);
    d_rng = (void*)(((uintptr_t)d_rng + 7) & ~(uintptr_t)7);
    int* d_abort = (int*)((char*)d_rng + 8);
    BMM_CUDA_TRY(cudaMemcpyAsync(d_win, windows, n_windows * t * 4, cudaMemcpyHostToDevice, s));
    BMM_CUDA_TRY(cudaMemcpyAsync(d_rng, &seed, 8, cudaMemcpyHostToDevice, s));
    BMM_CUDA_TRY(cudaMemsetAsync(d_state, 0, n_windows * sizeof(sweep::WinState), s));
    BMM_CUDA_TRY(cudaMemsetAsync(d_abort, 0, sizeof(int), s));
    sweep::WinState* states_d = (sweep::WinState*)d_state;
    const unsigned gx = (unsigned)std::min<size_t>((W + 255) / 256, 64);
    const unsigned tb = (unsigned)std::min<size_t>((t * W + 255) / 256, (size_t)ws->sm_count * 4);
    for (size_t q = 0; q < n_windows; ++q) {
        const uint32_t* win = (const uint32_t*)d_win + q * t;
        sweep::WinState* st = states_d + q;
        sweep::gather_kernel<<<dim3(gx, (unsigned)t), 256, 0, s>>>(words, stride, (int)W, win,
                                                                  (int)t, (uint64_t*)d_rows, st);
        BMM_CUDA_TRY(cudaGetLastError());
        BMM_TRY(spectrum_topk_launch(ws, (const uint64_t*)d_rows, (int)t, (int)W,
                                     (long long)cols, (int)kk, (bmm_candidate*)d_cand, s));
        if (cfg->applier == 0) {
            sweep::greedy_decide_kernel<<<1, 32, 0, s>>>(
                (const bmm_candidate*)d_cand, (int)kk, (int)t, cfg->min_gain,
                cfg->stochastic ? 1 : 0, (unsigned long long*)d_rng, (int*)d_order, d_abort, st);
            sweep::transform_kernel<<<tb, 256, 0, s>>>((const uint64_t*)d_rows, (int)t, (int)W,
                                                       st, (uint64_t*)d_new, nullptr);
        } else {
            sweep::global_decide_kernel<<<1, 32, 0, s>>>((const bmm_candidate*)d_cand, (int)kk,
                                                         (int)t, (int*)d_order, d_abort, st);
            sweep::transform_kernel<<<tb, 256, 0, s>>>((const uint64_t*)d_rows, (int)t, (int)W,
                                                       st, (uint64_t*)d_new, &st->new_weight);
        }
        sweep::scatter_kernel<<<tb, 256, 0, s>>>((const uint64_t*)d_new, (int)t, (int)W, win,
                                                 words, stride, st, (int)cfg->applier,
                                                 cfg->require_improvement ? 1 : 0);
        BMM_CUDA_TRY(cudaGetLastError());
    }
    std::vector<sweep::WinState> h(n_windows);
    BMM_CUDA_TRY(cudaMemcpyAsync(h.data(), d_state, n_windows * sizeof(sweep::WinState),
                                 cudaMemcpyDeviceToHost, s));
    unsigned long long last = seed;
    BMM_CUDA_TRY(cudaMemcpyAsync(&last, d_rng, 8, cudaMemcpyDeviceToHost, s));
    BMM_CUDA_TRY(cudaStreamSynchronize(s));
    if (final_state)
        *final_state = last;
    for (size_t q = 0; q < n_windows; ++q) {
        if (h[q].error)
            return fail(BMM_ERUNTIME,
                        "GlobalGreedyApplier: failed to assemble a full invertible transform");
        results[q].applied_count = h[q].applied;
        results[q].weight_improvement = h[q].improvement;
    }
    return BMM_OK;
}

}  // extern "C"
