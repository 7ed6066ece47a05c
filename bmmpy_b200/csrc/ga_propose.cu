// Learned proposal step of the genetic algorithm (no reference counterpart:
// the reference mutates with uniformly drawn row pairs, operators.cpp:100-129).
//
// Per generation, for qpc target rows i of every elite individual (the
// islands' best, copied into the next population):
//  1. features_kernel: the network input of (individual, i): the exact
//     relative weight change d_j = (w_j - 2 popc(r_i & r_j)) / w_i that
//     XORing r_j into r_i would cause, for the rows j ranked by d_j, then the
//     ±1 bits of r_i's 256-column sketch (r_i sampled at 256 fixed columns);
//  2. the proposal network (mlp.cu, tcgen05 GEMMs) scores every rank position;
//  3. search_kernel: a window of 16 rows j != i is drawn -- Gumbel-top-16 of
//     the position scores (learned), or uniformly -- and the exact best subset of the
//     window to XOR into r_i is found by the packed FWHT over all 2^16 subsets
//     (target_item.cuh); an improving subset is applied (row, mask and exact
//     weight) and becomes a training example whose target spreads the mass
//     evenly over the rank positions of the subset's rows;
//  4. the improving examples, compacted in query order, train the network
//     with `train_steps` Adam steps.
// The share of learned windows adapts to the measured success rates of
// learned and uniform windows (the uniform draw stays as the fallback and the
// yardstick the learned windows are compared with).
// All random draws are counter-based hashes of (seed, generation, query), so
// a run is deterministic for a seed.
#include "common.cuh"
#include "ga.cuh"
#include "mlp.cuh"
#include "target_item.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace bmm {
namespace ga {

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

__device__ __forceinline__ uint64_t qhash(uint64_t seed, unsigned long long gen, uint64_t q,
                                          uint64_t salt) {
    return mix64(seed ^ mix64(gen * 0x100000001B3ull ^ mix64(q * 0x9E37ull + salt)));
}

// uniform in (0, 1)
__device__ __forceinline__ float hunit(uint64_t h) {
    return ((float)(h >> 40) + 0.5f) * (1.0f / 16777216.0f);
}

// Query q works on elite e of island `island` (the island's e-th best,
// copied unchanged into the next population): slot cs = island * P + e.
__device__ __forceinline__ uint32_t query_slot(const State& st, const PropBuf& pb, uint64_t q) {
    const uint64_t per_island = (uint64_t)st.c.E * pb.qpc;
    const uint32_t island = (uint32_t)(q / per_island);
    const uint32_t e = (uint32_t)((q % per_island) / pb.qpc);
    return island * st.c.P + e;
}

// CTA (256 threads) per query: exact overlaps popc(r_i & r_j) for every row
// j (warp per j, lanes over words) give the pairwise weight changes
// d_j = (w_j - 2 ov_ij) / w_i; the rows are ranked by (d_j, j) (bitonic sort;
// row i and rows past N last) and the network input is
// [d of the rank-k row for k < 256 | ±1 sketch bits of r_i]; perm[q][k] is
// the rank-k row, so the network scores rank positions.
constexpr float kNoRow = 1e30f;

__global__ void __launch_bounds__(256) features_kernel(State st, PropBuf pb,
                                                       unsigned long long gen) {
    __shared__ float sd[256];
    __shared__ uint16_t sj[256];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    const int N = st.c.N, W = st.c.W;
    const uint64_t Q = (uint64_t)st.I * st.c.E * pb.qpc;
    for (uint64_t q = blockIdx.x; q < Q; q += gridDim.x) {
        const uint32_t cs = query_slot(st, pb, q);
        const IslandStat& is = st.stat[cs / st.c.P];
        if (!is.stepped)
            continue;
        const Pop p = st.pop[is.cur ^ 1];
        const uint64_t* R = p.rows + (size_t)cs * N * W;
        const uint32_t* wt = p.wts + (size_t)cs * N;
        const int i = (int)(qhash(pb.seed, gen, q, 0x7a) % (uint64_t)N);
        if (tid == 0)
            pb.target[q] = (uint16_t)i;
        const float wi = (float)max(wt[i], 1u);
        const uint64_t* ri = R + (size_t)i * W;
        for (int j = warp; j < 256; j += nw) {
            float d = kNoRow;
            if (j < N && j != i) {
                uint32_t ov = 0;
                const uint64_t* rj = R + (size_t)j * W;
                for (int w = lane; w < W; w += 32)
                    ov += __popcll(ri[w] & rj[w]);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1)
                    ov += __shfl_xor_sync(kFull, ov, o);
                d = ((float)wt[j] - 2.f * (float)ov) / wi;
            }
            if (lane == 0) {
                sd[j] = d;
                sj[j] = (uint16_t)j;
            }
        }
        __syncthreads();
        for (int size = 2; size <= 256; size <<= 1)
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
                const int o = tid ^ stride;
                if (o > tid) {
                    const bool up = (tid & size) == 0;
                    const bool gt = sd[tid] > sd[o] || (sd[tid] == sd[o] && sj[tid] > sj[o]);
                    if (gt == up) {
                        const float t0 = sd[tid];
                        sd[tid] = sd[o];
                        sd[o] = t0;
                        const uint16_t u0 = sj[tid];
                        sj[tid] = sj[o];
                        sj[o] = u0;
                    }
                }
                __syncthreads();
            }
        __nv_bfloat16* x = pb.X + q * 512;
        const float d = sd[tid];
        x[tid] = __float2bfloat16_rn(d >= kNoRow ? 4.f : d);
        pb.perm[q * 256 + tid] = sj[tid];
        const uint32_t c = pb.cols[tid];
        x[256 + tid] = __float2bfloat16_rn(((ri[c >> 6] >> (c & 63)) & 1ull) ? 1.f : -1.f);
        __syncthreads();
    }
}

struct WinOthers {
    const uint16_t* w;
    __device__ __forceinline__ uint32_t operator()(int j) const { return w[j]; }
};

// CTA (512 threads, 128 KB of shared memory) per elite individual; its
// queries in order (a later query sees the moves of the earlier ones; its
// features were computed before them).
__global__ void __launch_bounds__(item::kFwht16Threads)
    search_kernel(State st, PropBuf pb, unsigned long long gen, int cols) {
    extern __shared__ __align__(16) int32_t Psm[];
    __shared__ uint32_t red[16];
    __shared__ uint16_t win[16];   // rows of the window
    __shared__ uint16_t wpos[16];  // their rank positions
    __shared__ uint64_t s_out_s;
    __shared__ uint32_t s_out_w;
    __shared__ int s_learned;
    const int N = st.c.N, W = st.c.W, P = st.c.P;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t E = (uint32_t)st.c.E;
    for (uint32_t es = blockIdx.x; es < (uint32_t)st.I * E; es += gridDim.x) {
        const uint32_t cs = (es / E) * P + es % E;
        const IslandStat& is = st.stat[cs / P];
        if (!is.stepped)
            continue;
        const Pop p = st.pop[is.cur ^ 1];
        uint64_t* R = p.rows + (size_t)cs * N * W;
        uint64_t* M = p.masks + (size_t)cs * N * 4;
        uint32_t* Wt = p.wts + (size_t)cs * N;
        for (int r = 0; r < pb.qpc; ++r) {
            const uint64_t q = (uint64_t)es * pb.qpc + r;
            const int i = pb.target[q];
            if (warp == 0) {
                const bool learned =
                    pb.mode == 1 && hunit(qhash(pb.seed, gen, q, 0x51)) < pb.learned_frac;
                // rank positions 0 .. N-2 hold the N-1 rows other than i
                float sc[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const int pos = lane + 32 * k;
                    if (pos >= N - 1) {
                        sc[k] = -INFINITY;
                    } else {
                        const float u = hunit(qhash(pb.seed, gen, q, 0x1000 + pos));
                        const float gum = -logf(-logf(u));
                        sc[k] = pb.mode == 3 ? -(float)pos  // the 16 best-ranked rows
                                : learned    ? pb.logits[q * 256 + pos] + gum
                                             : gum;
                    }
                }
                for (int t = 0; t < 16; ++t) {  // Gumbel-top-16: sampling without replacement
                    float bv = -INFINITY;
                    int bj = 1 << 30;
#pragma unroll
                    for (int k = 0; k < 8; ++k)
                        if (sc[k] > bv) {
                            bv = sc[k];
                            bj = lane + 32 * k;
                        }
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        const float ov = __shfl_xor_sync(kFull, bv, o);
                        const int oj = __shfl_xor_sync(kFull, bj, o);
                        if (ov > bv || (ov == bv && oj < bj)) {
                            bv = ov;
                            bj = oj;
                        }
                    }
#pragma unroll
                    for (int k = 0; k < 8; ++k)
                        if (lane + 32 * k == bj)
                            sc[k] = -INFINITY;
                    if (lane == 0) {
                        wpos[t] = (uint16_t)bj;
                        win[t] = pb.perm[q * 256 + bj];
                    }
                }
                if (lane == 0)
                    s_learned = learned ? 1 : 0;
            }
            __syncthreads();
            item::fwht16(Psm, red, R, W, cols, WinOthers{win}, (uint32_t)i, &s_out_s, &s_out_w);
            const uint32_t wi = Wt[i], wnew = s_out_w;
            const uint32_t S = (uint32_t)s_out_s;
            const bool improved = wnew < wi;
            const int learned = s_learned;
            if (tid == 0) {
                atomicAdd(pb.counters + (learned ? 0 : 2), 1ull);
                if (improved)
                    atomicAdd(pb.counters + (learned ? 1 : 3), 1ull);
                pb.valid[q] = improved ? 1 : 0;
            }
            if (improved) {
                for (int w = tid; w < W; w += blockDim.x) {
                    uint64_t acc = R[(size_t)i * W + w];
                    for (int t = 0; t < 16; ++t)
                        if ((S >> t) & 1u)
                            acc ^= R[(size_t)win[t] * W + w];
                    R[(size_t)i * W + w] = acc;
                }
                if (tid < 4) {
                    uint64_t acc = M[i * 4 + tid];
                    for (int t = 0; t < 16; ++t)
                        if ((S >> t) & 1u)
                            acc ^= M[win[t] * 4 + tid];
                    M[i * 4 + tid] = acc;
                }
                if (tid == 0)
                    Wt[i] = wnew;
                const float share = 1.f / (float)__popc(S);
                for (int pos = tid; pos < 256; pos += blockDim.x) {
                    float v = 0.f;
                    for (int t = 0; t < 16; ++t)
                        if (wpos[t] == pos && ((S >> t) & 1u))
                            v = share;
                    pb.T[q * 256 + pos] = v;
                }
            }
            __syncthreads();
        }
    }
}

// Single CTA: indices of the improving queries in query order, at most cap.
__global__ void compact_kernel(const uint8_t* __restrict__ valid, uint64_t Q, uint32_t* idx,
                               int cap, int* count) {
    __shared__ int warp_sum[32];
    __shared__ int s_base;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0)
        s_base = 0;
    __syncthreads();
    for (uint64_t b = 0; b < Q; b += blockDim.x) {
        const uint64_t q = b + tid;
        const int f = (q < Q && valid[q]) ? 1 : 0;
        const unsigned m = __ballot_sync(kFull, f);
        const int pre = __popc(m & ((1u << lane) - 1u));
        if (lane == 0)
            warp_sum[warp] = __popc(m);
        __syncthreads();
        int off = 0;
        for (int w = 0; w < warp; ++w)
            off += warp_sum[w];
        const int pos = s_base + off + pre;
        if (f && pos < cap)
            idx[pos] = (uint32_t)q;
        __syncthreads();
        if (tid == 0) {
            int t = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
                t += warp_sum[w];
            s_base += t;
        }
        __syncthreads();
    }
    if (tid == 0)
        *count = s_base < cap ? s_base : cap;
}

// Block per new example b: append the query's inputs and targets to the
// replay ring at (head + b) mod kPropBatchCap.
__global__ void gather_kernel(PropBuf pb, const uint32_t* __restrict__ idx, int head) {
    const int b = blockIdx.x;
    const uint64_t q = idx[b];
    const size_t dst = (size_t)((head + b) % kPropBatchCap);
    for (int k = threadIdx.x; k < 512; k += blockDim.x)
        pb.Xb[dst * 512 + k] = pb.X[q * 512 + k];
    for (int k = threadIdx.x; k < 256; k += blockDim.x)
        pb.Tb[dst * 256 + k] = pb.T[q * 256 + k];
}

// ---------------------------------------------------------------------------
namespace {
int palloc(bmm_ga* g, size_t bytes, void** p) {
    const cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return fail(BMM_ENOMEM, "ga: proposal buffers (%zu bytes) failed: %s", bytes,
                    cudaGetErrorString(e));
    }
    g->allocs.push_back(*p);
    return BMM_OK;
}
}  // namespace

int propose_setup(bmm_ga* g, int mode, int qpc, int train_steps, float lr, float learned_frac,
                  uint64_t seed) {
    const Config& c = g->st.c;
    PropBuf& pb = g->prop;
    const uint64_t Q = (uint64_t)g->I * c.E * qpc;
    pb.mode = mode;
    pb.qpc = qpc;
    pb.seed = seed;
    pb.learned_frac = learned_frac;
    g->train_steps = train_steps;
    void* p = nullptr;
    BMM_TRY(palloc(g, 256 * 4, &p));
    pb.cols = (const uint32_t*)p;
    BMM_TRY(palloc(g, Q * 2, &p));
    pb.target = (uint16_t*)p;
    BMM_TRY(palloc(g, Q * 256 * 2, &p));
    pb.perm = (uint16_t*)p;
    BMM_TRY(palloc(g, Q * 512 * 2, &p));
    pb.X = (__nv_bfloat16*)p;
    BMM_TRY(palloc(g, Q * 256 * 4, &p));
    pb.logits = (float*)p;
    BMM_TRY(palloc(g, Q * 256 * 4, &p));
    pb.T = (float*)p;
    BMM_TRY(palloc(g, Q, &p));
    pb.valid = (uint8_t*)p;
    BMM_TRY(palloc(g, 4 * 8, &p));
    pb.counters = (unsigned long long*)p;
    BMM_TRY(palloc(g, (size_t)kPropBatchCap * 512 * 2, &p));
    pb.Xb = (__nv_bfloat16*)p;
    BMM_TRY(palloc(g, (size_t)kPropBatchCap * 256 * 4, &p));
    pb.Tb = (float*)p;
    BMM_TRY(palloc(g, 4 + (size_t)kPropBatchCap * 4, &p));
    pb.batch_rows = (int*)p;
    // sketch columns: 256 distinct columns drawn from the seed, sorted
    std::vector<uint32_t> colv;
    {
        const uint32_t ncols = g->cols;
        uint64_t s = mix64(seed ^ 0xC0C0ull);
        std::vector<uint32_t> pick;
        if (ncols <= 256) {
            for (uint32_t k = 0; k < 256; ++k)
                pick.push_back(k % ncols);
        } else {
            std::vector<uint8_t> used(ncols, 0);
            while (pick.size() < 256) {
                s = mix64(s);
                const uint32_t c0 = (uint32_t)(s % ncols);
                if (!used[c0]) {
                    used[c0] = 1;
                    pick.push_back(c0);
                }
            }
        }
        std::sort(pick.begin(), pick.end());
        colv = pick;
    }
    BMM_CUDA_TRY(cudaMemcpyAsync((void*)pb.cols, colv.data(), 256 * 4, cudaMemcpyHostToDevice,
                                 g->stream));
    BMM_CUDA_TRY(cudaMemsetAsync(pb.counters, 0, 32, g->stream));
    BMM_CUDA_TRY(cudaMemsetAsync(pb.valid, 0, Q, g->stream));
    BMM_CUDA_TRY(cudaMallocHost((void**)&g->h_counters, 5 * 8));
    BMM_CUDA_TRY(cudaFuncSetAttribute(search_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      32768 * 4));
    if (mode == 1) {
        BMM_TRY(mlp::create(seed ^ 0x5eedull, lr, g->stream, &g->net));
        BMM_TRY(mlp::ensure_cap(g->net, std::max<uint64_t>(Q, kPropBatchCap)));
    }
    return BMM_OK;
}

void propose_free(bmm_ga* g) {
    if (g->net) {
        mlp::destroy(g->net);
        g->net = nullptr;
    }
    if (g->h_counters) {
        cudaFreeHost(g->h_counters);
        g->h_counters = nullptr;
    }
}

int propose_generation(bmm_ga* g) {
    const State& st = g->st;
    const Config& c = st.c;
    PropBuf& pb = g->prop;
    cudaStream_t s = g->stream;
    const uint64_t Q = (uint64_t)g->I * c.E * pb.qpc;
    const unsigned long long gen = g->gen;
    if (Q == 0)
        return BMM_OK;
    features_kernel<<<(unsigned)std::min<uint64_t>(Q, 65535), 256, 0, s>>>(st, pb, gen);
    if (pb.mode == 1)
        BMM_TRY(mlp::forward_dev(g->net, pb.X, 1, (int)Q, pb.logits, false));
    BMM_CUDA_TRY(cudaMemsetAsync(pb.counters, 0, 32, s));
    search_kernel<<<g->search_grid, item::kFwht16Threads, 32768 * 4, s>>>(st, pb, gen,
                                                                          (int)g->cols);
    BMM_CUDA_TRY(cudaGetLastError());
    if (pb.mode == 1) {
        uint32_t* idx = (uint32_t*)(pb.batch_rows + 1);
        compact_kernel<<<1, 1024, 0, s>>>(pb.valid, Q, idx, kPropBatchCap, pb.batch_rows);
        BMM_CUDA_TRY(cudaMemcpyAsync(g->h_counters + 4, pb.batch_rows, 4, cudaMemcpyDeviceToHost, s));
    }
    BMM_CUDA_TRY(cudaMemcpyAsync(g->h_counters, pb.counters, 32, cudaMemcpyDeviceToHost, s));
    BMM_CUDA_TRY(cudaStreamSynchronize(s));
    if (pb.mode == 1) {
        const int fresh = (int)(uint32_t)g->h_counters[4];
        if (fresh > 0) {
            gather_kernel<<<fresh, 256, 0, s>>>(pb, (const uint32_t*)(pb.batch_rows + 1),
                                                g->replay_head);
            g->replay_head = (g->replay_head + fresh) % kPropBatchCap;
            g->replay_fill = std::min(g->replay_fill + fresh, kPropBatchCap);
            g->examples += (unsigned long long)fresh;
        }
        // Adam steps on minibatches: contiguous blocks of the replay buffer at
        // seeded offsets
        const int rows = std::min(g->replay_fill, kPropMinibatch);
        for (int k = 0; k < g->train_steps && rows > 0; ++k) {
            const uint64_t r = mix64(pb.seed ^ mix64(gen * 131 + (uint64_t)k));
            const int start = (int)(r % (uint64_t)(g->replay_fill - rows + 1));
            BMM_TRY(mlp::train_step_dev(g->net, pb.Xb + (size_t)start * 512, 1,
                                        pb.Tb + (size_t)start * 256, rows));
        }
        if (rows > 0) {
            BMM_CUDA_TRY(cudaMemcpyAsync(&g->last_loss, g->net->loss, 4, cudaMemcpyDeviceToHost, s));
            BMM_CUDA_TRY(cudaStreamSynchronize(s));
            int err = 0;
            BMM_CUDA_TRY(cudaMemcpy(&err, g->net->err, 4, cudaMemcpyDeviceToHost));
            if (err)
                return fail(BMM_ETIMEOUT, "ga: a tensor-core wait timed out in the proposal network");
        }
        // learned share: decayed success counts of both window sources;
        // the learned share moves towards the better one
        const unsigned long long* k = g->h_counters;
        if (k[0] > 0 && k[2] > 0) {
            g->paired_rate[0] += (double)k[1] / (double)k[0];
            g->paired_rate[1] += (double)k[3] / (double)k[2];
            ++g->paired_gens;
        }
        for (int src = 0; src < 2; ++src) {
            g->ema_tried[src] = 0.95 * g->ema_tried[src] + (double)k[2 * src];
            g->ema_improved[src] = 0.95 * g->ema_improved[src] + (double)k[2 * src + 1];
        }
        if (g->ema_tried[0] > 0 && g->ema_tried[1] > 0) {
            const double rl = g->ema_improved[0] / g->ema_tried[0];
            const double ru = g->ema_improved[1] / g->ema_tried[1];
            float f = pb.learned_frac + (rl >= ru ? 0.02f : -0.02f);
            pb.learned_frac = std::min(0.95f, std::max(0.05f, f));
        }
    }
    g->tot[0] += g->h_counters[0];
    g->tot[1] += g->h_counters[1];
    g->tot[2] += g->h_counters[2];
    g->tot[3] += g->h_counters[3];
    return BMM_OK;
}

}  // namespace ga
}  // namespace bmm
