// Island-model genetic algorithm on the B200.
//
// Reference behaviour (MortimerDe/bmmpy, src/ga/*): an individual is N
// candidates -- masks over the N window rows with weight = popcount of the
// XOR of the selected rows (genetic_algorithm_internal.hpp:41-103); fitness is
// the sum of weights (genetic_algorithm_core.cpp:10-15).  A generation
// (genetic_algorithm_lifecycle.cpp:112-200): adapt the mutation rate
// (core.cpp:33-41), keep the elites, fill the rest with children made by
// tournament selection (operators.cpp:39-56), greedy GF(2)-basis crossover
// over the parents' candidates sorted by (weight, mask popcount)
// (operators.cpp:58-98, xor_basis.hpp:117-155), pair-XOR mutation with an
// exact re-score (operators.cpp:100-129) and, every third generation,
// pairwise local improvement (operators.cpp:131-192); once the island is more
// than 15 generations without improvement, each new slot is a random
// individual with probability 0.2.  Optional catastrophe (operators.cpp:15-37).
// Islands exchange their best individual every `interval` generations
// (island.cpp:149-228; import rule lifecycle.cpp:83-110), here along a ring.
//
// Exactness.  The reference draws every random number of an island from one
// xorshift64 stream in a fixed order, and every draw count is known before
// the draws are made: a restart check (1 draw, only while stagnating), a
// tournament (parents x tournament_size index draws), a mutation (2 draws per
// pair), a random individual (6N draws).  xorshift64 is linear over GF(2), so
// a schedule kernel walks each island's slots and jumps the stream over a
// child's mutation draws with a precomputed 64 x 64 bit matrix.  Every slot
// then knows its generator state and its parents, and all children of all
// islands are built in parallel while reproducing the reference's sequential
// trajectory bit for bit (same population order, same best individual and
// score every generation).
//
// B200 layout.  All islands live in HBM: two population buffers (current and
// next, selected per island by IslandStat::cur) of masks [I*P][N][4] u64,
// MATERIALISED candidate rows [I*P][N][W] u64, weights [I*P][N] and fitness
// [I*P].  Children are composed as a GF(2) combination T of source rows
// (parent candidate rows or window rows): crossover and mutation only touch
// the 256 x 4-word T and mask matrices in shared memory, then one streaming
// pass writes every child row once (row i = XOR of the sources in T_i) and
// recounts the weights of mutated candidates.  Local improvement builds the
// N x N overlap matrix popc(r_i & r_j) from shared-memory tiles.
#include "common.cuh"
#include "ga.cuh"

#include <algorithm>
#include <cstring>
#include <vector>

namespace bmm {
namespace ga {

constexpr uint64_t kDefaultSeed = 0x9E3779B97F4A7C15ull;  // xorshift64.hpp:8

__host__ __device__ __forceinline__ uint64_t xs_step(uint64_t x) {
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    return x;
}

// detail::XorShift64 (xorshift64.hpp:10-40) from an already reseeded state.
struct Rng {
    uint64_t s;
    __device__ __forceinline__ explicit Rng(uint64_t state) : s(state) {}
    __device__ __forceinline__ uint64_t next() {
        s = xs_step(s);
        return s;
    }
    __device__ __forceinline__ uint32_t index(uint32_t n) {
        return n ? (uint32_t)(next() % (uint64_t)n) : 0u;
    }
    __device__ __forceinline__ double unit() {
        return (double)(next() >> 11) * (1.0 / 9007199254740992.0);
    }
};

// s -> M s for a GF(2) matrix given as 64 columns.
__device__ __forceinline__ uint64_t jump(const uint64_t* __restrict__ J, uint64_t s) {
    uint64_t r = 0;
    while (s) {
        r ^= __ldg(J + (__ffsll((long long)s) - 1));
        s &= s - 1;
    }
    return r;
}

// The generator state after `count` mutation pairs (2 draws each).
__device__ uint64_t jump_pairs(const uint64_t* __restrict__ tab, int N, uint64_t s, uint32_t count) {
    while (count > (uint32_t)N) {
        s = jump(tab + (size_t)N * 64, s);
        count -= (uint32_t)N;
    }
    return jump(tab + (size_t)count * 64, s);
}

// Warp-wide jump with the matrix columns held by the lanes (c0: column lane,
// c1: column lane + 32).  Every lane returns the result.
__device__ __forceinline__ uint64_t warp_jump(uint64_t s, uint64_t c0, uint64_t c1) {
    const int lane = threadIdx.x & 31;
    uint64_t v = (((s >> lane) & 1ull) ? c0 : 0ull) ^ (((s >> (lane + 32)) & 1ull) ? c1 : 0ull);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v ^= __shfl_xor_sync(kFull, v, o);
    return v;
}

__device__ __forceinline__ int first_bit4(const uint64_t* t) {
#pragma unroll
    for (int w = 0; w < 4; ++w)
        if (t[w])
            return w * 64 + __ffsll((long long)t[w]) - 1;
    return -1;
}

__device__ __forceinline__ int highest_bit4(const uint64_t (&v)[4]) {
#pragma unroll
    for (int w = 3; w >= 0; --w)
        if (v[w])
            return w * 64 + 63 - __clzll((long long)v[w]);
    return -1;
}

__device__ __forceinline__ uint4 vxor(uint4 a, uint4 b) {
    return make_uint4(a.x ^ b.x, a.y ^ b.y, a.z ^ b.z, a.w ^ b.w);
}
__device__ __forceinline__ uint2 vxor(uint2 a, uint2 b) { return make_uint2(a.x ^ b.x, a.y ^ b.y); }
__device__ __forceinline__ uint4 vand(uint4 a, uint4 b) {
    return make_uint4(a.x & b.x, a.y & b.y, a.z & b.z, a.w & b.w);
}
__device__ __forceinline__ uint2 vand(uint2 a, uint2 b) { return make_uint2(a.x & b.x, a.y & b.y); }
__device__ __forceinline__ uint32_t vpopc(uint4 a) {
    return __popc(a.x) + __popc(a.y) + __popc(a.z) + __popc(a.w);
}
__device__ __forceinline__ uint32_t vpopc(uint2 a) { return __popc(a.x) + __popc(a.y); }
template <typename V>
__device__ __forceinline__ V vzero();
template <>
__device__ __forceinline__ uint4 vzero<uint4>() {
    return make_uint4(0, 0, 0, 0);
}
template <>
__device__ __forceinline__ uint2 vzero<uint2>() {
    return make_uint2(0, 0);
}

// ---------------------------------------------------------------------------
// Materialisation: dst row i = XOR over j in T_i of src[j] (W words each);
// weight i = popcount if recount[i], else keepw[i].  Warp per 4 rows, lanes
// over 16-byte (W even) or 8-byte elements, every row's first source loaded
// before any reduction so that 8 loads per lane are in flight.
template <typename V>
__device__ void materialize_v(const uint64_t* T, const uint64_t* const* srcp, uint64_t* dst,
                              uint32_t* dw, const uint32_t* keepw, const uint8_t* recount, int N,
                              int W) {
    constexpr int kPer = (int)(sizeof(V) / 8);
    constexpr int kEl = 2;  // elements per lane per row and pass
    const int W2 = W / kPer;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int r0 = warp * 4; r0 < N; r0 += nw * 4) {
        uint32_t pc[4] = {0, 0, 0, 0};
        for (int e0 = 0; e0 < W2; e0 += 32 * kEl) {
            V acc[4][kEl];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int i = r0 + r;
                const V* s = nullptr;
                const int f = i < N ? first_bit4(T + i * 4) : -1;
                if (f >= 0)  // a zero combination materialises a zero row
                    s = reinterpret_cast<const V*>(srcp[f]);
#pragma unroll
                for (int k = 0; k < kEl; ++k) {
                    const int e = e0 + lane + 32 * k;
                    acc[r][k] = (s && e < W2) ? s[e] : vzero<V>();
                }
            }
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int i = r0 + r;
                if (i >= N)
                    continue;
                const int f = first_bit4(T + i * 4);
                for (int q = 0; q < 4 && f >= 0; ++q) {
                    uint64_t m = T[i * 4 + q];
                    if (q == (f >> 6))
                        m &= m - 1;  // drop the first source
                    while (m) {
                        const V* s = reinterpret_cast<const V*>(
                            srcp[q * 64 + __ffsll((long long)m) - 1]);
                        m &= m - 1;
#pragma unroll
                        for (int k = 0; k < kEl; ++k) {
                            const int e = e0 + lane + 32 * k;
                            if (e < W2)
                                acc[r][k] = vxor(acc[r][k], s[e]);
                        }
                    }
                }
                V* d = reinterpret_cast<V*>(dst + (size_t)i * W);
#pragma unroll
                for (int k = 0; k < kEl; ++k) {
                    const int e = e0 + lane + 32 * k;
                    if (e < W2) {
                        d[e] = acc[r][k];
                        pc[r] += vpopc(acc[r][k]);
                    }
                }
            }
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            uint32_t s = pc[r];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
                s += __shfl_xor_sync(kFull, s, o);
            const int i = r0 + r;
            if (lane == 0 && i < N && dw)
                dw[i] = (!recount || recount[i]) ? s : keepw[i];
        }
    }
}

__device__ __forceinline__ void materialize(const uint64_t* T, const uint64_t* const* srcp,
                                            uint64_t* dst, uint32_t* dw, const uint32_t* keepw,
                                            const uint8_t* recount, int N, int W) {
    if ((W & 1) == 0)
        materialize_v<uint4>(T, srcp, dst, dw, keepw, recount, N, W);
    else
        materialize_v<uint2>(T, srcp, dst, dw, keepw, recount, N, W);
}

// `count` pair XORs (i = next_index(N), j = next_index(N), skipped when equal;
// GeneticAlgorithm::mutate and make_random) applied to the combination matrix
// T and the masks M, word q by thread q (q < 4): no barrier between pairs.
// touched[i] = 1 for every modified i (may be null).
__device__ void apply_pairs(uint64_t* T, uint64_t* M, uint8_t* touched, int N, uint32_t count,
                            uint64_t state) {
    const int q = threadIdx.x;
    if (q >= 4)
        return;
    Rng rng(state);
    for (uint32_t m = 0; m < count; ++m) {
        const uint32_t i = rng.index(N);
        const uint32_t j = rng.index(N);
        if (i == j)
            continue;
        T[i * 4 + q] ^= T[j * 4 + q];
        M[i * 4 + q] ^= M[j * 4 + q];
        if (q == 0 && touched)
            touched[i] = 1;
    }
}

// Crossover (operators.cpp:58-98) of np parents of N candidates: the np*N
// candidates stable-sorted by (weight, mask popcount) and inserted greedily
// into a GF(2) basis (PivotBasis, xor_basis.hpp:117-155: a candidate is kept
// when independent of those kept before) until N are independent, then unit vectors pad the
// basis with weight 1 (as the reference does; a full-rank parent makes the
// padding unreachable).  Child candidate n: source row srcp[n] (parent
// candidate row, or window row u for unit u), mask M[n], weight keepw[n].
// pm[p], pw[p], pr[p]: parent p's masks (N x 4), weights, rows (N x W).
struct CrossSmem {
    unsigned long long* key;  // pool2
    uint64_t* pmask;          // pool x 4
    uint64_t* basis;          // N x 4
    uint8_t* used;            // N
};

__device__ void crossover(const uint64_t* const* pm, const uint32_t* const* pw,
                          const uint64_t* const* pr, int np, const uint64_t* base, int N, int W,
                          CrossSmem sm, const uint64_t** srcp, uint64_t* M, uint32_t* keepw) {
    const int tid = threadIdx.x;
    const int pool = np * N;
    int pool2 = 32;
    while (pool2 < pool)
        pool2 <<= 1;
    for (int q = tid; q < pool2; q += blockDim.x) {
        if (q < pool) {
            const int p = q / N, n = q % N;
            const uint64_t* m = pm[p] + n * 4;
            const uint64_t m0 = m[0], m1 = m[1], m2 = m[2], m3 = m[3];
            sm.pmask[q * 4 + 0] = m0;
            sm.pmask[q * 4 + 1] = m1;
            sm.pmask[q * 4 + 2] = m2;
            sm.pmask[q * 4 + 3] = m3;
            const uint32_t pc = __popcll(m0) + __popcll(m1) + __popcll(m2) + __popcll(m3);
            sm.key[q] = ((unsigned long long)pw[p][n] << 20) | ((unsigned long long)pc << 10) |
                        (unsigned long long)q;
        } else {
            sm.key[q] = ~0ull;
        }
    }
    for (int q = tid; q < N; q += blockDim.x)
        sm.used[q] = 0;
    __syncthreads();
    for (int size = 2; size <= pool2; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = tid; t < pool2; t += blockDim.x) {
                const int o = t ^ stride;
                if (o > t) {
                    const unsigned long long a = sm.key[t], b = sm.key[o];
                    if ((a > b) == ((t & size) == 0)) {
                        sm.key[t] = b;
                        sm.key[o] = a;
                    }
                }
            }
            __syncthreads();
        }
    // Greedy insertion, warp 0.  The basis is kept fully reduced (each pivot
    // row is zero in every other pivot column), so a candidate reduces in one
    // step -- XOR of the pivot rows at its set pivot bits -- and lane l owns
    // pivot rows l, l+32, ...  Independence does not depend on the basis
    // representation, so the accepted candidates are PivotBasis's.
    if (tid < 32) {
        const int lane = tid;
        int nchild = 0;
        for (int q = 0; q < pool + N && nchild < N; ++q) {
            uint64_t v[4];
            int id = -1, unit = -1;
            if (q < pool) {
                id = (int)(sm.key[q] & 1023u);
#pragma unroll
                for (int w = 0; w < 4; ++w)
                    v[w] = sm.pmask[id * 4 + w];
            } else {
                unit = q - pool;
                v[0] = v[1] = v[2] = v[3] = 0;
                v[unit >> 6] = 1ull << (unit & 63);
            }
            uint64_t r[4] = {0, 0, 0, 0};
            for (int p = lane; p < N; p += 32)
                if (sm.used[p] && ((v[p >> 6] >> (p & 63)) & 1ull)) {
#pragma unroll
                    for (int w = 0; w < 4; ++w)
                        r[w] ^= sm.basis[p * 4 + w];
                }
#pragma unroll
            for (int w = 0; w < 4; ++w) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1)
                    r[w] ^= __shfl_xor_sync(kFull, r[w], o);
                r[w] ^= v[w];
            }
            const int hb = highest_bit4(r);
            if (hb < 0)
                continue;  // dependent
            for (int p = lane; p < N; p += 32)
                if (sm.used[p] && ((sm.basis[p * 4 + (hb >> 6)] >> (hb & 63)) & 1ull)) {
#pragma unroll
                    for (int w = 0; w < 4; ++w)
                        sm.basis[p * 4 + w] ^= r[w];
                }
            __syncwarp();
            if (lane == 0) {
                sm.used[hb] = 1;
#pragma unroll
                for (int w = 0; w < 4; ++w)
                    sm.basis[hb * 4 + w] = r[w];
                // the child keeps the original candidate, not the reduced vector
                if (id >= 0) {
                    const int p = id / N, n = id % N;
                    srcp[nchild] = pr[p] + (size_t)n * W;
#pragma unroll
                    for (int w = 0; w < 4; ++w)
                        M[nchild * 4 + w] = sm.pmask[id * 4 + w];
                    keepw[nchild] = pw[p][n];
                } else {
                    srcp[nchild] = base + (size_t)unit * W;
#pragma unroll
                    for (int w = 0; w < 4; ++w)
                        M[nchild * 4 + w] = (unit >> 6) == w ? 1ull << (unit & 63) : 0ull;
                    keepw[nchild] = 1;
                }
            }
            __syncwarp();
            ++nchild;
        }
    }
    __syncthreads();
}

// make_heuristic's probe loop (genetic_algorithm_population.cpp:42-83) on an
// identity individual already materialised in global memory: for the 5
// heaviest rows (stable descending order), the first other row whose XOR
// lowers the weight is applied.
__device__ void heuristic_probe(uint64_t* masks, uint64_t* rows, uint32_t* wts, int N, int W,
                                uint32_t* red) {
    const int tid = threadIdx.x;
    __shared__ int s_order[5];
    __shared__ uint32_t s_cw;
    if (N < 2)
        return;
    __syncthreads();
    if (tid == 0) {
        uint8_t taken[kMaxN];
        for (int r = 0; r < N; ++r)
            taken[r] = 0;
        for (int p = 0; p < 5 && p < N; ++p) {
            int bi = -1;
            for (int r = 0; r < N; ++r)
                if (!taken[r] && (bi < 0 || wts[r] > wts[bi]))
                    bi = r;
            taken[bi] = 1;
            s_order[p] = bi;
        }
    }
    __syncthreads();
    const int probes = N < 5 ? N : 5;
    const int nw = blockDim.x >> 5;
    for (int p = 0; p < probes; ++p) {
        const int i = s_order[p];
        const uint32_t cur = wts[i];
        for (int j = 0; j < N; ++j) {
            if (j == i)
                continue;
            uint32_t part = 0;
            for (int w = tid; w < W; w += blockDim.x)
                part += __popcll(rows[(size_t)i * W + w] ^ rows[(size_t)j * W + w]);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
                part += __shfl_xor_sync(kFull, part, o);
            if ((tid & 31) == 0)
                red[tid >> 5] = part;
            __syncthreads();
            if (tid == 0) {
                uint32_t t = 0;
                for (int q = 0; q < nw; ++q)
                    t += red[q];
                s_cw = t;
            }
            __syncthreads();
            const uint32_t cw = s_cw;
            if (cw < cur) {
                for (int w = tid; w < W; w += blockDim.x)
                    rows[(size_t)i * W + w] ^= rows[(size_t)j * W + w];
                if (tid < 4)
                    masks[i * 4 + tid] ^= masks[j * 4 + tid];
                if (tid == 0)
                    wts[i] = cw;
                __syncthreads();
                break;
            }
            __syncthreads();
        }
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Build: one CTA per (island, slot) of the next population.
constexpr int kBuildThreads = 256;

struct BuildSmem {
    uint64_t* T;         // N x 4 (aliases the crossover basis)
    uint64_t* M;         // N x 4
    const uint64_t** srcp;  // N
    uint32_t* keepw;     // N
    uint8_t* recount;    // N
    CrossSmem cross;
};

__host__ __device__ inline int pool2_for(int np, int N) {
    int p2 = 32;
    while (p2 < np * N)
        p2 <<= 1;
    return p2;
}

__host__ __device__ inline size_t build_smem_bytes(int N, int np) {
    const int pool = np * N, p2 = pool2_for(np, N);
    return (size_t)N * 32 * 2 + (size_t)N * 8 + (size_t)N * 4 + (size_t)p2 * 8 +
           (size_t)pool * 32 + (size_t)N * 2 + 64;
}

__device__ BuildSmem carve_build(unsigned char* smem, int N, int np) {
    BuildSmem s;
    const int pool = np * N, p2 = pool2_for(np, N);
    unsigned char* p = smem;
    s.T = reinterpret_cast<uint64_t*>(p);
    p += (size_t)N * 32;
    s.M = reinterpret_cast<uint64_t*>(p);
    p += (size_t)N * 32;
    s.srcp = reinterpret_cast<const uint64_t**>(p);
    p += (size_t)N * 8;
    s.cross.key = reinterpret_cast<unsigned long long*>(p);
    p += (size_t)p2 * 8;
    s.cross.pmask = reinterpret_cast<uint64_t*>(p);
    p += (size_t)pool * 32;
    s.keepw = reinterpret_cast<uint32_t*>(p);
    p += (size_t)N * 4;
    s.recount = p;
    p += N;
    s.cross.used = p;
    s.cross.basis = s.T;
    return s;
}

// Identity combination over N sources, unit masks.
__device__ void set_identity(BuildSmem& s, int N, bool unit_masks) {
    for (int e = threadIdx.x; e < N * 4; e += blockDim.x) {
        const int r = e >> 2, w = e & 3;
        const uint64_t u = (r >> 6) == w ? (1ull << (r & 63)) : 0ull;
        s.T[e] = u;
        if (unit_masks)
            s.M[e] = u;
    }
}

// mode 0: generation (and initial population) slots of stepped islands;
// mode 1: catastrophe slots of islands with cat_now.
__global__ void __launch_bounds__(kBuildThreads, 4) build_kernel(State st, int mode) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint32_t red[kBuildThreads / 32];
    const Config& c = st.c;
    const int N = c.N, W = c.W, P = c.P;
    BuildSmem s = carve_build(smem, N, c.parents);
    const int tid = threadIdx.x;
    for (uint32_t cs = blockIdx.x; cs < (uint32_t)(st.I * P); cs += gridDim.x) {
        const uint32_t island = cs / P;
        const IslandStat& is = st.stat[island];
        if (!is.stepped || (mode == 1 && !is.cat_now))
            continue;
        const Sched rec = st.sched[cs];
        const int cur = (int)is.cur;
        const Pop src = st.pop[cur], dst = st.pop[cur ^ 1];
        uint64_t* dm = dst.masks + (size_t)cs * N * 4;
        uint64_t* dr = dst.rows + (size_t)cs * N * W;
        uint32_t* dwt = dst.wts + (size_t)cs * N;
        const size_t ibase = (size_t)island * P;
        if (rec.kind == kCopy) {
            const size_t si = ibase + rec.par[0];
            set_identity(s, N, false);
            for (int n = tid; n < N; n += blockDim.x) {
                s.srcp[n] = src.rows + (si * N + n) * W;
                s.keepw[n] = src.wts[si * N + n];
                s.recount[n] = 0;
            }
            for (int e = tid; e < N * 4; e += blockDim.x)
                s.M[e] = src.masks[si * N * 4 + e];
            __syncthreads();
            materialize(s.T, s.srcp, dr, dwt, s.keepw, s.recount, N, W);
        } else if (rec.kind == kChild) {
            const uint64_t* pm[4];
            const uint32_t* pw[4];
            const uint64_t* pr[4];
            for (int p = 0; p < (int)rec.np; ++p) {
                const size_t pi = ibase + rec.par[p];
                pm[p] = src.masks + pi * N * 4;
                pw[p] = src.wts + pi * N;
                pr[p] = src.rows + pi * N * W;
            }
            crossover(pm, pw, pr, (int)rec.np, st.base, N, W, s.cross, s.srcp, s.M, s.keepw);
            set_identity(s, N, false);
            for (int n = tid; n < N; n += blockDim.x)
                s.recount[n] = 0;
            __syncthreads();
            if (N >= 2)
                apply_pairs(s.T, s.M, s.recount, N, is.count, rec.rng);
            __syncthreads();
            materialize(s.T, s.srcp, dr, dwt, s.keepw, s.recount, N, W);
        } else {  // kRandom, kIdentity, kHeuristic: combinations of window rows
            set_identity(s, N, true);
            for (int n = tid; n < N; n += blockDim.x)
                s.srcp[n] = st.base + (size_t)n * W;
            __syncthreads();
            if (rec.kind == kRandom)
                apply_pairs(s.T, s.M, nullptr, N, 3u * (uint32_t)N, rec.rng);
            __syncthreads();
            materialize(s.T, s.srcp, dr, dwt, nullptr, nullptr, N, W);
        }
        for (int e = tid; e < N * 4; e += blockDim.x)
            dm[e] = s.M[e];
        __syncthreads();
        if (rec.kind == kHeuristic)
            heuristic_probe(dm, dr, dwt, N, W, red);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Schedule: one warp per island.  Adapts the mutation rate, then walks the
// next population's slots in the reference's order, consuming the island's
// generator exactly as GeneticAlgorithm::step would.
__global__ void schedule_kernel(State st) {
    const int island = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (island >= st.I)
        return;
    const Config& c = st.c;
    const int N = c.N, P = c.P;
    IslandStat& is = st.stat[island];
    const uint32_t stepped = is.done ? 0u : 1u;
    __syncwarp();
    if (lane == 0) {
        is.stepped = stepped;
        is.cat_now = 0;
        is.migrated = 0;
    }
    if (!stepped)
        return;
    // adapt_mutation_rate (genetic_algorithm_core.cpp:33-41)
    double rate = is.rate;
    if (is.no_improvement > 10)
        rate = fmin(0.8, rate * 1.5);
    else if (is.no_improvement > 5)
        rate = fmin(0.6, rate * 1.3);
    else
        rate = fmax(0.3, rate * 0.95);
    const double prod = (double)N * rate;
    uint32_t count = prod >= 4294967295.0 ? 0xffffffffu : (uint32_t)prod;
    count = count < 1u ? 1u : count;
    const uint32_t pairs = N >= 2 ? count : 0u;
    // this generation's mutation jump and the make_random jump, column-wise
    const uint64_t m0 = jump_pairs(st.jump_mut, N, 1ull << lane, pairs);
    const uint64_t m1 = jump_pairs(st.jump_mut, N, 1ull << (lane + 32), pairs);
    const uint64_t r0 = __ldg(st.jump_rand + lane), r1 = __ldg(st.jump_rand + lane + 32);
    Rng rng(is.rng);
    const unsigned long long* fit = st.pop[is.cur].fit + (size_t)island * P;
    Sched* sc = st.sched + (size_t)island * P;
    const uint32_t* ord = st.order + (size_t)island * P;
    const int E = c.E < P ? c.E : P;
    for (int e = lane; e < E; e += 32) {
        Sched r;
        r.rng = 0;
        r.kind = kCopy;
        r.np = 1;
        r.par[0] = (uint16_t)ord[e];
        r.par[1] = r.par[2] = r.par[3] = 0;
        sc[e] = r;
    }
    const bool may_restart = is.no_improvement > 15;
    int slot = E;
    while (slot < P) {
        if (may_restart && rng.unit() < 0.2) {
            if (lane == 0) {
                Sched r;
                r.rng = rng.s;
                r.kind = kRandom;
                r.np = 0;
                r.par[0] = r.par[1] = r.par[2] = r.par[3] = 0;
                sc[slot] = r;
            }
            rng.s = warp_jump(rng.s, r0, r1);
            ++slot;
            continue;
        }
        Sched r;
        r.kind = kChild;
        r.np = (uint32_t)c.parents;
        r.par[0] = r.par[1] = r.par[2] = r.par[3] = 0;
        for (int p = 0; p < c.parents; ++p) {  // tournament_selection
            uint32_t best = rng.index(P);
            for (int t = 1; t < c.T; ++t) {
                const uint32_t cand = rng.index(P);
                if (fit[cand] < fit[best])
                    best = cand;
            }
            r.par[p] = (uint16_t)best;
        }
        for (int o = 0; o < c.offspring && slot < P; ++o) {
            r.rng = rng.s;
            if (lane == 0)
                sc[slot] = r;
            if (pairs)
                rng.s = warp_jump(rng.s, m0, m1);
            ++slot;
        }
    }
    if (lane == 0) {
        is.rng = rng.s;
        is.rate = rate;
        is.count = pairs;
    }
}

// ---------------------------------------------------------------------------
// which: 0 = current population of every island (initialisation),
//        1 = next population of stepped islands,
//        2 = next population of islands with a catastrophe this generation.
__global__ void fitness_kernel(State st, int which) {
    const int lane = threadIdx.x & 31;
    const uint32_t ind = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int N = st.c.N, P = st.c.P;
    if (ind >= (uint32_t)(st.I * P))
        return;
    const IslandStat& is = st.stat[ind / P];
    if (which == 1 && !is.stepped)
        return;
    if (which == 2 && !(is.stepped && is.cat_now))
        return;
    const Pop p = st.pop[which == 0 ? is.cur : is.cur ^ 1];
    unsigned long long s = 0;
    for (int r = lane; r < N; r += 32)
        s += p.wts[(size_t)ind * N + r];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        s += __shfl_xor_sync(kFull, s, o);
    if (lane == 0)
        p.fit[ind] = s;
}

// ---------------------------------------------------------------------------
enum RankMode : int { kRankInit = 0, kRankStep = 1, kRankCat = 2, kRankMigrate = 3 };

__device__ bool should_stop(const IslandCfg& c, const IslandStat& is) {
    if ((c.flags & 1u) && is.generations >= c.max_gen)
        return true;
    if ((c.flags & 2u) && is.stale >= c.max_stale)
        return true;
    if ((c.flags & 4u) && is.best <= c.target)
        return true;
    return false;
}

// One CTA per island, blockDim = power of two >= P.  Flips to the population
// just built where the mode says so, sorts (fitness, position) ascending into
// `order`, and applies the reference's bookkeeping:
//  kRankInit    initialize(): best, counters, evaluations = P;
//  kRankStep    end of step(): generations, evaluations, best / stale /
//               no_improvement / catastrophe counters; schedules a
//               catastrophe when its counter reaches the threshold;
//  kRankCat     end of catastrophe(): adopt a better best, counters kept;
//  kRankMigrate after import_migrants(): the migrant becomes the best and
//               the counters reset.
// `finish`: evaluate should_stop() at the end.
__global__ void __launch_bounds__(1024) rank_kernel(State st, int mode, int finish) {
    __shared__ unsigned long long key[1024];
    __shared__ uint32_t idx[1024];
    __shared__ int s_run, s_copy;
    const Config& c = st.c;
    const int island = blockIdx.x, t = threadIdx.x, P = c.P, n2 = blockDim.x;
    IslandStat& is = st.stat[island];
    if (t == 0) {
        int run;
        if (mode == kRankInit)
            run = 1;
        else if (mode == kRankStep)
            run = is.stepped;
        else if (mode == kRankCat)
            run = is.stepped && is.cat_now;
        else
            run = is.stepped && is.migrated;
        s_run = run;
        if (run && (mode == kRankInit || mode == kRankStep || mode == kRankCat))
            is.cur ^= 1u;
    }
    __syncthreads();
    if (!s_run) {
        if (finish && t == 0 && is.stepped)
            is.done = should_stop(st.icfg[island], is) ? 1u : 0u;
        return;
    }
    const unsigned long long* fit = st.pop[is.cur].fit + (size_t)island * P;
    key[t] = t < P ? fit[t] : ~0ull;
    idx[t] = t;
    __syncthreads();
    for (int size = 2; size <= n2; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            const int o = t ^ stride;
            if (o > t) {
                const bool up = (t & size) == 0;
                const bool gt = key[t] > key[o] || (key[t] == key[o] && idx[t] > idx[o]);
                if (gt == up) {
                    const unsigned long long k0 = key[t];
                    key[t] = key[o];
                    key[o] = k0;
                    const uint32_t i0 = idx[t];
                    idx[t] = idx[o];
                    idx[o] = i0;
                }
            }
            __syncthreads();
        }
    if (t < P)
        st.order[(size_t)island * P + t] = idx[t];
    if (t == 0) {
        const unsigned long long b = key[0];
        int copy = 0;
        if (mode == kRankInit) {
            is.best = b;
            is.generations = 0;
            is.evaluations = (unsigned long long)P;
            is.stale = 0;
            is.no_improvement = 0;
            is.catastrophe = 0;
            copy = 1;
        } else if (mode == kRankStep) {
            is.evaluations += (unsigned long long)P;
            is.generations += 1;
            if (b < is.best) {
                is.best = b;
                is.stale = 0;
                is.no_improvement = 0;
                is.catastrophe = 0;
                copy = 1;
            } else {
                is.stale += 1;
                is.no_improvement += 1;
                is.catastrophe += 1;
            }
            if (c.cat_enable && is.catastrophe == (uint32_t)c.cat_threshold) {
                // catastrophe(): ranked survivors, then make_random for the rest
                is.cat_now = 1;
                is.catastrophe = 0;
                Sched* sc = st.sched + (size_t)island * P;
                const int sv = c.cat_survivors < P ? c.cat_survivors : P;
                uint64_t rs = is.rng;
                for (int q = 0; q < P; ++q) {
                    Sched r;
                    r.np = 1;
                    r.par[0] = r.par[1] = r.par[2] = r.par[3] = 0;
                    if (q < sv) {
                        r.kind = kCopy;
                        r.rng = 0;
                        r.par[0] = (uint16_t)idx[q];
                    } else {
                        r.kind = kRandom;
                        r.rng = rs;
                        rs = jump(st.jump_rand, rs);
                    }
                    sc[q] = r;
                }
                is.rng = rs;
            }
        } else if (mode == kRankCat) {
            if (b < is.best) {
                is.best = b;
                copy = 1;
            }
        } else {  // kRankMigrate: the imported migrant is the unique minimum
            is.best = b;
            is.stale = 0;
            is.no_improvement = 0;
            is.catastrophe = 0;
            copy = 1;
        }
        s_copy = copy;
    }
    __syncthreads();
    if (s_copy) {  // keep a copy of the island's best individual
        const size_t ind = (size_t)island * P + idx[0];
        const int N = c.N, W = c.W;
        const Pop p = st.pop[is.cur];
        for (int i = t; i < N * 4; i += n2)
            st.best_masks[(size_t)island * N * 4 + i] = p.masks[ind * N * 4 + i];
        for (int i = t; i < N; i += n2)
            st.best_wts[(size_t)island * N + i] = p.wts[ind * N + i];
        const uint4* s4 = reinterpret_cast<const uint4*>(p.rows + ind * N * W);
        uint64_t* d = st.best_rows + (size_t)island * N * W;
        if ((W & 1) == 0) {
            uint4* d4 = reinterpret_cast<uint4*>(d);
            for (size_t i = t; i < (size_t)N * W / 2; i += n2)
                d4[i] = s4[i];
        } else {
            for (size_t i = t; i < (size_t)N * W; i += n2)
                d[i] = p.rows[ind * N * W + i];
        }
    }
    if (finish && t == 0)
        is.done = should_stop(st.icfg[island], is) ? 1u : 0u;
}

// ---------------------------------------------------------------------------
// Ring migration: island i imports the best individual of island i - 1 when
// both ran this generation, the source's interval divides its generation
// count (island.cpp:163-168) and the destination imports at all.
// import_migrants: the migrant is taken only when it beats the island's best;
// it replaces the first individual of maximal fitness.  The bookkeeping
// follows in rank_kernel(kRankMigrate).
__global__ void migrate_kernel(State st) {
    const int I = st.I, dst = blockIdx.x, src = (dst + I - 1) % I;
    const Config& c = st.c;
    const int N = c.N, W = c.W, P = c.P;
    __shared__ unsigned long long s_key[32];
    __shared__ int s_ok;
    IslandStat& ds = st.stat[dst];
    const IslandStat& ss = st.stat[src];
    const uint32_t iv = st.icfg[src].interval;
    if (I < 2 || !ds.stepped || !ss.stepped || iv == 0 || ss.generations % iv != 0 ||
        st.icfg[dst].import_count == 0 || !(ss.best < ds.best))
        return;
    const Pop p = st.pop[ds.cur];
    const unsigned long long* fit = p.fit + (size_t)dst * P;
    // first maximum: max over (fit, P - 1 - position)
    unsigned long long best = 0;
    int bi = -1;
    for (int q = threadIdx.x; q < P; q += blockDim.x)
        if (bi < 0 || fit[q] > fit[bi])
            bi = q;
    if (bi >= 0)
        best = fit[bi];
    // pack: fitness in the high bits would overflow; reduce (value, index) pairs
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long ov = __shfl_xor_sync(kFull, best, o);
        const int oi = __shfl_xor_sync(kFull, bi, o);
        if (oi >= 0 && (bi < 0 || ov > best || (ov == best && oi < bi))) {
            best = ov;
            bi = oi;
        }
    }
    __shared__ int s_idx[32];
    if (lane == 0) {
        s_key[warp] = best;
        s_idx[warp] = bi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long bv = 0;
        int bidx = -1;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            const int oi = s_idx[w];
            if (oi >= 0 && (bidx < 0 || s_key[w] > bv || (s_key[w] == bv && oi < bidx))) {
                bv = s_key[w];
                bidx = oi;
            }
        }
        s_ok = bidx;
    }
    __syncthreads();
    const int worst = s_ok;
    if (worst < 0)
        return;
    const size_t d = (size_t)dst * P + worst;
    for (int i = threadIdx.x; i < N * 4; i += blockDim.x)
        p.masks[d * N * 4 + i] = st.best_masks[(size_t)src * N * 4 + i];
    for (int i = threadIdx.x; i < N; i += blockDim.x)
        p.wts[d * N + i] = st.best_wts[(size_t)src * N + i];
    for (size_t i = threadIdx.x; i < (size_t)N * W; i += blockDim.x)
        p.rows[d * N * W + i] = st.best_rows[(size_t)src * N * W + i];
    if (threadIdx.x == 0) {
        p.fit[d] = ss.best;
        ds.migrated = 1;
    }
}

// ---------------------------------------------------------------------------
// Local improvement (operators.cpp:131-192) of one individual: rows R (N x W,
// global), masks M, weights Wt.  G: N x N u32 scratch (global, L2 resident).
// The overlap matrix G[i][j] = popc(r_i & r_j) is built from 32-row tiles of
// up to 128 words staged in shared memory (A, B: 32 x 129 words each); then
// up to 10 greedy passes: for each i with w_i > 0 the first j minimising
// w_i + w_j - 2 G_ij among w_j < 2 w_i is applied when it beats w_i, and row i
// of G is recomputed.
constexpr int kLiTile = 32;
constexpr int kLiChunk = 128;
constexpr int kLocalThreads = 512;

__device__ void local_improve(uint64_t* R, uint64_t* M, uint32_t* Wt, int N, int W, uint32_t* G,
                              uint64_t* A, uint64_t* B, uint32_t* w,
                              unsigned long long* s_best /* 2 x 32 */, int* s_flag) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    constexpr int WS = kLiChunk + 1;
    const int ntile = (N + kLiTile - 1) / kLiTile;
    const int per = (kLiTile * kLiTile) / blockDim.x;  // products per thread (2 at 512)
    for (int ti = 0; ti < ntile; ++ti)
        for (int tj = ti; tj < ntile; ++tj) {
            uint32_t acc[4] = {0, 0, 0, 0};
            for (int w0 = 0; w0 < W; w0 += kLiChunk) {
                const int wc = min(kLiChunk, W - w0);
                __syncthreads();
                for (int e = tid; e < kLiTile * wc; e += blockDim.x) {
                    const int r = e / wc, q = e % wc;
                    const int ra = ti * kLiTile + r, rb = tj * kLiTile + r;
                    A[r * WS + q] = ra < N ? R[(size_t)ra * W + w0 + q] : 0ull;
                    B[r * WS + q] = rb < N ? R[(size_t)rb * W + w0 + q] : 0ull;
                }
                __syncthreads();
                const int i = tid / (kLiTile / per), j0 = (tid % (kLiTile / per)) * per;
                const uint64_t* a = A + i * WS;
                for (int q = 0; q < wc; ++q) {
                    const uint64_t av = a[q];
                    for (int u = 0; u < per; ++u)
                        acc[u] += __popcll(av & B[(j0 + u) * WS + q]);
                }
            }
            const int i = tid / (kLiTile / per), j0 = (tid % (kLiTile / per)) * per;
            const int gi = ti * kLiTile + i;
            for (int u = 0; u < per; ++u) {
                const int gj = tj * kLiTile + j0 + u;
                if (gi < N && gj < N) {
                    G[gi * N + gj] = acc[u];
                    G[gj * N + gi] = acc[u];
                }
            }
        }
    __syncthreads();
    // the reference re-materialises and recounts every weight first
    for (int i = tid; i < N; i += blockDim.x)
        w[i] = G[i * N + i];
    __syncthreads();
    int parity = 0;
    for (int iter = 0; iter < 10; ++iter) {
        if (tid == 0)
            *s_flag = 0;
        __syncthreads();
        for (int i = 0; i < N; ++i) {
            const uint32_t wi = w[i];
            if (wi == 0)
                continue;
            unsigned long long best = ~0ull;
            for (int j = tid; j < N; j += blockDim.x) {
                if (j == i)
                    continue;
                const uint32_t wj = w[j];
                if ((unsigned long long)wj >= 2ull * wi)
                    continue;
                const uint32_t cw = wi + wj - 2u * G[i * N + j];
                if (cw < wi) {
                    const unsigned long long k = ((unsigned long long)cw << 32) | (uint32_t)j;
                    best = k < best ? k : best;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const unsigned long long ot = __shfl_xor_sync(kFull, best, o);
                best = ot < best ? ot : best;
            }
            unsigned long long* sb = s_best + parity * 32;
            parity ^= 1;
            if (lane == 0)
                sb[warp] = best;
            __syncthreads();
            best = ~0ull;
            for (int q = 0; q < nw; ++q)
                best = sb[q] < best ? sb[q] : best;
            if (best == ~0ull)
                continue;
            const int j = (int)(best & 0xffffffffu);
            for (int q = tid; q < W; q += blockDim.x)
                R[(size_t)i * W + q] ^= R[(size_t)j * W + q];
            if (tid < 4)
                M[i * 4 + tid] ^= M[j * 4 + tid];
            __syncthreads();
            if (tid == 0) {
                w[i] = (uint32_t)(best >> 32);
                *s_flag = 1;
            }
            for (int k = warp; k < N; k += nw) {
                uint32_t sacc = 0;
                for (int q = lane; q < W; q += 32)
                    sacc += __popcll(R[(size_t)i * W + q] & R[(size_t)k * W + q]);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1)
                    sacc += __shfl_xor_sync(kFull, sacc, o);
                if (lane == 0) {
                    G[i * N + k] = sacc;
                    G[k * N + i] = sacc;
                }
            }
            __syncthreads();
        }
        __syncthreads();
        const int improved = *s_flag;
        __syncthreads();
        if (!improved)
            break;
    }
    for (int i = tid; i < N; i += blockDim.x)
        Wt[i] = w[i];
    __syncthreads();
}

__host__ __device__ inline size_t local_smem_bytes() {
    return (size_t)2 * kLiTile * (kLiChunk + 1) * 8;
}

// Local improvement with the overlap matrix in shared memory (u16: rows of at
// most 1023 words, so every overlap fits).  Same moves as local_improve.  The
// warps scan consecutive rows i at once (nothing changes before a move, so
// every scan is the one the sequential pass would make) and the smallest
// improving i wins; the whole CTA then applies the move and recomputes row and
// column i of G (four rows per warp, eight 16-byte or 8-byte loads in flight
// per lane; the moved row itself from shared memory).  s_move: 4 ints then 32
// u64 of scratch.
constexpr int kLi16Chunk = 64;
constexpr int kLi16MaxW = 1023;  // 64 * 1023 < 65536: overlaps fit in u16

// G (u16) rounded up to 16 bytes so that the 64-bit tiles after it are aligned.
__host__ __device__ inline size_t local16_g_bytes(int N) {
    return ((size_t)N * N * 2 + 15) & ~(size_t)15;
}

__host__ __device__ inline size_t local16_smem_bytes(int N) {
    return local16_g_bytes(N) + (size_t)2 * kLiTile * (kLi16Chunk + 1) * 8;
}

template <typename V>
__device__ void overlap_row(const uint64_t* R, const uint64_t* rnew, int N, int W, int i,
                            uint16_t* G) {
    constexpr int kPer = (int)(sizeof(V) / 8);
    const int W2 = W / kPer;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const V* ri = reinterpret_cast<const V*>(rnew);  // row i after the move (shared)
    for (int k0 = warp * 4; k0 < N; k0 += nw * 4) {
        uint32_t pc[4] = {0, 0, 0, 0};
        for (int e0 = 0; e0 < W2; e0 += 64) {
            V a[2], b[4][2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int e = e0 + lane + 32 * u;
                a[u] = e < W2 ? ri[e] : vzero<V>();
            }
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int k = k0 + r;
                const V* rk = k == i ? ri
                                     : reinterpret_cast<const V*>(R + (size_t)(k < N ? k : 0) * W);
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int e = e0 + lane + 32 * u;
                    b[r][u] = (k < N && e < W2) ? rk[e] : vzero<V>();
                }
            }
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int u = 0; u < 2; ++u)
                    pc[r] += vpopc(vand(a[u], b[r][u]));
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            uint32_t t = pc[r];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
                t += __shfl_xor_sync(kFull, t, o);
            const int k = k0 + r;
            if (lane == 0 && k < N) {
                G[i * N + k] = (uint16_t)t;
                G[k * N + i] = (uint16_t)t;
            }
        }
    }
}

__device__ void local_improve16(uint64_t* R, uint64_t* M, uint32_t* Wt, int N, int W,
                                unsigned char* smem, uint32_t* w, int* s_move) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint16_t* G = reinterpret_cast<uint16_t*>(smem);
    uint64_t* A = reinterpret_cast<uint64_t*>(smem + local16_g_bytes(N));
    uint64_t* B = A + kLiTile * (kLi16Chunk + 1);
    constexpr int WS = kLi16Chunk + 1;
    const int ntile = (N + kLiTile - 1) / kLiTile;
    const int per = (kLiTile * kLiTile) / blockDim.x;
    const int ti_div = kLiTile / per;
    for (int ti = 0; ti < ntile; ++ti)
        for (int tj = ti; tj < ntile; ++tj) {
            uint32_t acc[4] = {0, 0, 0, 0};
            for (int w0 = 0; w0 < W; w0 += kLi16Chunk) {
                const int wc = min(kLi16Chunk, W - w0);
                __syncthreads();
                for (int e = tid; e < kLiTile * wc; e += blockDim.x) {
                    const int r = e / wc, q = e % wc;
                    const int ra = ti * kLiTile + r, rb = tj * kLiTile + r;
                    A[r * WS + q] = ra < N ? R[(size_t)ra * W + w0 + q] : 0ull;
                    B[r * WS + q] = rb < N ? R[(size_t)rb * W + w0 + q] : 0ull;
                }
                __syncthreads();
                const int i = tid / ti_div, j0 = (tid % ti_div) * per;
                const uint64_t* a = A + i * WS;
                for (int q = 0; q < wc; ++q) {
                    const uint64_t av = a[q];
                    for (int u = 0; u < per; ++u)
                        acc[u] += __popcll(av & B[(j0 + u) * WS + q]);
                }
            }
            const int i = tid / ti_div, j0 = (tid % ti_div) * per;
            const int gi = ti * kLiTile + i;
            for (int u = 0; u < per; ++u) {
                const int gj = tj * kLiTile + j0 + u;
                if (gi < N && gj < N) {
                    G[gi * N + gj] = (uint16_t)acc[u];
                    G[gj * N + gi] = (uint16_t)acc[u];
                }
            }
        }
    __syncthreads();
    for (int i = tid; i < N; i += blockDim.x)
        w[i] = G[i * N + i];  // re-materialised weights
    __syncthreads();
    // After the overlap matrix is built the tiles are free: the moved row is
    // staged there (W words; rows wider than the tile area use global memory).
    uint64_t* rnew = A;
    const bool rnew_shared = (size_t)W * 8 <= (size_t)2 * kLiTile * (kLi16Chunk + 1) * 8;
    const int nw = blockDim.x >> 5;
    unsigned long long* s_found = reinterpret_cast<unsigned long long*>(s_move + 4);
    for (int iter = 0; iter < 10; ++iter) {
        int improved = 0;
        int start = 0;
        for (;;) {
            // warps scan rows start + warp, start + nw + warp, ... in rounds;
            // the first round with an improving row decides (its smallest i)
            int fi = -1;
            unsigned long long fk = 0;
            for (int base = start; base < N; base += nw) {
                const int i = base + warp;
                unsigned long long best = ~0ull;
                const uint32_t wi = i < N ? w[i] : 0u;
                if (wi != 0) {
                    for (int j = lane; j < N; j += 32) {
                        const uint32_t wj = w[j];
                        if (j == i || (unsigned long long)wj >= 2ull * wi)
                            continue;
                        const uint32_t cw = wi + wj - 2u * (uint32_t)G[i * N + j];
                        if (cw < wi) {
                            const unsigned long long k = ((unsigned long long)cw << 32) | (uint32_t)j;
                            best = k < best ? k : best;
                        }
                    }
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        const unsigned long long ot = __shfl_xor_sync(kFull, best, o);
                        best = ot < best ? ot : best;
                    }
                }
                if (lane == 0)
                    s_found[warp] = best;
                __syncthreads();
                for (int q = 0; q < nw; ++q)
                    if (s_found[q] != ~0ull) {
                        fi = base + q;
                        fk = s_found[q];
                        break;
                    }
                __syncthreads();
                if (fi >= 0)
                    break;
            }
            if (fi < 0)
                break;
            const int i = fi, j = (int)(fk & 0xffffffffu);
            const uint32_t cw = (uint32_t)(fk >> 32);
            uint64_t* rn = rnew_shared ? rnew : R + (size_t)i * W;
            for (int q = tid; q < W; q += blockDim.x) {
                const uint64_t v = R[(size_t)i * W + q] ^ R[(size_t)j * W + q];
                rn[q] = v;
                if (rnew_shared)
                    R[(size_t)i * W + q] = v;
            }
            if (tid < 4)
                M[i * 4 + tid] ^= M[j * 4 + tid];
            __syncthreads();
            if ((W & 1) == 0)
                overlap_row<uint4>(R, rn, N, W, i, G);
            else
                overlap_row<uint2>(R, rn, N, W, i, G);
            if (tid == 0)
                w[i] = cw;
            __syncthreads();
            improved = 1;
            start = i + 1;
        }
        if (!improved)
            break;
    }
    for (int i = tid; i < N; i += blockDim.x)
        Wt[i] = w[i];
    __syncthreads();
}

// Children (slot kind kChild) of stepped islands, next population.
template <bool kSmemG>
__global__ void __launch_bounds__(kLocalThreads) local_kernel(State st) {
    extern __shared__ __align__(16) unsigned char lsmem[];
    __shared__ uint32_t w[kMaxN];
    __shared__ unsigned long long s_best[64];
    __shared__ __align__(8) int s_flag[4 + 2 * 32];
    const Config& c = st.c;
    const int N = c.N, W = c.W, P = c.P;
    uint32_t* G = st.Gs + (size_t)blockIdx.x * N * N;
    uint64_t* tiles = reinterpret_cast<uint64_t*>(lsmem);
    for (uint32_t cs = blockIdx.x; cs < (uint32_t)(st.I * P); cs += gridDim.x) {
        const IslandStat& is = st.stat[cs / P];
        if (!is.stepped || st.sched[cs].kind != kChild)
            continue;
        const Pop p = st.pop[is.cur ^ 1];
        if (kSmemG)
            local_improve16(p.rows + (size_t)cs * N * W, p.masks + (size_t)cs * N * 4,
                            p.wts + (size_t)cs * N, N, W, lsmem, w, s_flag);
        else
            local_improve(p.rows + (size_t)cs * N * W, p.masks + (size_t)cs * N * 4,
                          p.wts + (size_t)cs * N, N, W, G, tiles,
                          tiles + kLiTile * (kLiChunk + 1), w, s_best, &s_flag[0]);
    }
}

// ---------------------------------------------------------------------------
// Operator kernels for one individual (parity tests of the building blocks).

// Candidate weights: warp per candidate, mask (4 words) over window rows.
__global__ void eval_kernel(const uint64_t* __restrict__ base, int N, int W,
                            const uint64_t* __restrict__ masks, size_t count,
                            uint32_t* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const size_t c = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (c >= count)
        return;
    const uint64_t* m = masks + c * 4;
    uint32_t s = 0;
    for (int w = lane; w < W; w += 32) {
        uint64_t acc = 0;
        for (int q = 0; q < 4; ++q) {
            uint64_t b = m[q];
            while (b) {
                const int r = q * 64 + __ffsll((long long)b) - 1;
                b &= b - 1;
                if (r < N)
                    acc ^= base[(size_t)r * W + w];
            }
        }
        s += __popcll(acc);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        s += __shfl_xor_sync(kFull, s, o);
    if (lane == 0)
        out[c] = s;
}

// op 0: mutate (count pairs from *rng); op 1: local improvement; op 2:
// crossover of np parents (masks/weights in pm/pw, rows materialised in prow).
// rows: N x W scratch holding the individual's materialised rows on entry
// for ops 0/1 (filled by a preceding op 3: materialise masks -> rows).
__global__ void __launch_bounds__(kLocalThreads) op_kernel(int op, const uint64_t* base, int N,
                                                           int W, uint64_t* masks, uint32_t* wts,
                                                           uint64_t* rows, uint64_t* rows2,
                                                           uint32_t count, uint64_t* rng,
                                                           uint32_t* G, int np,
                                                           const uint64_t* prow) {
    extern __shared__ __align__(16) unsigned char smem[];
    BuildSmem s = carve_build(smem, N, np > 0 ? np : 1);
    const int tid = threadIdx.x;
    if (op == 3) {  // materialise: rows = masks over window rows, weights kept
        for (int e = tid; e < N * 4; e += blockDim.x)
            s.T[e] = masks[e];
        for (int n = tid; n < N; n += blockDim.x)
            s.srcp[n] = base + (size_t)n * W;
        __syncthreads();
        materialize(s.T, s.srcp, rows, nullptr, nullptr, nullptr, N, W);
    } else if (op == 0) {
        set_identity(s, N, false);
        for (int e = tid; e < N * 4; e += blockDim.x)
            s.M[e] = masks[e];
        for (int n = tid; n < N; n += blockDim.x) {
            s.srcp[n] = rows + (size_t)n * W;
            s.keepw[n] = wts[n];
            s.recount[n] = 0;
        }
        __syncthreads();
        if (N >= 2)
            apply_pairs(s.T, s.M, s.recount, N, count, *rng);
        __syncthreads();
        materialize(s.T, s.srcp, rows2, wts, s.keepw, s.recount, N, W);
        for (int e = tid; e < N * 4; e += blockDim.x)
            masks[e] = s.M[e];
        if (tid == 0 && N >= 2) {  // advance the caller's generator past the draws
            Rng r(*rng);
            for (uint32_t m = 0; m < 2u * count; ++m)
                r.next();
            *rng = r.s;
        }
    } else if (op == 1) {
        uint64_t* A = reinterpret_cast<uint64_t*>(smem);
        __shared__ uint32_t w[kMaxN];
        __shared__ unsigned long long s_best[64];
        __shared__ __align__(8) int s_flag[4 + 2 * 32];
        if (W <= kLi16MaxW)
            local_improve16(rows, masks, wts, N, W, smem, w, s_flag);
        else
            local_improve(rows, masks, wts, N, W, G, A, A + kLiTile * (kLiChunk + 1), w, s_best,
                          &s_flag[0]);
    } else if (op == 2) {
        const uint64_t* pm[4];
        const uint32_t* pw[4];
        const uint64_t* pr[4];
        for (int p = 0; p < np; ++p) {
            pm[p] = masks + (size_t)p * N * 4;
            pw[p] = wts + (size_t)p * N;
            pr[p] = prow + (size_t)p * N * W;
        }
        crossover(pm, pw, pr, np, base, N, W, s.cross, s.srcp, s.M, s.keepw);
        // outputs after the parents: masks[np*N*4 ..], wts[np*N ..]
        for (int e = tid; e < N * 4; e += blockDim.x)
            masks[(size_t)np * N * 4 + e] = s.M[e];
        for (int n = tid; n < N; n += blockDim.x)
            wts[(size_t)np * N + n] = s.keepw[n];
    }
}

// ---------------------------------------------------------------------------
// Host side.

// xorshift64^(d) as 64 columns.
void jump_columns(uint64_t d, uint64_t* cols) {
    for (int b = 0; b < 64; ++b) {
        uint64_t x = 1ull << b;
        for (uint64_t k = 0; k < d; ++k)
            x = xs_step(x);
        cols[b] = x;
    }
}

uint64_t host_jump(const uint64_t* cols, uint64_t s) {
    uint64_t r = 0;
    for (int b = 0; b < 64; ++b)
        if ((s >> b) & 1ull)
            r ^= cols[b];
    return r;
}

int pow2_at_least(int n) {
    int p = 32;
    while (p < n)
        p <<= 1;
    return p;
}

// Window rows compacted to W words, tail bits cleared.
std::vector<uint64_t> compact_window(const uint64_t* words, size_t stride, size_t cols,
                                     const size_t* win, size_t n) {
    const size_t W = (cols + 63) / 64;
    std::vector<uint64_t> base(n * W);
    const uint64_t tail = (cols & 63) ? ((1ull << (cols & 63)) - 1) : ~0ull;
    for (size_t r = 0; r < n; ++r)
        for (size_t w = 0; w < W; ++w) {
            uint64_t v = words[win[r] * stride + w];
            if (w == W - 1)
                v &= tail;
            base[r * W + w] = v;
        }
    return base;
}

int check_window_args(const uint64_t* words, size_t stride, size_t cols, const size_t* win,
                      size_t n, size_t rows_hint) {
    (void)rows_hint;
    if (!words || !win)
        return fail(BMM_EINVAL, "ga: null window");
    if (n == 0 || cols == 0)
        return fail(BMM_EINVAL, "GeneticAlgorithm::initialize: empty window is not supported");
    if (n > (size_t)kMaxN)
        return fail(BMM_EINVAL, "ga: at most %d window rows are supported, got %zu", kMaxN, n);
    if (stride < (cols + 63) / 64)
        return fail(BMM_EINVAL, "ga: stride is smaller than the row width");
    if (cols > 0xffffffffull)
        return fail(BMM_EINVAL, "ga: too many columns");
    return BMM_OK;
}

// Reference mask layout (ceil(n/64) words per candidate) <-> device (4 words).
// Bits at and above n select no window row and are cleared.
void masks_to_device_layout(const uint64_t* in, size_t n, size_t count, uint64_t* out) {
    const size_t mw = (n + 63) / 64;
    for (size_t c = 0; c < count; ++c)
        for (size_t w = 0; w < 4; ++w) {
            uint64_t v = w < mw ? in[c * mw + w] : 0ull;
            if (w * 64 + 64 > n)
                v &= (w * 64 >= n) ? 0ull : ((1ull << (n - w * 64)) - 1);
            out[c * 4 + w] = v;
        }
}
void masks_from_device_layout(const uint64_t* in, size_t n, size_t count, uint64_t* out) {
    const size_t mw = (n + 63) / 64;
    for (size_t c = 0; c < count; ++c)
        for (size_t w = 0; w < mw; ++w)
            out[c * mw + w] = in[c * 4 + w];
}

}  // namespace ga
}  // namespace bmm

using namespace bmm;
using namespace bmm::ga;

namespace {

int ga_alloc(bmm_ga* g, size_t bytes, void** p) {
    *p = nullptr;
    const cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? BMM_ENOMEM : BMM_ECUDA,
                    "ga: device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    }
    g->allocs.push_back(*p);
    return BMM_OK;
}

void ga_free(bmm_ga* g) {
    if (!g)
        return;
    int prev = -1;
    cudaGetDevice(&prev);
    if (g->device >= 0)
        cudaSetDevice(g->device);
    if (g->stream)
        cudaStreamSynchronize(g->stream);
    for (void* p : g->allocs)
        cudaFree(p);
    propose_free(g);
    if (g->h_stat)
        cudaFreeHost(g->h_stat);
    if (g->stream)
        cudaStreamDestroy(g->stream);
    if (prev >= 0)
        cudaSetDevice(prev);
    delete g;
}

int launch_check(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return fail(BMM_ECUDA, "ga: %s launch failed: %s", what, cudaGetErrorString(e));
    return BMM_OK;
}

int ga_generation(bmm_ga* g) {
    const State& st = g->st;
    const Config& c = st.c;
    const int I = g->I, P = c.P;
    cudaStream_t s = g->stream;
    schedule_kernel<<<(I + 3) / 4, 128, 0, s>>>(st);
    build_kernel<<<g->build_grid, kBuildThreads, g->build_smem, s>>>(st, 0);
    if (g->prop.mode != 0)
        BMM_TRY(propose_generation(g));
    if (g->gen % 3 == 0) {  // k_local_improvement_period
        if (c.W <= kLi16MaxW)
            local_kernel<true><<<g->local_grid, kLocalThreads, local16_smem_bytes(c.N), s>>>(st);
        else
            local_kernel<false><<<g->local_grid, kLocalThreads, local_smem_bytes(), s>>>(st);
    }
    const int fit_blocks = (int)(((size_t)I * P * 32 + 255) / 256);
    fitness_kernel<<<fit_blocks, 256, 0, s>>>(st, 1);
    bool mig = false;  // some island exports after this generation
    if (I > 1)
        for (int i = 0; i < I && !mig; ++i)
            mig = g->intervals[i] && (g->gen + 1) % g->intervals[i] == 0;
    const bool cat = c.cat_enable != 0;
    rank_kernel<<<I, g->rank_threads, 0, s>>>(st, kRankStep, (!cat && !mig) ? 1 : 0);
    if (cat) {
        build_kernel<<<g->build_grid, kBuildThreads, g->build_smem, s>>>(st, 1);
        fitness_kernel<<<fit_blocks, 256, 0, s>>>(st, 2);
        rank_kernel<<<I, g->rank_threads, 0, s>>>(st, kRankCat, mig ? 0 : 1);
    }
    if (mig) {
        migrate_kernel<<<I, 256, 0, s>>>(st);
        rank_kernel<<<I, g->rank_threads, 0, s>>>(st, kRankMigrate, 1);
    }
    g->gen += 1;
    return launch_check("generation");
}

int ga_fetch_stats(bmm_ga* g) {
    BMM_CUDA_TRY(cudaMemcpyAsync(g->h_stat, g->st.stat, sizeof(IslandStat) * g->I,
                                 cudaMemcpyDeviceToHost, g->stream));
    BMM_CUDA_TRY(cudaStreamSynchronize(g->stream));
    return BMM_OK;
}

int ga_device_guard(const bmm_ga* g) {
    int dev = -1;
    BMM_CUDA_TRY(cudaGetDevice(&dev));
    if (dev != g->device)
        return fail(BMM_EINVAL, "ga: created on device %d, used on device %d", g->device, dev);
    return BMM_OK;
}

// One-CTA operator launch on a scratch copy of the window.
struct OpScratch {
    void* base = nullptr;
    void* masks = nullptr;
    void* wts = nullptr;
    void* rows = nullptr;
    void* rows2 = nullptr;
    void* rng = nullptr;
    void* G = nullptr;
    ~OpScratch() {
        cudaFree(base);
        cudaFree(masks);
        cudaFree(wts);
        cudaFree(rows);
        cudaFree(rows2);
        cudaFree(rng);
        cudaFree(G);
    }
};

int op_alloc(void** p, size_t bytes) {
    const cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return fail(BMM_ENOMEM, "ga: device allocation failed: %s", cudaGetErrorString(e));
    }
    return BMM_OK;
}

size_t op_smem(int N, int np) {
    return std::max(std::max(build_smem_bytes(N, np > 0 ? np : 1), local_smem_bytes()),
                    local16_smem_bytes(N));
}

}  // namespace

extern "C" {

BMM_API int bmm_ga_create(const uint64_t* words, size_t stride, size_t cols, const size_t* win,
                          size_t n, const bmm_ga_config* cfgs, size_t islands,
                          const bmm_ga_migration* migration, bmm_ga** out) {
    clear_error();
    if (!out)
        return fail(BMM_EINVAL, "ga: null output");
    *out = nullptr;
    if (!cfgs)
        return fail(BMM_EINVAL, "ga: null config");
    BMM_TRY(check_window_args(words, stride, cols, win, n, 0));
    if (islands < 1 || islands > 65535)
        return fail(BMM_EINVAL, "ga: islands must be in [1, 65535]");
    const bmm_ga_config* cfg = &cfgs[0];
    if (cfg->population_size == 0)
        return fail(BMM_EINVAL,
                    "GeneticAlgorithm::initialize: population_size must be greater than zero");
    if (cfg->population_size > 1024)
        return fail(BMM_EINVAL, "ga: population_size above 1024 is not supported");
    if (cfg->num_parents < 1 || cfg->num_parents > 4)
        return fail(BMM_EINVAL, "ga: num_parents must be in [1, 4]");
    if (cfg->num_offspring < 1)
        return fail(BMM_EINVAL, "ga: num_offspring must be at least 1");
    if (cfg->tournament_size > 65536)
        return fail(BMM_EINVAL, "ga: tournament_size above 65536 is not supported");
    for (size_t i = 0; i < islands; ++i) {
        const bmm_ga_config& o = cfgs[i];
        if (o.population_size != cfg->population_size || o.elite_count != cfg->elite_count ||
            o.num_parents != cfg->num_parents || o.num_offspring != cfg->num_offspring ||
            o.tournament_size != cfg->tournament_size ||
            (o.enable_catastrophe != 0) != (cfg->enable_catastrophe != 0) ||
            o.catastrophe_threshold != cfg->catastrophe_threshold ||
            o.catastrophe_survival_rate != cfg->catastrophe_survival_rate)
            return fail(BMM_EINVAL,
                        "ga: islands must share population_size, elite_count, num_parents, "
                        "num_offspring, tournament_size and the catastrophe settings "
                        "(island %zu differs)", i);
        if (!(o.mutation_rate >= 0.0) || !(o.catastrophe_survival_rate >= 0.0))
            return fail(BMM_EINVAL, "ga: rates must be non-negative");
        if (o.mutation_rate > 1000.0)
            return fail(BMM_EINVAL, "ga: mutation_rate above 1000 is not supported");
    }

    int st_code = 0;
    Workspace* ws = workspace(&st_code);
    if (!ws)
        return st_code;
    bmm_ga* g = new bmm_ga();
    g->device = ws->device;
    g->I = (int)islands;
    g->seeds.resize(islands);
    for (size_t i = 0; i < islands; ++i)
        g->seeds[i] = cfgs[i].seed;
    const int N = (int)n, W = (int)((cols + 63) / 64), P = (int)cfg->population_size;
    Config& c = g->st.c;
    c.N = N;
    c.W = W;
    c.P = P;
    c.E = (int)std::min<uint32_t>(cfg->elite_count, (uint32_t)P);
    c.T = (int)cfg->tournament_size;
    c.parents = (int)cfg->num_parents;
    c.offspring = (int)std::min<uint32_t>(cfg->num_offspring, (uint32_t)P);
    c.cat_enable = cfg->enable_catastrophe ? 1 : 0;
    c.cat_threshold = (int)std::min<uint32_t>(cfg->catastrophe_threshold, 0x7fffffffu);
    {
        const double sv = (double)P * cfg->catastrophe_survival_rate;
        c.cat_survivors = sv >= (double)P ? P : (int)sv;
    }
    std::vector<IslandCfg> icfg(islands);
    g->intervals.resize(islands);
    for (size_t i = 0; i < islands; ++i) {
        IslandCfg& ic = icfg[i];
        std::memset(&ic, 0, sizeof(ic));
        ic.flags = cfgs[i].flags & 7u;
        ic.max_gen = cfgs[i].max_generations;
        ic.max_stale = cfgs[i].max_stale_generations;
        ic.target = cfgs[i].target_total_weight;
        ic.interval = migration ? migration[i].interval_generations : 0u;
        ic.import_count = migration ? migration[i].import_count : 0u;
        g->intervals[i] = ic.interval;
    }
    g->st.I = (int)islands;
    g->cols = (uint32_t)cols;
    g->search_grid = ws->sm_count;
    g->rank_threads = pow2_at_least(P);
    g->build_smem = build_smem_bytes(N, c.parents);
    g->build_grid = ws->sm_count * 4;
    g->local_grid = W <= kLi16MaxW ? ws->sm_count : ws->sm_count * 2;

    const std::vector<uint64_t> base = compact_window(words, stride, cols, win, n);
    std::vector<uint64_t> jm((size_t)(N + 1) * 64), jr(64);
    {
        uint64_t col[64];
        for (int b = 0; b < 64; ++b)
            col[b] = 1ull << b;
        for (int cnt = 0; cnt <= N; ++cnt) {
            if (cnt > 0)
                for (int b = 0; b < 64; ++b)
                    col[b] = xs_step(xs_step(col[b]));
            std::memcpy(&jm[(size_t)cnt * 64], col, sizeof(col));
        }
        jump_columns(6ull * (uint64_t)N, jr.data());
    }
    // initial population (initialize(), lifecycle.cpp:16-64): identity,
    // min(P/4, P-1) heuristic individuals, then make_random
    const int n_heur = std::min(P / 4, P - 1);
    std::vector<Sched> sched((size_t)islands * P);
    std::vector<IslandStat> stat(islands);
    for (size_t i = 0; i < islands; ++i) {
        uint64_t s = cfgs[i].seed ? cfgs[i].seed : kDefaultSeed;
        for (int p = 0; p < P; ++p) {
            Sched& r = sched[i * P + p];
            std::memset(&r, 0, sizeof(r));
            if (p == 0) {
                r.kind = kIdentity;
            } else if (p <= n_heur) {
                r.kind = kHeuristic;
            } else {
                r.kind = kRandom;
                r.rng = s;
                s = host_jump(jr.data(), s);
            }
        }
        IslandStat& is = stat[i];
        std::memset(&is, 0, sizeof(is));
        is.rng = s;
        is.rate = cfgs[i].mutation_rate;
        is.cur = 1;  // the initial population is built into buffer 0
        is.stepped = 1;
    }

    State& S = g->st;
    const size_t ind = (size_t)islands * P;
    int rc = BMM_OK;
    void* p = nullptr;
    auto A = [&](size_t bytes) -> void* {
        if (rc != BMM_OK)
            return nullptr;
        rc = ga_alloc(g, bytes, &p);
        return rc == BMM_OK ? p : nullptr;
    };
    S.icfg = (const IslandCfg*)A(islands * sizeof(IslandCfg));
    S.base = (const uint64_t*)A(base.size() * 8);
    for (int b = 0; b < 2; ++b) {
        S.pop[b].masks = (uint64_t*)A(ind * N * 32);
        S.pop[b].rows = (uint64_t*)A(ind * N * W * 8);
        S.pop[b].wts = (uint32_t*)A(ind * N * 4);
        S.pop[b].fit = (unsigned long long*)A(ind * 8);
    }
    S.order = (uint32_t*)A(ind * 4);
    S.stat = (IslandStat*)A(islands * sizeof(IslandStat));
    S.sched = (Sched*)A(ind * sizeof(Sched));
    S.jump_mut = (const uint64_t*)A(jm.size() * 8);
    S.jump_rand = (const uint64_t*)A(64 * 8);
    S.best_masks = (uint64_t*)A(islands * N * 32);
    S.best_rows = (uint64_t*)A(islands * N * W * 8);
    S.best_wts = (uint32_t*)A(islands * N * 4);
    S.Gs = (uint32_t*)A(W <= kLi16MaxW ? 16 : (size_t)g->local_grid * N * N * 4);
    if (rc != BMM_OK) {
        ga_free(g);
        return rc;
    }
    cudaError_t e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = cudaMallocHost((void**)&g->h_stat, sizeof(IslandStat) * islands);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync((void*)S.icfg, icfg.data(), icfg.size() * sizeof(IslandCfg),
                            cudaMemcpyHostToDevice, g->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync((void*)S.base, base.data(), base.size() * 8, cudaMemcpyHostToDevice,
                            g->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync((void*)S.jump_mut, jm.data(), jm.size() * 8, cudaMemcpyHostToDevice,
                            g->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync((void*)S.jump_rand, jr.data(), 64 * 8, cudaMemcpyHostToDevice,
                            g->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(S.sched, sched.data(), sched.size() * sizeof(Sched),
                            cudaMemcpyHostToDevice, g->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(S.stat, stat.data(), stat.size() * sizeof(IslandStat),
                            cudaMemcpyHostToDevice, g->stream);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(build_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)g->build_smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(local_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)local_smem_bytes());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(local_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)local16_smem_bytes(N));
    if (e != cudaSuccess) {
        ga_free(g);
        return fail(BMM_ECUDA, "ga: setup failed: %s", cudaGetErrorString(e));
    }
    build_kernel<<<g->build_grid, kBuildThreads, g->build_smem, g->stream>>>(S, 0);
    const int fit_blocks = (int)((ind * 32 + 255) / 256);
    // fitness of buffer 0 (cur is still 1 here: "next" population)
    fitness_kernel<<<fit_blocks, 256, 0, g->stream>>>(S, 1);
    rank_kernel<<<(int)islands, g->rank_threads, 0, g->stream>>>(S, kRankInit, 1);
    rc = launch_check("initialisation");
    if (rc == BMM_OK)
        rc = ga_fetch_stats(g);
    if (rc != BMM_OK) {
        ga_free(g);
        return rc;
    }
    *out = g;
    return BMM_OK;
}

BMM_API int bmm_ga_run(bmm_ga* g, uint64_t generations, uint32_t check_every, uint64_t* ran,
                       int* all_done) {
    clear_error();
    if (!g)
        return fail(BMM_EINVAL, "ga: null handle");
    BMM_TRY(ga_device_guard(g));
    if (check_every == 0)
        check_every = 1;
    uint64_t k = 0;
    int done = 1;
    for (int i = 0; i < g->I; ++i)
        done &= g->h_stat[i].done ? 1 : 0;
    while (!done && k < generations) {
        const uint64_t chunk = std::min<uint64_t>(check_every, generations - k);
        for (uint64_t q = 0; q < chunk; ++q)
            BMM_TRY(ga_generation(g));
        k += chunk;
        BMM_TRY(ga_fetch_stats(g));
        done = 1;
        for (int i = 0; i < g->I; ++i)
            done &= g->h_stat[i].done ? 1 : 0;
    }
    if (ran)
        *ran = k;
    if (all_done)
        *all_done = done;
    return BMM_OK;
}

BMM_API int bmm_ga_stats(bmm_ga* g, size_t island, bmm_ga_island_stats* out) {
    clear_error();
    if (!g || !out)
        return fail(BMM_EINVAL, "ga: null argument");
    if (island >= (size_t)g->I)
        return fail(BMM_EINVAL, "ga: island %zu out of range", island);
    const IslandStat& is = g->h_stat[island];
    out->generations = is.generations;
    out->evaluations = is.evaluations;
    out->stale_generations = is.stale;
    out->seed = g->seeds[island];
    out->best_score = is.best;
    out->done = is.done;
    out->no_improvement = is.no_improvement;
    out->mutation_rate = is.rate;
    return BMM_OK;
}

BMM_API int bmm_ga_best(bmm_ga* g, size_t island, uint64_t* masks, uint32_t* weights,
                        uint64_t* score) {
    clear_error();
    if (!g)
        return fail(BMM_EINVAL, "ga: null handle");
    BMM_TRY(ga_device_guard(g));
    size_t isl = island;
    if (island == (size_t)-1) {  // IslandModel::best_individual: first strict minimum
        isl = 0;
        for (int i = 1; i < g->I; ++i)
            if (g->h_stat[i].best < g->h_stat[isl].best)
                isl = (size_t)i;
    }
    if (isl >= (size_t)g->I)
        return fail(BMM_EINVAL, "ga: island %zu out of range", island);
    const int N = g->st.c.N;
    std::vector<uint64_t> m((size_t)N * 4);
    std::vector<uint32_t> w(N);
    BMM_CUDA_TRY(cudaMemcpyAsync(m.data(), g->st.best_masks + isl * N * 4, m.size() * 8,
                                 cudaMemcpyDeviceToHost, g->stream));
    BMM_CUDA_TRY(cudaMemcpyAsync(w.data(), g->st.best_wts + isl * N, w.size() * 4,
                                 cudaMemcpyDeviceToHost, g->stream));
    BMM_CUDA_TRY(cudaStreamSynchronize(g->stream));
    if (masks)
        masks_from_device_layout(m.data(), N, N, masks);
    if (weights)
        std::memcpy(weights, w.data(), w.size() * 4);
    if (score)
        *score = g->h_stat[isl].best;
    return BMM_OK;
}

BMM_API int bmm_ga_population(bmm_ga* g, size_t island, uint64_t* masks, uint32_t* weights,
                              uint64_t* fitness) {
    clear_error();
    if (!g)
        return fail(BMM_EINVAL, "ga: null handle");
    BMM_TRY(ga_device_guard(g));
    if (island >= (size_t)g->I)
        return fail(BMM_EINVAL, "ga: island %zu out of range", island);
    const int N = g->st.c.N, P = g->st.c.P;
    const Pop& p = g->st.pop[g->h_stat[island].cur];
    const size_t first = island * (size_t)P;
    std::vector<uint64_t> m((size_t)P * N * 4);
    BMM_CUDA_TRY(cudaMemcpyAsync(m.data(), p.masks + first * N * 4, m.size() * 8,
                                 cudaMemcpyDeviceToHost, g->stream));
    if (weights)
        BMM_CUDA_TRY(cudaMemcpyAsync(weights, p.wts + first * N, (size_t)P * N * 4,
                                     cudaMemcpyDeviceToHost, g->stream));
    if (fitness)
        BMM_CUDA_TRY(cudaMemcpyAsync(fitness, p.fit + first, (size_t)P * 8,
                                     cudaMemcpyDeviceToHost, g->stream));
    BMM_CUDA_TRY(cudaStreamSynchronize(g->stream));
    if (masks)
        masks_from_device_layout(m.data(), N, (size_t)P * N, masks);
    return BMM_OK;
}

BMM_API int bmm_ga_destroy(bmm_ga* g) {
    ga_free(g);
    return BMM_OK;
}

BMM_API int bmm_ga_set_proposal(bmm_ga* g, const bmm_ga_proposal* p) {
    clear_error();
    if (!g || !p)
        return fail(BMM_EINVAL, "ga: null argument");
    if (p->mode > 3)
        return fail(BMM_EINVAL, "ga: proposal mode must be 0, 1, 2 or 3");
    if (p->mode == 0)
        return BMM_OK;
    if (g->prop.mode != 0)
        return fail(BMM_EINVAL, "ga: the proposal step is already configured");
    const Config& c = g->st.c;
    if (c.N < 17)
        return fail(BMM_EINVAL, "ga: the proposal step needs at least 17 window rows");
    if (g->cols > 32767)
        return fail(BMM_EINVAL, "ga: the proposal step needs at most 32767 columns");
    if (p->queries_per_elite < 1 || p->queries_per_elite > 64)
        return fail(BMM_EINVAL, "ga: queries_per_elite must be in [1, 64]");
    if (p->mode == 1 && !(p->learning_rate > 0.f))
        return fail(BMM_EINVAL, "ga: learning_rate must be positive");
    if (!(p->learned_fraction >= 0.f && p->learned_fraction <= 1.f))
        return fail(BMM_EINVAL, "ga: learned_fraction must be in [0, 1]");
    BMM_TRY(ga_device_guard(g));
    return propose_setup(g, (int)p->mode, (int)p->queries_per_elite, (int)p->train_steps,
                         p->learning_rate, p->learned_fraction, p->seed);
}

BMM_API int bmm_ga_get_proposal_stats(bmm_ga* g, bmm_ga_proposal_stats* out) {
    clear_error();
    if (!g || !out)
        return fail(BMM_EINVAL, "ga: null argument");
    out->tried_learned = g->tot[0];
    out->improved_learned = g->tot[1];
    out->tried_uniform = g->tot[2];
    out->improved_uniform = g->tot[3];
    out->examples = g->examples;
    out->last_loss = g->last_loss;
    out->learned_fraction = g->prop.learned_frac;
    out->paired_generations = g->paired_gens;
    out->paired_rate_learned = g->paired_gens ? g->paired_rate[0] / (double)g->paired_gens : 0.0;
    out->paired_rate_uniform = g->paired_gens ? g->paired_rate[1] / (double)g->paired_gens : 0.0;
    return BMM_OK;
}

BMM_API int bmm_ga_eval(const uint64_t* words, size_t stride, size_t cols, const size_t* win,
                        size_t n, const uint64_t* masks, size_t count, uint32_t* weights) {
    clear_error();
    BMM_TRY(check_window_args(words, stride, cols, win, n, 0));
    if (count && (!masks || !weights))
        return fail(BMM_EINVAL, "ga: null masks or weights");
    if (count == 0)
        return BMM_OK;
    const int N = (int)n, W = (int)((cols + 63) / 64);
    const std::vector<uint64_t> base = compact_window(words, stride, cols, win, n);
    std::vector<uint64_t> dm(count * 4);
    masks_to_device_layout(masks, n, count, dm.data());
    OpScratch s;
    BMM_TRY(op_alloc(&s.base, base.size() * 8));
    BMM_TRY(op_alloc(&s.masks, dm.size() * 8));
    BMM_TRY(op_alloc(&s.wts, count * 4));
    BMM_CUDA_TRY(cudaMemcpy(s.base, base.data(), base.size() * 8, cudaMemcpyHostToDevice));
    BMM_CUDA_TRY(cudaMemcpy(s.masks, dm.data(), dm.size() * 8, cudaMemcpyHostToDevice));
    const size_t blocks = (count * 32 + 255) / 256;
    eval_kernel<<<(unsigned)blocks, 256>>>((const uint64_t*)s.base, N, W,
                                           (const uint64_t*)s.masks, count, (uint32_t*)s.wts);
    BMM_TRY(launch_check("eval"));
    BMM_CUDA_TRY(cudaMemcpy(weights, s.wts, count * 4, cudaMemcpyDeviceToHost));
    return BMM_OK;
}

BMM_API int bmm_ga_mutate(const uint64_t* words, size_t stride, size_t cols, const size_t* win,
                          size_t n, uint64_t* masks, uint32_t* weights, double mutation_rate,
                          uint64_t* rng_state) {
    clear_error();
    BMM_TRY(check_window_args(words, stride, cols, win, n, 0));
    if (!masks || !weights || !rng_state)
        return fail(BMM_EINVAL, "ga: null argument");
    if (!(mutation_rate >= 0.0) || mutation_rate > 1000.0)
        return fail(BMM_EINVAL, "ga: mutation_rate must be in [0, 1000]");
    const int N = (int)n, W = (int)((cols + 63) / 64);
    const double prod = (double)N * mutation_rate;
    uint32_t count = prod >= 4294967295.0 ? 0xffffffffu : (uint32_t)prod;
    count = count < 1u ? 1u : count;
    const std::vector<uint64_t> base = compact_window(words, stride, cols, win, n);
    std::vector<uint64_t> dm((size_t)N * 4);
    masks_to_device_layout(masks, n, n, dm.data());
    uint64_t rs = *rng_state ? *rng_state : kDefaultSeed;
    OpScratch s;
    BMM_TRY(op_alloc(&s.base, base.size() * 8));
    BMM_TRY(op_alloc(&s.masks, dm.size() * 8));
    BMM_TRY(op_alloc(&s.wts, (size_t)N * 4));
    BMM_TRY(op_alloc(&s.rows, (size_t)N * W * 8));
    BMM_TRY(op_alloc(&s.rows2, (size_t)N * W * 8));
    BMM_TRY(op_alloc(&s.rng, 8));
    BMM_CUDA_TRY(cudaMemcpy(s.base, base.data(), base.size() * 8, cudaMemcpyHostToDevice));
    BMM_CUDA_TRY(cudaMemcpy(s.masks, dm.data(), dm.size() * 8, cudaMemcpyHostToDevice));
    BMM_CUDA_TRY(cudaMemcpy(s.wts, weights, (size_t)N * 4, cudaMemcpyHostToDevice));
    BMM_CUDA_TRY(cudaMemcpy(s.rng, &rs, 8, cudaMemcpyHostToDevice));
    const size_t sm = op_smem(N, 1);
    BMM_CUDA_TRY(
        cudaFuncSetAttribute(op_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    op_kernel<<<1, kLocalThreads, sm>>>(3, (const uint64_t*)s.base, N, W, (uint64_t*)s.masks,
                                        (uint32_t*)s.wts, (uint64_t*)s.rows, nullptr, 0, nullptr,
                                        nullptr, 1, nullptr);
    op_kernel<<<1, kLocalThreads, sm>>>(0, (const uint64_t*)s.base, N, W, (uint64_t*)s.masks,
                                        (uint32_t*)s.wts, (uint64_t*)s.rows, (uint64_t*)s.rows2,
                                        count, (uint64_t*)s.rng, nullptr, 1, nullptr);
    BMM_TRY(launch_check("mutate"));
    BMM_CUDA_TRY(cudaMemcpy(dm.data(), s.masks, dm.size() * 8, cudaMemcpyDeviceToHost));
    BMM_CUDA_TRY(cudaMemcpy(weights, s.wts, (size_t)N * 4, cudaMemcpyDeviceToHost));
    BMM_CUDA_TRY(cudaMemcpy(rng_state, s.rng, 8, cudaMemcpyDeviceToHost));
    masks_from_device_layout(dm.data(), n, n, masks);
    return BMM_OK;
}

BMM_API int bmm_ga_local_improve(const uint64_t* words, size_t stride, size_t cols,
                                 const size_t* win, size_t n, uint64_t* masks, uint32_t* weights) {
    clear_error();
    BMM_TRY(check_window_args(words, stride, cols, win, n, 0));
    if (!masks || !weights)
        return fail(BMM_EINVAL, "ga: null argument");
    const int N = (int)n, W = (int)((cols + 63) / 64);
    if (N < 2)
        return BMM_OK;  // candidate_count < 2: unchanged
    const std::vector<uint64_t> base = compact_window(words, stride, cols, win, n);
    std::vector<uint64_t> dm((size_t)N * 4);
    masks_to_device_layout(masks, n, n, dm.data());
    OpScratch s;
    BMM_TRY(op_alloc(&s.base, base.size() * 8));
    BMM_TRY(op_alloc(&s.masks, dm.size() * 8));
    BMM_TRY(op_alloc(&s.wts, (size_t)N * 4));
    BMM_TRY(op_alloc(&s.rows, (size_t)N * W * 8));
    BMM_TRY(op_alloc(&s.G, (size_t)N * N * 4));
    BMM_CUDA_TRY(cudaMemcpy(s.base, base.data(), base.size() * 8, cudaMemcpyHostToDevice));
    BMM_CUDA_TRY(cudaMemcpy(s.masks, dm.data(), dm.size() * 8, cudaMemcpyHostToDevice));
    BMM_CUDA_TRY(cudaMemcpy(s.wts, weights, (size_t)N * 4, cudaMemcpyHostToDevice));
    const size_t sm = op_smem(N, 1);
    BMM_CUDA_TRY(
        cudaFuncSetAttribute(op_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    op_kernel<<<1, kLocalThreads, sm>>>(3, (const uint64_t*)s.base, N, W, (uint64_t*)s.masks,
                                        (uint32_t*)s.wts, (uint64_t*)s.rows, nullptr, 0, nullptr,
                                        nullptr, 1, nullptr);
    op_kernel<<<1, kLocalThreads, sm>>>(1, (const uint64_t*)s.base, N, W, (uint64_t*)s.masks,
                                        (uint32_t*)s.wts, (uint64_t*)s.rows, nullptr, 0, nullptr,
                                        (uint32_t*)s.G, 1, nullptr);
    BMM_TRY(launch_check("local improvement"));
    BMM_CUDA_TRY(cudaMemcpy(dm.data(), s.masks, dm.size() * 8, cudaMemcpyDeviceToHost));
    BMM_CUDA_TRY(cudaMemcpy(weights, s.wts, (size_t)N * 4, cudaMemcpyDeviceToHost));
    masks_from_device_layout(dm.data(), n, n, masks);
    return BMM_OK;
}

BMM_API int bmm_ga_crossover(size_t n, size_t parents, const uint64_t* parent_masks,
                             const uint32_t* parent_weights, uint64_t* child_masks,
                             uint32_t* child_weights) {
    clear_error();
    if (n == 0 || n > (size_t)kMaxN)
        return fail(BMM_EINVAL, "ga: crossover needs 1..%d candidates", kMaxN);
    if (parents < 1 || parents > 4)
        return fail(BMM_EINVAL, "ga: crossover needs 1..4 parents");
    if (!parent_masks || !parent_weights || !child_masks || !child_weights)
        return fail(BMM_EINVAL, "ga: null argument");
    const int N = (int)n, np = (int)parents;
    std::vector<uint64_t> dm((size_t)(np + 1) * N * 4, 0ull);
    masks_to_device_layout(parent_masks, n, (size_t)np * N, dm.data());
    OpScratch s;
    BMM_TRY(op_alloc(&s.masks, dm.size() * 8));
    BMM_TRY(op_alloc(&s.wts, (size_t)(np + 1) * N * 4));
    BMM_TRY(op_alloc(&s.base, 8));  // row pointers only; W = 1 dummy rows are never read
    BMM_TRY(op_alloc(&s.rows, (size_t)np * N * 8));
    BMM_CUDA_TRY(cudaMemcpy(s.masks, dm.data(), dm.size() * 8, cudaMemcpyHostToDevice));
    BMM_CUDA_TRY(
        cudaMemcpy(s.wts, parent_weights, (size_t)np * N * 4, cudaMemcpyHostToDevice));
    const size_t sm = op_smem(N, np);
    BMM_CUDA_TRY(
        cudaFuncSetAttribute(op_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    op_kernel<<<1, kLocalThreads, sm>>>(2, (const uint64_t*)s.base, N, 1, (uint64_t*)s.masks,
                                        (uint32_t*)s.wts, nullptr, nullptr, 0, nullptr, nullptr,
                                        np, (const uint64_t*)s.rows);
    BMM_TRY(launch_check("crossover"));
    BMM_CUDA_TRY(cudaMemcpy(dm.data(), s.masks, dm.size() * 8, cudaMemcpyDeviceToHost));
    std::vector<uint32_t> w((size_t)(np + 1) * N);
    BMM_CUDA_TRY(cudaMemcpy(w.data(), s.wts, w.size() * 4, cudaMemcpyDeviceToHost));
    masks_from_device_layout(dm.data() + (size_t)np * N * 4, n, n, child_masks);
    std::memcpy(child_weights, w.data() + (size_t)np * N, (size_t)N * 4);
    return BMM_OK;
}

}  // extern "C"
