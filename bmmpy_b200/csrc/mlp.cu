// Proposal network for the genetic algorithm: a 512 -> 256 -> 256 -> 256 MLP
// (ReLU) whose three GEMMs run on the 5th-generation tensor cores (tcgen05,
// BF16 operands, FP32 accumulators in TMEM), with hand-written backward and
// Adam kernels.  No reference counterpart: the reference GA draws its
// mutation partners uniformly (operators.cpp:100-129).
//
// Inputs per query (a target row i of an individual): 256 per-row weight
// features -- the pairwise weight changes of the other rows, in ascending
// order -- and the ±1 bits of row i's 256-column sketch; outputs: one logit
// per rank position (how likely the row at that position belongs to an
// improving XOR subset for i).
//
// GEMM kernel.  C[M x N] = A[M x K] . B[N x K]^T for any element strides of A
// and B (transposes are folded into the staging loads), FP32 or BF16 sources
// rounded to BF16 while they are written to shared memory in the canonical
// K-major layout (as 16-byte vectors where the strides allow: K-contiguous
// rows directly, row-contiguous operands through 8 x 8 register transposes);
// one CTA per 128 x 256 output tile, K in chunks of 64 (four K=16 MMAs per
// chunk) in two buffers so that staging overlaps the MMAs, TMEM accumulator
// of 256 columns; the epilogue reads
// TMEM (tcgen05.ld 32x32b) and applies scale, bias, the ReLU-backward mask and
// ReLU, writing FP32 (pre-activation) and/or BF16 (activation) outputs.
#include "common.cuh"
#include "mlp.cuh"
#include "umma.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstring>
#include <vector>

namespace bmm {
namespace mlp {

constexpr int kBM = 128, kBN = 256, kBK = 64;
constexpr int kGemmThreads = 256;  // 8 warps stage; in the epilogue warp w reads TMEM lanes
                                    // 32 (w % 4).., columns 128 (w / 4)..
constexpr uint32_t kWaitLimit = 1u << 22;
// Two buffers of 48 KB of operand tiles; 100 KB keeps at most two CTAs (2 x 256
// TMEM columns) resident per SM.
constexpr size_t kGemmSmem = 100 * 1024;

struct GemmArgs {
    const void* A;
    int a_bf16;
    long long lda_m, lda_k;
    const void* B;
    int b_bf16;
    long long ldb_n, ldb_k;
    int M, N, K;
    float scale;
    const float* bias;       // [N] or null
    const float* relu_mask;  // [M][ldm]: output *= (mask > 0), or null
    long long ldm;
    int relu;                // the BF16 output is max(value, 0)
    float* out_f;            // value before ReLU, [M][ldo_f], or null
    long long ldo_f;
    __nv_bfloat16* out_b;    // [M][ldo_b], or null
    long long ldo_b;
    int ksplit;              // K split over gridDim.z: partial z goes to out_f + z * split_stride
    long long split_stride;
    int* err;
    int a_mode, b_mode;      // staging path per operand (kStage*), chosen on the host
    int vec_f, vec_b, vec_mask;  // epilogue rows 16-byte aligned: vector stores / loads
};

// Staging paths: kStageElem reads element by element with any strides;
// kStageKVec reads 8 consecutive K elements (K-contiguous rows) as one vector
// (BF16 sources by a 16-byte cp.async straight into place, FP32 ones through
// registers, rounded);
// kStageRVec reads an 8 x 8 block as 8 vectors of 8 consecutive rows
// (row-contiguous, K-strided sources: the transposed operands of the backward
// GEMMs) and transposes it in registers.  Vector paths need 16-byte aligned
// vectors: the base pointer and the strided dimension's stride in bytes.
constexpr int kStageElem = 0, kStageKVec = 1, kStageRVec = 2;

__device__ __forceinline__ float load_elem(const void* p, int bf16, long long idx) {
    return bf16 ? __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(p)[idx])
                : reinterpret_cast<const float*>(p)[idx];
}

// rows x kBK tile, element (r, k) = src[(row0 + r) * ld_r + (k0 + k) * ld_k],
// zero outside [0, nrows) x [0, K).
__device__ void stage(unsigned char* dst, int rows, const void* src, int bf16, long long ld_r,
                      long long ld_k, int row0, int nrows, int k0, int K) {
    const int total = rows * kBK;
    const bool kfast = ld_k == 1 || ld_r != 1;  // walk the contiguous index fastest
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        int r, k;
        if (kfast) {
            r = e / kBK;
            k = e % kBK;
        } else {
            k = e / rows;
            r = e % rows;
        }
        const int gr = row0 + r, gk = k0 + k;
        float v = 0.f;
        if (gr < nrows && gk < K)
            v = load_elem(src, bf16, (long long)gr * ld_r + (long long)gk * ld_k);
        *reinterpret_cast<__nv_bfloat16*>(dst + umma::kmajor_offset(r, k, kBK)) =
            __float2bfloat16_rn(v);
    }
}

// 8 elements from src[idx ..] (16-byte aligned) as floats.
__device__ __forceinline__ void load8(const void* p, int bf16, long long idx, float (&v)[8]) {
    if (bf16) {
        const uint4 u = *reinterpret_cast<const uint4*>(
            reinterpret_cast<const __nv_bfloat16*>(p) + idx);
        const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float2 f = __bfloat1622float2(h[i]);
            v[2 * i] = f.x;
            v[2 * i + 1] = f.y;
        }
    } else {
        const float4 a = *reinterpret_cast<const float4*>(reinterpret_cast<const float*>(p) + idx);
        const float4 b =
            *reinterpret_cast<const float4*>(reinterpret_cast<const float*>(p) + idx + 4);
        v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w;
        v[4] = b.x, v[5] = b.y, v[6] = b.z, v[7] = b.w;
    }
}

// Eight values rounded to BF16 (nearest even), packed as one 16-byte chunk.
__device__ __forceinline__ uint4 pack8(const float (&v)[8]) {
    uint4 u;
    __nv_bfloat16* h = reinterpret_cast<__nv_bfloat16*>(&u);
#pragma unroll
    for (int i = 0; i < 8; ++i)
        h[i] = __float2bfloat16_rn(v[i]);
    return u;
}

// Vector staging of a rows x kBK tile (see kStageKVec / kStageRVec); partial
// chunks at the matrix edges go element by element with zero fill.
__device__ void stage_vec(unsigned char* dst, int rows, int mode, const void* src, int bf16,
                          long long ld_r, long long ld_k, int row0, int nrows, int k0, int K) {
    constexpr int KG = kBK / 8;  // 8-element groups along K
    if (mode == kStageKVec) {
        // four chunks per thread in flight: all loads first, then convert and store
        constexpr int B = 4;
        for (int c0 = threadIdx.x; c0 < rows * KG; c0 += blockDim.x * B) {
            float v[B][8];
            uint4 raw[B];
#pragma unroll
            for (int j = 0; j < B; ++j) {
                const int c = c0 + j * blockDim.x;
                const int r = c / KG, kg = c % KG;
                const int gr = row0 + r, gk = k0 + kg * 8;
                if (c < rows * KG && gr < nrows && gk + 7 < K) {
                    if (bf16) {
                        // BF16 source: copied asynchronously straight into place
                        const int r = c / KG, kg = c % KG;
                        const uint32_t sa = (uint32_t)__cvta_generic_to_shared(
                            dst + umma::kmajor_offset(r, kg * 8, kBK));
                        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa),
                                     "l"(reinterpret_cast<const __nv_bfloat16*>(src) +
                                         (long long)gr * ld_r + gk)
                                     : "memory");
                    } else {
                        load8(src, 0, (long long)gr * ld_r + gk, v[j]);
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                        v[j][i] = (c < rows * KG && gr < nrows && gk + i < K)
                                      ? load_elem(src, bf16, (long long)gr * ld_r + gk + i)
                                      : 0.f;
                    if (bf16)
                        raw[j] = pack8(v[j]);
                }
            }
#pragma unroll
            for (int j = 0; j < B; ++j) {
                const int c = c0 + j * blockDim.x;
                if (c >= rows * KG)
                    break;
                const int r = c / KG, kg = c % KG;
                const int gr = row0 + r, gk = k0 + kg * 8;
                if (bf16 && gr < nrows && gk + 7 < K)
                    continue;  // written by its cp.async
                *reinterpret_cast<uint4*>(dst + umma::kmajor_offset(r, kg * 8, kBK)) =
                    bf16 ? raw[j] : pack8(v[j]);
            }
        }
    } else {
        const int RG = rows / 8;
        for (int c = threadIdx.x; c < RG * KG; c += blockDim.x) {
            const int rg = c % RG, kg = c / RG;  // neighbouring threads: neighbouring rows
            const int gr = row0 + rg * 8, gk = k0 + kg * 8;
            float v[8][8];  // v[k][r]
            if (gr + 7 < nrows && gk + 7 < K) {
#pragma unroll
                for (int kk = 0; kk < 8; ++kk)
                    load8(src, bf16, gr + (long long)(gk + kk) * ld_k, v[kk]);
            } else {
#pragma unroll
                for (int kk = 0; kk < 8; ++kk)
#pragma unroll
                    for (int rr = 0; rr < 8; ++rr)
                        v[kk][rr] = (gr + rr < nrows && gk + kk < K)
                                        ? load_elem(src, bf16, gr + rr + (long long)(gk + kk) * ld_k)
                                        : 0.f;
            }
#pragma unroll
            for (int rr = 0; rr < 8; ++rr) {
                float row[8];
#pragma unroll
                for (int kk = 0; kk < 8; ++kk)
                    row[kk] = v[kk][rr];
                *reinterpret_cast<uint4*>(dst + umma::kmajor_offset(rg * 8 + rr, kg * 8, kBK)) =
                    pack8(row);
            }
        }
    }
}

__device__ __forceinline__ void stage_any(unsigned char* dst, int rows, int mode, const void* src,
                                          int bf16, long long ld_r, long long ld_k, int row0,
                                          int nrows, int k0, int K) {
    if (mode == kStageElem)
        stage(dst, rows, src, bf16, ld_r, ld_k, row0, nrows, k0, K);
    else
        stage_vec(dst, rows, mode, src, bf16, ld_r, ld_k, row0, nrows, k0, K);
}

// Epilogue of a 128 x 256 tile: warp w reads TMEM lanes 32 (w % 4).. and
// columns 128 (w / 4)..; scale, bias, ReLU-backward mask, FP32 / BF16 outputs.
__device__ __forceinline__ void gemm_epilogue(const GemmArgs& g, uint32_t tmem, int m0, int n0,
                                              bool empty, float* out_f, const float* s_bias) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int quarter = warp & 3, half = warp >> 2;
    const int m = m0 + quarter * 32 + lane;
    for (int c = half * (kBN / 64); c < (half + 1) * (kBN / 64); ++c) {
        float v[32];
        umma::tmem_ld32(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(c * 32), v);
        if (m >= g.M)
            continue;
        if (empty)
#pragma unroll
            for (int i = 0; i < 32; ++i)
                v[i] = 0.f;
        // 32 consecutive outputs of row m: 16-byte vector loads and stores
        // where the host found the rows aligned, element by element else
        const int nb = n0 + c * 32;
        const bool full = nb + 31 < g.N;
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            float val = v[i] * g.scale;
            if (s_bias)
                val += s_bias[c * 32 + i];  // the tile's biases, staged at set-up
            v[i] = val;
        }
        if (g.relu_mask) {
            const float* mrow = g.relu_mask + (long long)m * g.ldm + nb;
            if (full && g.vec_mask) {
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const float4 mk = reinterpret_cast<const float4*>(mrow)[q];
                    if (!(mk.x > 0.f)) v[4 * q] = 0.f;
                    if (!(mk.y > 0.f)) v[4 * q + 1] = 0.f;
                    if (!(mk.z > 0.f)) v[4 * q + 2] = 0.f;
                    if (!(mk.w > 0.f)) v[4 * q + 3] = 0.f;
                }
            } else {
#pragma unroll
                for (int i = 0; i < 32; ++i)
                    if (nb + i < g.N && !(mrow[i] > 0.f))
                        v[i] = 0.f;
            }
        }
        if (out_f) {
            float* orow = out_f + (long long)m * g.ldo_f + nb;
            if (full && g.vec_f) {
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    reinterpret_cast<float4*>(orow)[q] =
                        make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            } else {
#pragma unroll
                for (int i = 0; i < 32; ++i)
                    if (nb + i < g.N)
                        orow[i] = v[i];
            }
        }
        if (g.out_b) {
            __nv_bfloat16* brow = g.out_b + (long long)m * g.ldo_b + nb;
            if (full && g.vec_b) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    float b8[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                        b8[i] = g.relu ? fmaxf(v[8 * q + i], 0.f) : v[8 * q + i];
                    reinterpret_cast<uint4*>(brow)[q] = pack8(b8);
                }
            } else {
#pragma unroll
                for (int i = 0; i < 32; ++i)
                    if (nb + i < g.N)
                        brow[i] = __float2bfloat16_rn(g.relu ? fmaxf(v[i], 0.f) : v[i]);
            }
        }
    }
}

// Two operand buffers: the K chunk after the current one is staged while
// the tensor cores work on the current one; buffer b is refilled only after
// the MMAs that read it have signalled its mbarrier.
__global__ void __launch_bounds__(kGemmThreads) gemm_kernel(GemmArgs g) {
    extern __shared__ __align__(1024) unsigned char smem[];
    constexpr int kTileA = kBM * kBK * 2, kTileB = kBN * kBK * 2;
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t tmem_slot;
    __shared__ int s_fail;
    __shared__ float s_bias[kBN];
    const int tid = threadIdx.x, warp = tid >> 5;
    const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * kBN;
    if (g.bias)
        for (int i = tid; i < kBN; i += blockDim.x)
            s_bias[i] = n0 + i < g.N ? g.bias[n0 + i] : 0.f;
    if (warp == 0)
        umma::tmem_alloc(&tmem_slot, 256);
    if (tid == 0) {
        umma::mbar_init(umma::smem_u32(&mbar[0]), 1);
        umma::mbar_init(umma::smem_u32(&mbar[1]), 1);
        s_fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = tmem_slot;
    const uint32_t idesc = umma::idesc_bf16(kBM, kBN);
    const int nk_all = (g.K + kBK - 1) / kBK;
    const int per = (nk_all + g.ksplit - 1) / g.ksplit;
    const int kbeg = blockIdx.z * per;
    const int nk = min(nk_all, kbeg + per);
    float* out_f = g.out_f ? g.out_f + (long long)blockIdx.z * g.split_stride : nullptr;
    auto sA = [&](int b) { return smem + b * (kTileA + kTileB); };
    auto sB = [&](int b) { return smem + b * (kTileA + kTileB) + kTileA; };
    // the k-th commit on a barrier completes its phase k: parity k & 1
    auto parity_of = [](int i) { return (uint32_t)((i >> 1) & 1); };
    int last = -1;  // index of the last chunk whose MMAs were committed
    if (kbeg < nk) {
        stage_any(sB(0), kBN, g.b_mode, g.B, g.b_bf16, g.ldb_n, g.ldb_k, n0, g.N, kbeg * kBK, g.K);
        stage_any(sA(0), kBM, g.a_mode, g.A, g.a_bf16, g.lda_m, g.lda_k, m0, g.M, kbeg * kBK, g.K);
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    umma::fence_async_smem();
    __syncthreads();
    for (int i = 0; kbeg + i < nk; ++i) {
        const int b = i & 1, kc = kbeg + i;
        if (tid == 0) {
            umma::fence_after_sync();
            const uint32_t a0 = umma::smem_u32(sA(b)), b0 = umma::smem_u32(sB(b));
#pragma unroll
            for (int s = 0; s < kBK / 16; ++s) {
                const uint64_t da = umma::smem_desc(a0 + s * 256, 128, (kBK / 8) * 128);
                const uint64_t db = umma::smem_desc(b0 + s * 256, 128, (kBK / 8) * 128);
                umma::mma_bf16(tmem, da, db, idesc, (i > 0 || s > 0) ? 1u : 0u);
            }
            umma::commit(umma::smem_u32(&mbar[b]));
        }
        last = i;
        if (kc + 1 < nk) {
            if (i >= 1 && !umma::mbar_wait(umma::smem_u32(&mbar[b ^ 1]), parity_of(i - 1),
                                           kWaitLimit))
                s_fail = 1;
            stage_any(sB(b ^ 1), kBN, g.b_mode, g.B, g.b_bf16, g.ldb_n, g.ldb_k, n0, g.N,
                      (kc + 1) * kBK, g.K);
            stage_any(sA(b ^ 1), kBM, g.a_mode, g.A, g.a_bf16, g.lda_m, g.lda_k, m0, g.M,
                      (kc + 1) * kBK, g.K);
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
        umma::fence_async_smem();
        __syncthreads();
        if (s_fail)
            break;
    }
    // all MMAs done: the last commit arrives after every earlier tcgen05 op
    if (last >= 0 && !s_fail &&
        !umma::mbar_wait(umma::smem_u32(&mbar[last & 1]), parity_of(last), kWaitLimit))
        s_fail = 1;
    __syncthreads();
    umma::fence_after_sync();
    const bool empty = kbeg >= nk;  // this split has no K chunk: its partial is zero
    if (!s_fail) {
        gemm_epilogue(g, tmem, m0, n0, empty, out_f, g.bias ? s_bias : nullptr);
    } else {
        if (tid == 0)
            atomicExch(g.err, 1);
        // let the MMAs in flight finish (bounded) before the TMEM is released
        if (last >= 0)
            umma::mbar_wait(umma::smem_u32(&mbar[last & 1]), parity_of(last), kWaitLimit);
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        umma::fence_after_sync();
        umma::tmem_dealloc(tmem, 256);
    }
}

// TMA-fed GEMM for BF16 operands whose rows are K-contiguous (the forward
// GEMMs: activations or features times the BF16 weight copy): a 4-stage ring
// of 128 x 64 (A) and 256 x 64 (B) tiles that the Tensor Memory Accelerator
// writes with 128-byte swizzling (cp.async.bulk.tensor, tensor maps over this
// GPU's memory, no multicast), one producer thread, one MMA thread
// (tcgen05.mma reading the swizzled tiles directly), the same epilogue.
// full[s] completes when a stage's two tiles have landed, empty[s] when the
// MMAs that read it are done; every wait is bounded.
constexpr int kTmaStages = 4;
constexpr int kTmaTileA = kBM * kBK * 2, kTmaTileB = kBN * kBK * 2;
constexpr size_t kTmaSmem = 1024 + (size_t)kTmaStages * (kTmaTileA + kTmaTileB);
constexpr uint32_t kTmaWaitLimit = 1u << 20;

__global__ void __launch_bounds__(kGemmThreads, 1)
    gemm_tma_kernel(const __grid_constant__ CUtensorMap tma_a,
                    const __grid_constant__ CUtensorMap tma_b, GemmArgs g) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    __shared__ __align__(8) uint64_t full[kTmaStages], empty[kTmaStages], done;
    __shared__ uint32_t tmem_slot;
    __shared__ int s_fail, s_issued, s_consumed;
    __shared__ float s_bias[kBN];
    const int tid = threadIdx.x, warp = tid >> 5;
    const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * kBN;
    if (g.bias)
        for (int i = tid; i < kBN; i += blockDim.x)
            s_bias[i] = n0 + i < g.N ? g.bias[n0 + i] : 0.f;
    if (warp == 0)
        umma::tmem_alloc(&tmem_slot, 256);
    if (tid == 0) {
        for (int i = 0; i < kTmaStages; ++i) {
            umma::mbar_init(umma::smem_u32(&full[i]), 1);
            umma::mbar_init(umma::smem_u32(&empty[i]), 1);
        }
        umma::mbar_init(umma::smem_u32(&done), 1);
        s_fail = 0;
        s_issued = 0;
        s_consumed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = tmem_slot;
    const int nk = g.K / kBK;
    auto sA = [&](int st) { return smem + st * (kTmaTileA + kTmaTileB); };
    auto sB = [&](int st) { return smem + st * (kTmaTileA + kTmaTileB) + kTmaTileA; };
    if (tid == 0) {  // producer
        int kb = 0;
        for (; kb < nk; ++kb) {
            const int st = kb % kTmaStages;
            if (kb >= kTmaStages &&
                !umma::mbar_wait(umma::smem_u32(&empty[st]), ((kb / kTmaStages) - 1) & 1,
                                 kTmaWaitLimit)) {
                atomicExch(&s_fail, 1);
                break;
            }
            if (*(volatile int*)&s_fail)
                break;
            const uint32_t fb = umma::smem_u32(&full[st]);
            umma::mbar_arrive_expect_tx(fb, kTmaTileA + kTmaTileB);
            umma::tma_load_2d(umma::smem_u32(sA(st)), &tma_a, kb * kBK, m0, fb);
            umma::tma_load_2d(umma::smem_u32(sB(st)), &tma_b, kb * kBK, n0, fb);
        }
        s_issued = kb;
    } else if (tid == 32) {  // MMA issuer
        const uint32_t idesc = umma::idesc_bf16(kBM, kBN);
        int kb = 0;
        for (; kb < nk; ++kb) {
            const int st = kb % kTmaStages;
            if (!umma::mbar_wait(umma::smem_u32(&full[st]), (kb / kTmaStages) & 1,
                                 kTmaWaitLimit)) {
                atomicExch(&s_fail, 1);
                break;
            }
            umma::fence_after_sync();
            const uint32_t a0 = umma::smem_u32(sA(st)), b0 = umma::smem_u32(sB(st));
#pragma unroll
            for (int s = 0; s < kBK / 16; ++s)
                umma::mma_bf16(tmem, umma::smem_desc_sw128(a0 + s * 32),
                               umma::smem_desc_sw128(b0 + s * 32), idesc,
                               (kb > 0 || s > 0) ? 1u : 0u);
            umma::commit(umma::smem_u32(&empty[st]));
        }
        s_consumed = kb;
        // arrives once every MMA issued above has completed
        umma::commit(umma::smem_u32(&done));
    }
    __syncthreads();
    const bool ok = !s_fail && umma::mbar_wait(umma::smem_u32(&done), 0, kTmaWaitLimit);
    umma::fence_after_sync();
    if (ok) {
        gemm_epilogue(g, tmem, m0, n0, nk == 0, g.out_f, g.bias ? s_bias : nullptr);
    } else if (tid == 0) {
        atomicExch(g.err, 1);
        // loads issued but never consumed still land in this CTA's shared
        // memory: wait for them (bounded) before the CTA exits
        for (int kb = s_consumed; kb < s_issued; ++kb)
            umma::mbar_wait(umma::smem_u32(&full[kb % kTmaStages]), (kb / kTmaStages) & 1,
                            kTmaWaitLimit);
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        umma::fence_after_sync();
        umma::tmem_dealloc(tmem, 256);
    }
}

// Softmax cross-entropy against target distributions: warp per row.
// dlogits = (softmax - target) / rows; row_loss[r] = -sum(target * log softmax) / rows.
__global__ void xent_kernel(const float* __restrict__ logits, const float* __restrict__ target,
                            float* __restrict__ dlogits, float* row_loss, int rows) {
    const int lane = threadIdx.x & 31;
    const int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (r >= rows)
        return;
    const float* z = logits + (size_t)r * kOut;
    const float* t = target + (size_t)r * kOut;
    float v[kOut / 32];
    float mx = -INFINITY;
#pragma unroll
    for (int q = 0; q < kOut / 32; ++q) {
        v[q] = z[lane + 32 * q];
        mx = fmaxf(mx, v[q]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        mx = fmaxf(mx, __shfl_xor_sync(kFull, mx, o));
    float se = 0.f;
#pragma unroll
    for (int q = 0; q < kOut / 32; ++q)
        se += expf(v[q] - mx);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        se += __shfl_xor_sync(kFull, se, o);
    const float lse = mx + logf(se);
    float l = 0.f;
    const float inv = 1.f / (float)rows;
#pragma unroll
    for (int q = 0; q < kOut / 32; ++q) {
        const int j = lane + 32 * q;
        const float p = expf(v[q] - lse);
        const float tj = t[j];
        dlogits[(size_t)r * kOut + j] = (p - tj) * inv;
        if (tj != 0.f)
            l -= tj * (v[q] - lse);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        l += __shfl_xor_sync(kFull, l, o);
    if (lane == 0)
        row_loss[r] = l * inv;
}

// *loss = sum of row_loss (one CTA of kLossThreads, fixed strided order and
// reduction tree: deterministic).
constexpr int kLossThreads = 1024;
__global__ void __launch_bounds__(kLossThreads)
    loss_sum_kernel(const float* __restrict__ row_loss, int rows, float* loss) {
    __shared__ float part[kLossThreads];
    float s = 0.f;
    for (int r = threadIdx.x; r < rows; r += blockDim.x)
        s += row_loss[r];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        *loss = part[0];
}

// Column sums of a [rows][256] matrix (bias gradients), in two fixed-order
// steps: CTA b sums rows [b * chunk, (b + 1) * chunk) of every column into
// part[b], then split_reduce_kernel adds the parts in b order.
__global__ void colsum_part_kernel(const float* __restrict__ d, int rows, int chunk,
                                   float* __restrict__ part) {
    const int r0 = blockIdx.x * chunk, r1 = min(rows, r0 + chunk);
    float s = 0.f;
    for (int r = r0; r < r1; ++r)
        s += d[(size_t)r * kOut + threadIdx.x];
    part[(size_t)blockIdx.x * kOut + threadIdx.x] = s;
}

// out[i] = sum over z < splits of part[z * n + i], in z order (deterministic).
__global__ void split_reduce_kernel(const float* __restrict__ part, int splits, size_t n,
                                    float* __restrict__ out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    float s = 0.f;
    for (int z = 0; z < splits; ++z)
        s += part[(size_t)z * n + i];
    out[i] = s;
}

// Bias gradient: column sums of d[rows][256] into out[256] (part: scratch of
// at most 8192 x 256 floats).
void colsum(const float* d, int rows, float* part, float* out, cudaStream_t s) {
    const int chunk = std::max(128, (rows + 8191) / 8192);
    const int parts = std::max(1, (rows + chunk - 1) / chunk);
    colsum_part_kernel<<<parts, kOut, 0, s>>>(d, rows, chunk, part);
    split_reduce_kernel<<<1, kOut, 0, s>>>(part, parts, kOut, out);
}

// Adam (Kingma & Ba) with bias correction on the FP32 master parameters.
// Also rewrites the BF16 copy of the weights that the GEMMs read.
__global__ void adam_kernel(float* __restrict__ w, __nv_bfloat16* __restrict__ wb,
                            float* __restrict__ m, float* __restrict__ v,
                            const float* __restrict__ grad, size_t n, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float g = grad[i];
    const float mi = b1 * m[i] + (1.f - b1) * g;
    const float vi = b2 * v[i] + (1.f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    wb[i] = __float2bfloat16_rn(wi);
}

// The BF16 copy of the weights: the same rounding the GEMM staging applies to
// FP32 operands, done once per update instead of once per CTA and K chunk.
__global__ void to_bf16_kernel(const float* __restrict__ w, __nv_bfloat16* __restrict__ wb,
                               size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        wb[i] = __float2bfloat16_rn(w[i]);
}

}  // namespace mlp
}  // namespace bmm

using namespace bmm;
using namespace bmm::mlp;

namespace {

// The vector paths need 16-byte aligned 8-element vectors: a 16-byte aligned
// base and a stride of the other dimension that keeps every vector aligned.
int stage_mode(const void* p, int bf16, long long ld_r, long long ld_k) {
    const long long vec = bf16 ? 8 : 4;  // elements per 16 bytes
    if ((reinterpret_cast<uintptr_t>(p) & 15) != 0)
        return kStageElem;
    if (ld_k == 1 && ld_r % vec == 0)
        return kStageKVec;
    if (ld_r == 1 && ld_k % vec == 0)
        return kStageRVec;
    return kStageElem;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// dependency on the driver library).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    }
    return fn;
}

// 2-D BF16 tensor map of `rows` rows of K elements (row pitch `row_bytes`),
// boxes of 64 x box_rows, 128-byte swizzle, zero fill outside the matrix.
bool make_bf16_map(CUtensorMap* m, const void* base, long long K, long long rows,
                   long long row_bytes, int box_rows) {
    const auto encode = tensor_map_encoder();
    if (!encode)
        return false;
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)row_bytes};
    const cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides,
                  box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

int g_mlp_use_tma = 1;

namespace {

int gemm_launch(const GemmArgs& a, cudaStream_t s) {
    static thread_local int attr_dev = -1;
    int dev = -1;
    cudaGetDevice(&dev);
    if (attr_dev != dev) {
        BMM_CUDA_TRY(cudaFuncSetAttribute(gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)kGemmSmem));
        BMM_CUDA_TRY(cudaFuncSetAttribute(gemm_tma_kernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)kTmaSmem));
        attr_dev = dev;
    }
    GemmArgs g = a;
    g.a_mode = stage_mode(a.A, a.a_bf16, a.lda_m, a.lda_k);
    g.b_mode = stage_mode(a.B, a.b_bf16, a.ldb_n, a.ldb_k);
    auto al16 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
    g.vec_f = a.out_f && al16(a.out_f) && a.ldo_f % 4 == 0 &&
              (a.ksplit <= 1 || a.split_stride % 4 == 0);
    g.vec_b = a.out_b && al16(a.out_b) && a.ldo_b % 8 == 0;
    g.vec_mask = a.relu_mask && al16(a.relu_mask) && a.ldm % 4 == 0;
    dim3 grid((a.M + kBM - 1) / kBM, (a.N + kBN - 1) / kBN, a.ksplit > 1 ? a.ksplit : 1);
    // BF16 operands with K-contiguous, 16-byte aligned rows and whole 64-wide
    // K chunks: TMA staging (box x coordinates are multiples of 64 elements)
    if (g_mlp_use_tma && a.a_bf16 && a.b_bf16 && g.a_mode == kStageKVec &&
        g.b_mode == kStageKVec && a.K % kBK == 0 && a.ksplit <= 1) {
        CUtensorMap ma, mb;
        if (make_bf16_map(&ma, a.A, a.K, a.M, a.lda_m * 2, kBM) &&
            make_bf16_map(&mb, a.B, a.K, a.N, a.ldb_n * 2, kBN)) {
            gemm_tma_kernel<<<grid, kGemmThreads, kTmaSmem, s>>>(ma, mb, g);
            const cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess)
                return fail(BMM_ECUDA, "mlp: gemm (TMA) launch failed: %s", cudaGetErrorString(e));
            return BMM_OK;
        }
    }
    gemm_kernel<<<grid, kGemmThreads, kGemmSmem, s>>>(g);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return fail(BMM_ECUDA, "mlp: gemm launch failed: %s", cudaGetErrorString(e));
    return BMM_OK;
}

GemmArgs gemm_args(const void* A, int a_bf16, long long lda_m, long long lda_k, const void* B,
                   int b_bf16, long long ldb_n, long long ldb_k, int M, int N, int K, int* err) {
    GemmArgs a;
    std::memset(&a, 0, sizeof(a));
    a.A = A;
    a.a_bf16 = a_bf16;
    a.lda_m = lda_m;
    a.lda_k = lda_k;
    a.B = B;
    a.b_bf16 = b_bf16;
    a.ldb_n = ldb_n;
    a.ldb_k = ldb_k;
    a.M = M;
    a.N = N;
    a.K = K;
    a.scale = 1.f;
    a.ksplit = 1;
    a.err = err;
    return a;
}

// Weight gradient dW[M][N] = A^T-like product with K = batch rows, split over
// K into `part` (ksplit partials of M * N) and reduced in a fixed order.
int gemm_wgrad(GemmArgs a, float* out, float* part, cudaStream_t s) {
    const int nk = (a.K + kBK - 1) / kBK;
    const int splits = std::max(1, std::min(nk, 16));
    const size_t n = (size_t)a.M * a.N;
    a.ksplit = splits;
    a.out_f = splits > 1 ? part : out;
    a.ldo_f = a.N;
    a.split_stride = (long long)n;
    BMM_TRY(gemm_launch(a, s));
    if (splits > 1)
        split_reduce_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(part, splits, n, out);
    return BMM_OK;
}

int check_err(bmm_mlp* h) {
    int e = 0;
    BMM_CUDA_TRY(cudaMemcpyAsync(&e, h->err, 4, cudaMemcpyDeviceToHost, h->stream));
    BMM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (e)
        return fail(BMM_ETIMEOUT, "mlp: a tensor-core wait timed out");
    return BMM_OK;
}

}  // namespace

int bmm::mlp::ensure_cap(bmm_mlp* h, size_t rows) {
    if (rows <= h->cap)
        return BMM_OK;
    size_t cap = std::max<size_t>(rows, 256);
    float** fs[] = {&h->z1, &h->z2, &h->z3, &h->dz3, &h->dz2, &h->dz1, &h->t, &h->row_loss};
    for (float** p : fs) {
        cudaFree(*p);
        *p = nullptr;
    }
    cudaFree(h->h1);
    cudaFree(h->h2);
    cudaFree(h->x);
    h->h1 = h->h2 = nullptr;
    h->x = nullptr;
    h->cap = 0;
    cudaError_t e = cudaSuccess;
    for (float** p : fs)
        if (e == cudaSuccess)
            e = cudaMalloc(p, cap * 256 * 4);
    if (e == cudaSuccess)
        e = cudaMalloc(&h->h1, cap * 256 * 2);
    if (e == cudaSuccess)
        e = cudaMalloc(&h->h2, cap * 256 * 2);
    if (e == cudaSuccess)
        e = cudaMalloc(&h->x, cap * kIn * 4);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(BMM_ENOMEM, "mlp: scratch allocation failed: %s", cudaGetErrorString(e));
    }
    h->cap = cap;
    return BMM_OK;
}


namespace bmm {
namespace mlp {

// Forward pass of `rows` inputs X (FP32 or BF16, row stride kIn) into the
// handle's scratch: z1/h1, z2/h2, logits z3 (or `logits` if given).
int forward_dev(bmm_mlp* h, const void* X, int x_bf16, int rows, float* logits, bool keep_pre) {
    // keep_pre: also write the FP32 pre-activations z1, z2 (the ReLU masks of
    // a following backward pass); inference needs only the BF16 activations
    GemmArgs a = gemm_args(X, x_bf16, kIn, 1, h->wb + kW1, 1, kIn, 1, rows, kHid, kIn, h->err);
    a.bias = h->w + kB1;
    a.relu = 1;
    a.out_f = keep_pre ? h->z1 : nullptr;
    a.ldo_f = kHid;
    a.out_b = h->h1;
    a.ldo_b = kHid;
    BMM_TRY(gemm_launch(a, h->stream));
    a = gemm_args(h->h1, 1, kHid, 1, h->wb + kW2, 1, kHid, 1, rows, kHid, kHid, h->err);
    a.bias = h->w + kB2;
    a.relu = 1;
    a.out_f = keep_pre ? h->z2 : nullptr;
    a.ldo_f = kHid;
    a.out_b = h->h2;
    a.ldo_b = kHid;
    BMM_TRY(gemm_launch(a, h->stream));
    a = gemm_args(h->h2, 1, kHid, 1, h->wb + kW3, 1, kHid, 1, rows, kOut, kHid, h->err);
    a.bias = h->w + kB3;
    a.out_f = logits ? logits : h->z3;
    a.ldo_f = kOut;
    return gemm_launch(a, h->stream);
}

// Gradients of the mean cross-entropy for the forward pass just run (rows,
// targets T [rows][256]) into h->g; the loss is written to *h->loss.
int backward_dev(bmm_mlp* h, const void* X, int x_bf16, const float* T, int rows) {
    cudaStream_t s = h->stream;
    xent_kernel<<<(rows * 32 + 255) / 256, 256, 0, s>>>(h->z3, T, h->dz3, h->row_loss, rows);
    loss_sum_kernel<<<1, kLossThreads, 0, s>>>(h->row_loss, rows, h->loss);
    // dW3 = dZ3^T H2, db3
    GemmArgs a = gemm_args(h->dz3, 0, 1, kOut, h->h2, 1, 1, kHid, kOut, kHid, rows, h->err);
    BMM_TRY(gemm_wgrad(a, h->g + kW3, h->part, s));
    colsum(h->dz3, rows, h->part, h->g + kB3, s);
    // dZ2 = (dZ3 W3) * (Z2 > 0)
    a = gemm_args(h->dz3, 0, kOut, 1, h->wb + kW3, 1, 1, kHid, rows, kHid, kOut, h->err);
    a.relu_mask = h->z2;
    a.ldm = kHid;
    a.out_f = h->dz2;
    a.ldo_f = kHid;
    BMM_TRY(gemm_launch(a, s));
    // dW2 = dZ2^T H1, db2
    a = gemm_args(h->dz2, 0, 1, kHid, h->h1, 1, 1, kHid, kHid, kHid, rows, h->err);
    BMM_TRY(gemm_wgrad(a, h->g + kW2, h->part, s));
    colsum(h->dz2, rows, h->part, h->g + kB2, s);
    // dZ1 = (dZ2 W2) * (Z1 > 0)
    a = gemm_args(h->dz2, 0, kHid, 1, h->wb + kW2, 1, 1, kHid, rows, kHid, kHid, h->err);
    a.relu_mask = h->z1;
    a.ldm = kHid;
    a.out_f = h->dz1;
    a.ldo_f = kHid;
    BMM_TRY(gemm_launch(a, s));
    // dW1 = dZ1^T X (N = 512: two column tiles), db1
    a = gemm_args(h->dz1, 0, 1, kHid, X, x_bf16, 1, kIn, kHid, kIn, rows, h->err);
    BMM_TRY(gemm_wgrad(a, h->g + kW1, h->part, s));
    colsum(h->dz1, rows, h->part, h->g + kB1, s);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return fail(BMM_ECUDA, "mlp: backward launch failed: %s", cudaGetErrorString(e));
    return BMM_OK;
}

int adam_dev(bmm_mlp* h) {
    h->step += 1;
    const float c1 = 1.f - (float)std::pow((double)h->b1, (double)h->step);
    const float c2 = 1.f - (float)std::pow((double)h->b2, (double)h->step);
    adam_kernel<<<(unsigned)((kParams + 255) / 256), 256, 0, h->stream>>>(
        h->w, h->wb, h->m, h->v, h->g, kParams, h->lr, h->b1, h->b2, h->eps, c1, c2);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return fail(BMM_ECUDA, "mlp: adam launch failed: %s", cudaGetErrorString(e));
    return BMM_OK;
}

// One optimizer step on device inputs; loss (mean cross-entropy) to *loss_out.
int train_step_dev(bmm_mlp* h, const void* X, int x_bf16, const float* T, int rows) {
    BMM_TRY(ensure_cap(h, (size_t)rows));
    BMM_CUDA_TRY(cudaMemsetAsync(h->loss, 0, 4, h->stream));
    BMM_TRY(forward_dev(h, X, x_bf16, rows, nullptr));
    BMM_TRY(backward_dev(h, X, x_bf16, T, rows));
    return adam_dev(h);
}

}  // namespace mlp
}  // namespace bmm

namespace {

// Glorot-uniform weights from a xorshift64 stream, zero biases.
void init_params(std::vector<float>& p, uint64_t seed) {
    uint64_t s = seed ? seed : 0x9E3779B97F4A7C15ull;
    auto unit = [&]() {
        s ^= s << 13;
        s ^= s >> 7;
        s ^= s << 17;
        return (double)(s >> 11) * (1.0 / 9007199254740992.0);
    };
    p.assign(kParams, 0.f);
    auto fill = [&](size_t off, int out, int in) {
        const double a = std::sqrt(6.0 / (double)(in + out));
        for (size_t i = 0; i < (size_t)out * in; ++i)
            p[off + i] = (float)((2.0 * unit() - 1.0) * a);
    };
    fill(kW1, kHid, kIn);
    fill(kW2, kHid, kHid);
    fill(kW3, kOut, kHid);
}

void mlp_free(bmm_mlp* h) {
    if (!h)
        return;
    if (h->stream)
        cudaStreamSynchronize(h->stream);
    float* fs[] = {h->w, h->m, h->v, h->g, h->z1, h->z2, h->z3, h->dz3, h->dz2, h->dz1, h->x,
                   h->t, h->loss, h->part, h->row_loss};
    for (float* p : fs)
        cudaFree(p);
    cudaFree(h->h1);
    cudaFree(h->h2);
    cudaFree(h->wb);
    cudaFree(h->err);
    if (h->stream && h->owns_stream)
        cudaStreamDestroy(h->stream);
    delete h;
}

}  // namespace

extern "C" {

BMM_API int bmm_mlp_create(uint64_t seed, float learning_rate, bmm_mlp** out) {
    clear_error();
    if (!out)
        return fail(BMM_EINVAL, "mlp: null output");
    *out = nullptr;
    if (!(learning_rate > 0.f))
        return fail(BMM_EINVAL, "mlp: learning rate must be positive");
    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws)
        return st;
    if (ws->sm_count <= 0)
        return fail(BMM_ENODEV, "mlp: no CUDA device");
    bmm_mlp* h = nullptr;
    BMM_TRY(bmm::mlp::create(seed, learning_rate, nullptr, &h));
    *out = h;
    return BMM_OK;
}

}  // extern "C"

namespace bmm {
namespace mlp {

int create(uint64_t seed, float learning_rate, cudaStream_t stream, bmm_mlp** out) {
    *out = nullptr;
    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws)
        return st;
    bmm_mlp* h = new bmm_mlp();
    h->device = ws->device;
    h->lr = learning_rate;
    std::vector<float> p;
    init_params(p, seed);
    cudaError_t e = cudaSuccess;
    if (stream) {
        h->stream = stream;
        h->owns_stream = false;
    } else {
        e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    }
    float** ps[] = {&h->w, &h->m, &h->v, &h->g};
    for (float** q : ps)
        if (e == cudaSuccess)
            e = cudaMalloc(q, kParams * 4);
    if (e == cudaSuccess)
        e = cudaMalloc(&h->wb, kParams * 2);
    if (e == cudaSuccess)
        e = cudaMalloc(&h->part, (size_t)16 * kHid * kIn * 4);
    if (e == cudaSuccess)
        e = cudaMalloc(&h->loss, 4);
    if (e == cudaSuccess)
        e = cudaMalloc(&h->err, 4);
    // everything on the network's stream, in order: the BF16 copy is made
    // from the uploaded weights (a pageable cudaMemcpy may return before its
    // DMA lands, and the network's stream need not wait for it)
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h->w, p.data(), kParams * 4, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(h->m, 0, kParams * 4, h->stream);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(h->v, 0, kParams * 4, h->stream);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(h->err, 0, 4, h->stream);
    if (e == cudaSuccess) {
        to_bf16_kernel<<<(unsigned)((kParams + 255) / 256), 256, 0, h->stream>>>(h->w, h->wb,
                                                                               kParams);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        mlp_free(h);
        return fail(BMM_ENOMEM, "mlp: allocation failed: %s", cudaGetErrorString(e));
    }
    *out = h;
    return BMM_OK;
}

void destroy(bmm_mlp* h) { mlp_free(h); }

}  // namespace mlp
}  // namespace bmm

extern "C" {

BMM_API int bmm_mlp_destroy(bmm_mlp* h) {
    mlp_free(h);
    return BMM_OK;
}

BMM_API size_t bmm_mlp_param_count(void) { return kParams; }

BMM_API int bmm_mlp_get_params(bmm_mlp* h, float* params) {
    clear_error();
    if (!h || !params)
        return fail(BMM_EINVAL, "mlp: null argument");
    BMM_CUDA_TRY(cudaMemcpyAsync(params, h->w, kParams * 4, cudaMemcpyDeviceToHost, h->stream));
    BMM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return BMM_OK;
}

BMM_API int bmm_mlp_set_params(bmm_mlp* h, const float* params) {
    clear_error();
    if (!h || !params)
        return fail(BMM_EINVAL, "mlp: null argument");
    BMM_CUDA_TRY(cudaMemcpyAsync(h->w, params, kParams * 4, cudaMemcpyHostToDevice, h->stream));
    to_bf16_kernel<<<(unsigned)((kParams + 255) / 256), 256, 0, h->stream>>>(h->w, h->wb,
                                                                           kParams);
    BMM_CUDA_TRY(cudaGetLastError());
    BMM_CUDA_TRY(cudaMemsetAsync(h->m, 0, kParams * 4, h->stream));
    BMM_CUDA_TRY(cudaMemsetAsync(h->v, 0, kParams * 4, h->stream));
    BMM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->step = 0;
    return BMM_OK;
}

BMM_API int bmm_mlp_create_on_stream(uint64_t seed, float learning_rate, void* stream,
                                     bmm_mlp** out) {
    clear_error();
    if (!out || !stream)
        return fail(BMM_EINVAL, "mlp: null output, or the null stream (pass a created stream)");
    *out = nullptr;
    if (!(learning_rate > 0.f))
        return fail(BMM_EINVAL, "mlp: learning rate must be positive");
    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws)
        return st;
    return bmm::mlp::create(seed, learning_rate, (cudaStream_t)stream, out);
}

// Device-pointer forms: enqueued on the handle's stream, no synchronisation.
BMM_API int bmm_mlp_forward_dev(bmm_mlp* h, const float* x, size_t rows, float* logits) {
    clear_error();
    if (!h || (rows && (!x || !logits)))
        return fail(BMM_EINVAL, "mlp: null argument");
    if (rows == 0)
        return BMM_OK;
    if (rows > (1u << 24))
        return fail(BMM_EINVAL, "mlp: too many rows");
    BMM_TRY(ensure_cap(h, rows));
    return forward_dev(h, x, 0, (int)rows, logits, false);
}

BMM_API int bmm_mlp_forward_bf16_dev(bmm_mlp* h, const void* x, size_t rows, float* logits) {
    clear_error();
    if (!h || (rows && (!x || !logits)))
        return fail(BMM_EINVAL, "mlp: null argument");
    if (rows == 0)
        return BMM_OK;
    if (rows > (1u << 24))
        return fail(BMM_EINVAL, "mlp: too many rows");
    BMM_TRY(ensure_cap(h, rows));
    return forward_dev(h, x, 1, (int)rows, logits, false);
}

BMM_API int bmm_mlp_tune(int use_tma) {
    clear_error();
    if (use_tma != 0 && use_tma != 1)
        return fail(BMM_EINVAL, "mlp tuning: use_tma must be 0 or 1");
    g_mlp_use_tma = use_tma;
    return BMM_OK;
}

BMM_API int bmm_mlp_train_dev(bmm_mlp* h, const float* x, const float* target, size_t rows,
                              int steps) {
    clear_error();
    if (!h || !x || !target || rows == 0 || steps < 1)
        return fail(BMM_EINVAL, "mlp: null argument, no rows or no steps");
    if (rows > (1u << 24))
        return fail(BMM_EINVAL, "mlp: too many rows");
    BMM_TRY(ensure_cap(h, rows));
    for (int s = 0; s < steps; ++s)
        BMM_TRY(train_step_dev(h, x, 0, target, (int)rows));
    return BMM_OK;
}

BMM_API int bmm_mlp_forward(bmm_mlp* h, const float* x, size_t rows, float* logits) {
    clear_error();
    if (!h || (rows && (!x || !logits)))
        return fail(BMM_EINVAL, "mlp: null argument");
    if (rows == 0)
        return BMM_OK;
    if (rows > (1u << 24))
        return fail(BMM_EINVAL, "mlp: too many rows");
    BMM_TRY(ensure_cap(h, rows));
    BMM_CUDA_TRY(cudaMemcpyAsync(h->x, x, rows * kIn * 4, cudaMemcpyHostToDevice, h->stream));
    BMM_TRY(forward_dev(h, h->x, 0, (int)rows, nullptr));
    BMM_CUDA_TRY(cudaMemcpyAsync(logits, h->z3, rows * kOut * 4, cudaMemcpyDeviceToHost, h->stream));
    return check_err(h);
}

BMM_API int bmm_mlp_grads(bmm_mlp* h, const float* x, const float* target, size_t rows,
                          float* grads, float* loss) {
    clear_error();
    if (!h || !x || !target || !grads || rows == 0)
        return fail(BMM_EINVAL, "mlp: null argument or no rows");
    if (rows > (1u << 24))
        return fail(BMM_EINVAL, "mlp: too many rows");
    BMM_TRY(ensure_cap(h, rows));
    BMM_CUDA_TRY(cudaMemcpyAsync(h->x, x, rows * kIn * 4, cudaMemcpyHostToDevice, h->stream));
    BMM_CUDA_TRY(cudaMemcpyAsync(h->t, target, rows * kOut * 4, cudaMemcpyHostToDevice, h->stream));
    BMM_CUDA_TRY(cudaMemsetAsync(h->loss, 0, 4, h->stream));
    BMM_TRY(forward_dev(h, h->x, 0, (int)rows, nullptr));
    BMM_TRY(backward_dev(h, h->x, 0, h->t, (int)rows));
    BMM_CUDA_TRY(cudaMemcpyAsync(grads, h->g, kParams * 4, cudaMemcpyDeviceToHost, h->stream));
    if (loss)
        BMM_CUDA_TRY(cudaMemcpyAsync(loss, h->loss, 4, cudaMemcpyDeviceToHost, h->stream));
    return check_err(h);
}

BMM_API int bmm_mlp_train(bmm_mlp* h, const float* x, const float* target, size_t rows,
                          int steps, float* loss) {
    clear_error();
    if (!h || !x || !target || rows == 0 || steps < 1)
        return fail(BMM_EINVAL, "mlp: null argument, no rows or no steps");
    if (rows > (1u << 24))
        return fail(BMM_EINVAL, "mlp: too many rows");
    BMM_TRY(ensure_cap(h, rows));
    BMM_CUDA_TRY(cudaMemcpyAsync(h->x, x, rows * kIn * 4, cudaMemcpyHostToDevice, h->stream));
    BMM_CUDA_TRY(cudaMemcpyAsync(h->t, target, rows * kOut * 4, cudaMemcpyHostToDevice, h->stream));
    for (int s = 0; s < steps; ++s)
        BMM_TRY(train_step_dev(h, h->x, 0, h->t, (int)rows));
    if (loss)
        BMM_CUDA_TRY(cudaMemcpyAsync(loss, h->loss, 4, cudaMemcpyDeviceToHost, h->stream));
    return check_err(h);
}

BMM_API int bmm_mlp_gemm(const float* A, const float* B, int M, int N, int K, float* C) {
    clear_error();
    if (!A || !B || !C || M <= 0 || N <= 0 || K <= 0)
        return fail(BMM_EINVAL, "mlp: bad gemm arguments");
    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws)
        return st;
    float *dA = nullptr, *dB = nullptr, *dC = nullptr;
    int* derr = nullptr;
    cudaError_t e = cudaMalloc(&dA, (size_t)M * K * 4);
    if (e == cudaSuccess)
        e = cudaMalloc(&dB, (size_t)N * K * 4);
    if (e == cudaSuccess)
        e = cudaMalloc(&dC, (size_t)M * N * 4);
    if (e == cudaSuccess)
        e = cudaMalloc(&derr, 4);
    int rc = BMM_OK;
    if (e == cudaSuccess)
        e = cudaMemcpy(dA, A, (size_t)M * K * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(dB, B, (size_t)N * K * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemset(derr, 0, 4);
    if (e != cudaSuccess) {
        cudaGetLastError();
        rc = fail(BMM_ECUDA, "mlp: gemm setup failed: %s", cudaGetErrorString(e));
    }
    if (rc == BMM_OK) {
        GemmArgs a = gemm_args(dA, 0, K, 1, dB, 0, K, 1, M, N, K, derr);
        a.out_f = dC;
        a.ldo_f = N;
        rc = gemm_launch(a, ws->stream);
    }
    int err = 0;
    if (rc == BMM_OK && (cudaMemcpyAsync(C, dC, (size_t)M * N * 4, cudaMemcpyDeviceToHost,
                                         ws->stream) != cudaSuccess ||
                         cudaMemcpyAsync(&err, derr, 4, cudaMemcpyDeviceToHost, ws->stream) !=
                             cudaSuccess ||
                         cudaStreamSynchronize(ws->stream) != cudaSuccess))
        rc = fail(BMM_ECUDA, "mlp: gemm failed: %s", cudaGetErrorString(cudaGetLastError()));
    if (rc == BMM_OK && err)
        rc = fail(BMM_ETIMEOUT, "mlp: a tensor-core wait timed out");
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dC);
    cudaFree(derr);
    return rc;
}

}  // extern "C"
