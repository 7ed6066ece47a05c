// Batched per-target searches over thousands of uneven instances in one
// persistent launch.
//
// Every row of every instance is an item: target row i of an n-row instance
// against the k others (i + 1 + j) mod n, j < k (the reference window search
// over [i, i+1..i+k], restricted to masks with bit 0 set).  The host plan
// lists the items longest-first; one persistent grid (one 512-thread CTA per
// SM, 128 KB of shared memory) pulls them from a global atomic counter and
// solves each with the method the autotuner chose for its shape:
//   FWHT16     k = 16: packed int16x2 transform of the signed histogram,
//   FWHT_SMALL k < 16: int32 transform in shared memory,
//   GRAY       narrow rows (W <= 8 words): direct reflected-Gray enumeration.
// The counter reset and the kernel are captured once into a CUDA graph and
// replayed (re-captured only when the device pointers change).
#include "common.cuh"
#include "target_item.cuh"

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

namespace bmm {
namespace {

constexpr int kThreads = item::kFwht16Threads;  // 512
constexpr int kGrayWords = 8;                   // GRAY items hold rows of <= 8 words

// kGray + log2(words per row, rounded up to 1, 2, 4 or 8)
enum Method : uint32_t { kFwht16 = 0, kFwhtSmall = 1, kGray = 2 };

struct BatchPolicy {
    // k = 16 items with W <= this use GRAY.  0: the packed transform for every
    // k = 16 item -- on B200 it beats the Gray enumeration at every row width
    // up to 8 words (C4 batch: 15.1 ms against 21.5 ms with a 4-word
    // crossover; bmmpy_b200.autotune measures it per device).
    int gray_max_words = 0;
    int force = -1;          // -1: policy; else every item uses this method where legal
};
BatchPolicy g_policy;
std::mutex g_policy_mu;

struct Cyclic {
    uint32_t row, n;
    __device__ __forceinline__ uint32_t operator()(int j) const {
        uint32_t r = row + 1 + (uint32_t)j;
        return r >= n ? r - n : r;  // k < n, so one wrap at most
    }
};

__global__ void __launch_bounds__(kThreads, 1)
    batch_kernel(const uint64_t* __restrict__ words, const bmm_instance* __restrict__ inst,
                 const uint64_t* __restrict__ items, long long n_items,
                 unsigned long long* __restrict__ counter, uint64_t* __restrict__ best_mask,
                 uint32_t* __restrict__ best_weight) {
    extern __shared__ __align__(16) int32_t P[];  // 128 KB
    __shared__ uint32_t red32[kThreads / 32];
    __shared__ unsigned long long red64[kThreads / 32];
    __shared__ long long s_item;
    for (;;) {
        if (threadIdx.x == 0)
            s_item = (long long)atomicAdd(counter, 1ull);
        __syncthreads();
        const long long it = s_item;
        __syncthreads();
        if (it >= n_items)
            break;
        const uint64_t code = items[it];
        const bmm_instance d = inst[(uint32_t)code];
        const uint32_t row = (uint32_t)((code >> 32) & 0xffffu);
        const uint32_t method = (uint32_t)(code >> 48);
        const uint64_t* base = words + d.word_offset;
        const Cyclic others{row, d.rows};
        uint64_t* om = best_mask + d.out_offset + row;
        uint32_t* ow = best_weight + d.out_offset + row;
        if (method == kFwht16) {
            item::fwht16(P, red32, base, (int)d.stride, (int)d.cols, others, row, om, ow);
        } else if (method == kFwhtSmall) {
            item::fwht_small(P, red64, base, (int)d.stride, (int)d.cols, others, (int)d.k, row, om,
                             ow);
        } else {
            uint64_t* srow = reinterpret_cast<uint64_t*>(P);
            const int W = (int)((d.cols + 63) / 64);
            switch (method - kGray) {
            case 0:
                item::gray<1>(srow, red64, base, (int)d.stride, W, others, (int)d.k, row, om, ow);
                break;
            case 1:
                item::gray<2>(srow, red64, base, (int)d.stride, W, others, (int)d.k, row, om, ow);
                break;
            case 2:
                item::gray<4>(srow, red64, base, (int)d.stride, W, others, (int)d.k, row, om, ow);
                break;
            default:
                item::gray<8>(srow, red64, base, (int)d.stride, W, others, (int)d.k, row, om, ow);
                break;
            }
        }
        __syncthreads();
    }
}

}  // namespace
}  // namespace bmm

using namespace bmm;

struct bmm_batch {
    int device = -1;
    long long n_items = 0;
    size_t n_inst = 0;
    size_t n_out = 0;
    bmm_instance* d_inst = nullptr;
    uint64_t* d_items = nullptr;
    unsigned long long* d_counter = nullptr;
    cudaStream_t capture_stream = nullptr;
    cudaGraphExec_t exec = nullptr;
    const void* bound[3] = {nullptr, nullptr, nullptr};  // words, mask, weight of the graph
    int grid = 0;
    int methods[3] = {0, 0, 0};
};

namespace {

int gray_code(uint32_t W) { return kGray + (W <= 1 ? 0 : W <= 2 ? 1 : W <= 4 ? 2 : 3); }

int method_for(const bmm_instance& d, const BatchPolicy& pol) {
    const uint32_t W = (d.cols + 63) / 64;
    const bool gray_ok = W <= (uint32_t)kGrayWords;
    const bool fwht_ok = d.cols <= 32767;
    if (pol.force == kGray && gray_ok)
        return gray_code(W);
    if (pol.force == kFwht16 || pol.force == kFwhtSmall) {
        if (fwht_ok)
            return d.k == 16 ? kFwht16 : kFwhtSmall;
    }
    if (gray_ok && (int)W <= pol.gray_max_words)
        return gray_code(W);
    if (fwht_ok)
        return d.k == 16 ? kFwht16 : kFwhtSmall;
    return gray_ok ? gray_code(W) : -1;
}

// Relative cost of one item, for longest-first ordering.
double item_cost(const bmm_instance& d, int method) {
    const double states = (double)(1u << d.k);
    if (method == kFwht16)
        return 1.0 + d.cols / 16384.0;
    if (method == kFwhtSmall)
        return states / 65536.0 * d.k / 16.0 + d.cols / 16384.0;
    return states / 65536.0 * (double)(1 << (method - kGray)) * 0.3;
}

int destroy_batch(bmm_batch* b) {
    if (!b)
        return BMM_OK;
    int prev = -1;
    cudaGetDevice(&prev);
    if (b->device >= 0)
        cudaSetDevice(b->device);
    if (b->exec)
        cudaGraphExecDestroy(b->exec);
    if (b->capture_stream)
        cudaStreamDestroy(b->capture_stream);
    cudaFree(b->d_inst);
    cudaFree(b->d_items);
    cudaFree(b->d_counter);
    if (prev >= 0)
        cudaSetDevice(prev);
    delete b;
    return BMM_OK;
}

}  // namespace

extern "C" {

BMM_API int bmm_batch_policy(int gray_max_words, int force_method) {
    clear_error();
    if (gray_max_words < 0 || gray_max_words > kGrayWords)
        return fail(BMM_EINVAL, "batch policy: gray_max_words must be in [0, %d]", kGrayWords);
    if (force_method < -1 || force_method > 2)
        return fail(BMM_EINVAL, "batch policy: force_method must be -1, 0, 1 or 2");
    std::lock_guard<std::mutex> lock(g_policy_mu);
    g_policy.gray_max_words = gray_max_words;
    g_policy.force = force_method;
    return BMM_OK;
}

BMM_API int bmm_batch_create(const bmm_instance* inst, size_t n_inst, bmm_batch** out) {
    clear_error();
    if (!out)
        return fail(BMM_EINVAL, "batch: null output");
    *out = nullptr;
    if (n_inst && !inst)
        return fail(BMM_EINVAL, "batch: null instance list");
    if (n_inst > 0xffffffffull)
        return fail(BMM_EINVAL, "batch: too many instances");
    BatchPolicy pol;
    {
        std::lock_guard<std::mutex> lock(g_policy_mu);
        pol = g_policy;
    }
    std::vector<std::pair<double, uint64_t>> order;
    size_t n_out = 0;
    int methods[3] = {0, 0, 0};
    for (size_t i = 0; i < n_inst; ++i) {
        const bmm_instance& d = inst[i];
        const uint32_t W = (d.cols + 63) / 64;
        if (d.rows < 2 || d.rows > 65535)
            return fail(BMM_EINVAL, "batch: instance %zu must have 2..65535 rows", i);
        if (d.k < 1 || d.k > 16 || d.k >= d.rows)
            return fail(BMM_EINVAL, "batch: instance %zu needs 1 <= k <= min(16, rows - 1)", i);
        if (W > d.stride)
            return fail(BMM_EINVAL, "batch: instance %zu stride is smaller than its row width", i);
        const int m = method_for(d, pol);
        if (m < 0)
            return fail(BMM_EINVAL, "batch: instance %zu has %u columns (> 32767 and > 512)", i,
                        d.cols);
        ++methods[m >= kGray ? kGray : m];
        const double c = item_cost(d, m);
        for (uint32_t r = 0; r < d.rows; ++r)
            order.emplace_back(c, (uint64_t)i | ((uint64_t)r << 32) | ((uint64_t)m << 48));
        n_out = std::max<size_t>(n_out, (size_t)d.out_offset + d.rows);
    }
    std::stable_sort(order.begin(), order.end(),
                     [](const auto& a, const auto& b) { return a.first > b.first; });
    std::vector<uint64_t> items(order.size());
    for (size_t i = 0; i < order.size(); ++i)
        items[i] = order[i].second;

    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws)
        return st;
    bmm_batch* b = new bmm_batch();
    b->device = ws->device;
    b->n_items = (long long)items.size();
    b->n_inst = n_inst;
    b->n_out = n_out;
    std::memcpy(b->methods, methods, sizeof(methods));
    b->grid = ws->sm_count;
    cudaError_t e = cudaMalloc(&b->d_inst, std::max<size_t>(n_inst, 1) * sizeof(bmm_instance));
    if (e == cudaSuccess)
        e = cudaMalloc(&b->d_items, std::max<size_t>(items.size(), 1) * 8);
    if (e == cudaSuccess)
        e = cudaMalloc(&b->d_counter, 8);
    if (e == cudaSuccess && n_inst)
        e = cudaMemcpy(b->d_inst, inst, n_inst * sizeof(bmm_instance), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !items.empty())
        e = cudaMemcpy(b->d_items, items.data(), items.size() * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 32768 * 4);
    if (e != cudaSuccess) {
        destroy_batch(b);
        return fail(BMM_ECUDA, "batch: setup failed: %s", cudaGetErrorString(e));
    }
    *out = b;
    return BMM_OK;
}

BMM_API int bmm_batch_info(const bmm_batch* b, long long* n_items, size_t* n_out, int* methods3) {
    if (!b)
        return fail(BMM_EINVAL, "batch: null handle");
    if (n_items)
        *n_items = b->n_items;
    if (n_out)
        *n_out = b->n_out;
    if (methods3)
        std::memcpy(methods3, b->methods, sizeof(b->methods));
    return BMM_OK;
}

BMM_API int bmm_batch_run(bmm_batch* b, const uint64_t* d_words, uint64_t* d_best_mask,
                          uint32_t* d_best_weight, void* stream) {
    clear_error();
    if (!b)
        return fail(BMM_EINVAL, "batch: null handle");
    if (b->n_items == 0)
        return BMM_OK;
    int dev = -1;
    BMM_CUDA_TRY(cudaGetDevice(&dev));
    if (dev != b->device)
        return fail(BMM_EINVAL, "batch: created on device %d, run on device %d", b->device, dev);
    if (!b->exec || b->bound[0] != d_words || b->bound[1] != d_best_mask ||
        b->bound[2] != d_best_weight) {
        if (b->exec) {
            cudaGraphExecDestroy(b->exec);
            b->exec = nullptr;
        }
        cudaGraph_t graph = nullptr;
        BMM_CUDA_TRY(cudaStreamBeginCapture(b->capture_stream, cudaStreamCaptureModeThreadLocal));
        cudaMemsetAsync(b->d_counter, 0, 8, b->capture_stream);
        batch_kernel<<<b->grid, kThreads, 32768 * 4, b->capture_stream>>>(
            d_words, b->d_inst, b->d_items, b->n_items, b->d_counter, d_best_mask, d_best_weight);
        const cudaError_t le = cudaGetLastError();
        const cudaError_t ce = cudaStreamEndCapture(b->capture_stream, &graph);
        if (le != cudaSuccess || ce != cudaSuccess) {
            if (graph)
                cudaGraphDestroy(graph);
            return fail(BMM_ECUDA, "batch: graph capture failed: %s",
                        cudaGetErrorString(le != cudaSuccess ? le : ce));
        }
        const cudaError_t ie = cudaGraphInstantiate(&b->exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) {
            b->exec = nullptr;
            return fail(BMM_ECUDA, "batch: graph instantiation failed: %s", cudaGetErrorString(ie));
        }
        b->bound[0] = d_words;
        b->bound[1] = d_best_mask;
        b->bound[2] = d_best_weight;
    }
    BMM_CUDA_TRY(cudaGraphLaunch(b->exec, (cudaStream_t)stream));
    return BMM_OK;
}

BMM_API int bmm_batch_destroy(bmm_batch* b) { return destroy_batch(b); }

BMM_API int bmm_batch_targets(const uint64_t* words, size_t n_words, const bmm_instance* inst,
                              size_t n_inst, uint64_t* best_mask, uint32_t* best_weight) {
    clear_error();
    if (n_inst == 0)
        return BMM_OK;
    if (!words || !inst || !best_mask || !best_weight)
        return fail(BMM_EINVAL, "batch: null argument");
    for (size_t i = 0; i < n_inst; ++i)
        if (inst[i].word_offset + (uint64_t)inst[i].rows * inst[i].stride > n_words)
            return fail(BMM_EINVAL, "batch: instance %zu extends past the word buffer", i);
    bmm_batch* b = nullptr;
    BMM_TRY(bmm_batch_create(inst, n_inst, &b));
    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws) {
        destroy_batch(b);
        return st;
    }
    void *d_words = nullptr, *d_m = nullptr, *d_w = nullptr;
    int rc = ws_buffer(ws, kSlotRows, n_words * 8, &d_words);
    if (rc == BMM_OK)
        rc = ws_buffer(ws, kSlotOut, b->n_out * 8, &d_m);
    if (rc == BMM_OK)
        rc = ws_buffer(ws, kSlotExtra0, b->n_out * 4, &d_w);
    if (rc == BMM_OK && cudaMemcpyAsync(d_words, words, n_words * 8, cudaMemcpyHostToDevice,
                                        ws->stream) != cudaSuccess)
        rc = fail(BMM_ECUDA, "batch: upload failed");
    if (rc == BMM_OK)
        rc = bmm_batch_run(b, (const uint64_t*)d_words, (uint64_t*)d_m, (uint32_t*)d_w, ws->stream);
    if (rc == BMM_OK &&
        (cudaMemcpyAsync(best_mask, d_m, b->n_out * 8, cudaMemcpyDeviceToHost, ws->stream) !=
             cudaSuccess ||
         cudaMemcpyAsync(best_weight, d_w, b->n_out * 4, cudaMemcpyDeviceToHost, ws->stream) !=
             cudaSuccess ||
         cudaStreamSynchronize(ws->stream) != cudaSuccess))
        rc = fail(BMM_ECUDA, "batch: download failed: %s", cudaGetErrorString(cudaGetLastError()));
    destroy_batch(b);
    return rc;
}

}  // extern "C"
