// extern "C" entry points (include/bmm_b200.h): argument validation with the
// reference's error classes, the per-thread device workspace, host<->device
// staging, and dispatch to the kernels.
#include "common.cuh"
#include "fwht.cuh"
#include "gray.cuh"
#include "spectrum.cuh"
#include "topk.cuh"

#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

namespace bmm {

namespace {
thread_local char g_err[512] = "";

struct ThreadWorkspaces {
    std::vector<Workspace*> per_device;
    ~ThreadWorkspaces() {
        for (Workspace* ws : per_device) {
            if (!ws)
                continue;
            // The process may be tearing down the CUDA context already; ignore errors.
            int prev = -1;
            if (cudaGetDevice(&prev) == cudaSuccess && cudaSetDevice(ws->device) == cudaSuccess) {
                for (int i = 0; i < kSlotCount; ++i)
                    if (ws->buf[i])
                        cudaFree(ws->buf[i]);
                if (ws->pinned)
                    cudaFreeHost(ws->pinned);
                if (ws->stream)
                    cudaStreamDestroy(ws->stream);
                cudaSetDevice(prev);
            }
            delete ws;
        }
    }
};
thread_local ThreadWorkspaces g_ws;
}  // namespace

int fail(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

void clear_error() { g_err[0] = 0; }

Workspace* workspace(int* status) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        *status = fail(BMM_ENODEV, "no CUDA device is available: %s", cudaGetErrorString(e));
        return nullptr;
    }
    if ((int)g_ws.per_device.size() <= dev)
        g_ws.per_device.resize(dev + 1, nullptr);
    Workspace*& ws = g_ws.per_device[dev];
    if (!ws) {
        Workspace* w = new Workspace();
        w->device = dev;
        cudaDeviceProp prop{};
        e = cudaGetDeviceProperties(&prop, dev);
        if (e == cudaSuccess)
            e = cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            delete w;
            *status = fail(BMM_ECUDA, "device setup failed: %s", cudaGetErrorString(e));
            return nullptr;
        }
        w->sm_count = prop.multiProcessorCount;
        w->smem_optin = (int)prop.sharedMemPerBlockOptin;
        ws = w;
    }
    *status = BMM_OK;
    return ws;
}

int ws_buffer(Workspace* ws, int slot, size_t bytes, void** out) {
    if (bytes == 0)
        bytes = 16;
    if (ws->cap[slot] < bytes) {
        if (ws->buf[slot]) {
            cudaFree(ws->buf[slot]);
            ws->buf[slot] = nullptr;
            ws->cap[slot] = 0;
        }
        size_t cap = 256;
        while (cap < bytes)
            cap *= 2;
        cudaError_t e = cudaMalloc(&ws->buf[slot], cap);
        if (e != cudaSuccess) {
            ws->buf[slot] = nullptr;
            return fail(e == cudaErrorMemoryAllocation ? BMM_ENOMEM : BMM_ECUDA,
                        "device allocation of %zu bytes failed: %s", cap, cudaGetErrorString(e));
        }
        ws->cap[slot] = cap;
    }
    *out = ws->buf[slot];
    return BMM_OK;
}

int ws_pinned(Workspace* ws, size_t bytes, void** out) {
    if (ws->pinned_cap < bytes) {
        if (ws->pinned)
            cudaFreeHost(ws->pinned);
        ws->pinned = nullptr;
        ws->pinned_cap = 0;
        size_t cap = 4096;
        while (cap < bytes)
            cap *= 2;
        BMM_CUDA_TRY(cudaMallocHost(&ws->pinned, cap));
        ws->pinned_cap = cap;
    }
    *out = ws->pinned;
    return BMM_OK;
}

int merge_topk_lists(const bmm_candidate* d_lists, int nlists, int kk, bmm_candidate* d_out,
                     cudaStream_t stream, const unsigned* d_limit) {
    auto run = [&](auto Ec) -> int {
        constexpr int E = decltype(Ec)::value;
        auto mk = merge_lists_kernel<E>;
        // every warp stages a 32*E list in shared memory: keep that under 128 KB
        const int warps = E >= 32 ? 8 : 32;
        const size_t msmem = (size_t)warps * 32 * E * sizeof(bmm_candidate);
        BMM_CUDA_TRY(
            cudaFuncSetAttribute(mk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)msmem));
        mk<<<1, warps * 32, msmem, stream>>>(d_lists, nlists, kk, d_out, d_limit);
        BMM_CUDA_TRY(cudaGetLastError());
        return BMM_OK;
    };
    if (kk <= 32)
        return run(std::integral_constant<int, 1>{});
    if (kk <= 128)
        return run(std::integral_constant<int, 4>{});
    if (kk <= 1024)
        return run(std::integral_constant<int, 32>{});
    return fail(BMM_EINVAL, "k must be <= 1024");
}

namespace {

// Pack the window rows (host) contiguously: t x W words.
std::vector<uint64_t> pack_window(const uint64_t* words, size_t stride, size_t W,
                                  const uint32_t* win, size_t t) {
    std::vector<uint64_t> out(t * W);
    for (size_t r = 0; r < t; ++r)
        std::memcpy(out.data() + r * W, words + (size_t)win[r] * stride, W * sizeof(uint64_t));
    return out;
}

int check_window(const uint64_t* words, size_t stride, size_t cols, const uint32_t* win, size_t t,
                 const char* who) {
    if (t > 64)
        return fail(BMM_EINVAL, "%s: window_rows size must be <= 64", who);
    if (t && (!words || !win))
        return fail(BMM_EINVAL, "%s: null matrix or window", who);
    const size_t W = (cols + 63) / 64;
    if (W > stride)
        return fail(BMM_EINVAL, "%s: stride %zu is smaller than %zu words per row", who, stride, W);
    // unique rows (RowWindow::initialize, src/core/row_window.cpp:119-137)
    for (size_t i = 0; i < t; ++i)
        for (size_t j = i + 1; j < t; ++j)
            if (win[i] == win[j])
                return fail(BMM_EINVAL, "%s: window rows must be unique", who);
    return BMM_OK;
}

// Copy kk device candidates back and compact away empty entries.
int finish_candidates(Workspace* ws, const bmm_candidate* d_out, size_t kk, bmm_candidate* out,
                      size_t* out_count) {
    std::vector<bmm_candidate> h(kk);
    BMM_CUDA_TRY(cudaMemcpyAsync(h.data(), d_out, kk * sizeof(bmm_candidate),
                                 cudaMemcpyDeviceToHost, ws->stream));
    BMM_CUDA_TRY(cudaStreamSynchronize(ws->stream));
    size_t n = 0;
    for (size_t i = 0; i < kk; ++i)
        if (h[i].weight != 0xffffffffu)
            out[n++] = h[i];
    *out_count = n;
    return BMM_OK;
}

int upload(Workspace* ws, int slot, const void* host, size_t bytes, void** dev) {
    BMM_TRY(ws_buffer(ws, slot, bytes, dev));
    if (bytes)
        BMM_CUDA_TRY(cudaMemcpyAsync(*dev, host, bytes, cudaMemcpyHostToDevice, ws->stream));
    return BMM_OK;
}

int fwht_size_log(size_t n, int* t) {
    if (n <= 1) {
        *t = 0;
        return BMM_OK;
    }
    if (n & (n - 1))
        return fail(BMM_EINVAL, "fwht_inplace: size must be a power of two");
    int l = 0;
    while (((size_t)1 << l) < n)
        ++l;
    if (l > 34)
        return fail(BMM_EINVAL, "fwht_inplace: size too large");
    *t = l;
    return BMM_OK;
}

template <typename T>
int fwht_host(T* data, size_t n) {
    clear_error();
    int t = 0;
    BMM_TRY(fwht_size_log(n, &t));
    if (t == 0)
        return BMM_OK;
    if (!data)
        return fail(BMM_EINVAL, "fwht_inplace: null data");
    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws)
        return st;
    void* d = nullptr;
    BMM_TRY(upload(ws, kSlotSpec, data, n * sizeof(T), &d));
    if (sizeof(T) == 4 && t >= 14)
        BMM_TRY(spectrum_dense_fwht(ws, (int32_t*)d, t, ws->stream));
    else
        BMM_TRY(fwht_global_launch<T>(ws, (T*)d, t, ws->stream));
    BMM_CUDA_TRY(cudaMemcpyAsync(data, d, n * sizeof(T), cudaMemcpyDeviceToHost, ws->stream));
    BMM_CUDA_TRY(cudaStreamSynchronize(ws->stream));
    return BMM_OK;
}

}  // namespace
}  // namespace bmm

using namespace bmm;

extern "C" {

uint64_t bmm_gen_instance(uint64_t* words, size_t rows, size_t cols, size_t stride, double p,
                          uint64_t seed, size_t scrambles) {
    uint64_t st = seed == 0 ? 0x9E3779B97F4A7C15ull : seed;
    auto next = [&st]() {
        st ^= st << 13;
        st ^= st >> 7;
        st ^= st << 17;
        return st;
    };
    std::memset(words, 0, rows * stride * sizeof(uint64_t));
    uint64_t planted = 0;
    for (size_t r = 0; r < rows; ++r)
        for (size_t c = 0; c < cols; ++c)
            if ((double)(next() >> 11) * (1.0 / 9007199254740992.0) < p) {
                words[r * stride + c / 64] |= 1ull << (c % 64);
                ++planted;
            }
    if (rows < 2)
        return planted;
    for (size_t s = 0; s < scrambles; ++s) {
        const size_t i = (size_t)(next() % rows);
        size_t j = (size_t)(next() % rows);
        while (j == i)
            j = (size_t)(next() % rows);
        for (size_t w = 0; w < stride; ++w)
            words[i * stride + w] ^= words[j * stride + w];
    }
    return planted;
}

int bmm_gray_tune(int hs_blocks, int chunk_bits) {
    clear_error();
    if (hs_blocks < -1 || hs_blocks > 8 || hs_blocks == 1 || hs_blocks == 7)
        return fail(BMM_EINVAL, "gray tuning: hs_blocks must be -1, 0, 2-6 or 8");
    if (chunk_bits < -1 || chunk_bits > 31)
        return fail(BMM_EINVAL, "gray tuning: chunk_bits must be -1 or in [0, 31]");
    g_gray_tuning.hs_blocks = hs_blocks;
    g_gray_tuning.chunk_bits = chunk_bits;
    return BMM_OK;
}

int bmm_gray_tune_lanes(int lanes) {
    clear_error();
    if (lanes != -1 && lanes != 1 && lanes != 2)
        return fail(BMM_EINVAL, "gray tuning: lanes must be -1, 1 or 2");
    g_gray_tuning.lanes = lanes;
    return BMM_OK;
}

int bmm_gray_tune_shape(size_t words_per_row, size_t k, int hs_blocks, int chunk_bits,
                        int lanes) {
    clear_error();
    if (words_per_row == 0 || k == 0 || k > 40)
        return fail(BMM_EINVAL, "gray tuning: words_per_row must be > 0 and k in [1, 40]");
    if (hs_blocks < -1 || hs_blocks > 8 || hs_blocks == 1 || hs_blocks == 7)
        return fail(BMM_EINVAL, "gray tuning: hs_blocks must be -1, 0, 2-6 or 8");
    if (chunk_bits < -1 || chunk_bits > 31)
        return fail(BMM_EINVAL, "gray tuning: chunk_bits must be -1 or in [0, 31]");
    if (lanes != -1 && lanes != 1 && lanes != 2)
        return fail(BMM_EINVAL, "gray tuning: lanes must be -1, 1 or 2");
    if (lanes == 2 && hs_blocks > 4)
        return fail(BMM_EINVAL, "gray tuning: 32-word lanes take at most 4 carry-save blocks");
    GrayTuning t;
    t.hs_blocks = hs_blocks;
    t.chunk_bits = chunk_bits;
    t.lanes = lanes;
    return gray_tune_shape(words_per_row, (int)k, t);
}

int bmm_spectrum_tune_shape(size_t t, int low_bits) {
    clear_error();
    if (t < 15 || t > 40)
        return fail(BMM_EINVAL, "spectrum tuning: t must be in [15, 40]");
    if (low_bits != -1 && (low_bits < 14 || low_bits > (int)(t < 33 ? t : 33)))
        return fail(BMM_EINVAL, "spectrum tuning: low_bits must be -1 or in [14, min(t, 33)]");
    g_spectrum_shape_low_bits[t] = low_bits;
    return BMM_OK;
}

int bmm_tune_reset(void) {
    clear_error();
    gray_tune_reset();
    for (int& v : g_spectrum_shape_low_bits)
        v = -1;
    g_spectrum_low_bits = -1;
    return BMM_OK;
}

int bmm_probe_xor_popc(double* words_per_second) {
    clear_error();
    if (!words_per_second)
        return fail(BMM_EINVAL, "null output");
    return popc_probe(words_per_second);
}

const char* bmm_last_error(void) { return g_err; }

const char* bmm_version(void) { return "0.5.3+b200"; }

int bmm_runtime_features(bmm_features* out) {
    if (!out)
        return fail(BMM_EINVAL, "null output");
    std::memset(out, 0, sizeof(*out));
    out->cuda_compiled = 1;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess)
        n = 0;
    out->device_count = n;
    out->cuda_available = n > 0;
    if (n > 0) {
        int dev = 0;
        cudaDeviceProp prop{};
        if (cudaGetDevice(&dev) == cudaSuccess && cudaGetDeviceProperties(&prop, dev) == cudaSuccess) {
            out->sm_count = prop.multiProcessorCount;
            out->cc_major = prop.major;
            out->cc_minor = prop.minor;
            std::snprintf(out->device_name, sizeof(out->device_name), "%s", prop.name);
        }
    }
    return BMM_OK;
}

int bmm_fwht_i32(int32_t* data, size_t n) { return fwht_host(data, n); }
int bmm_fwht_i16(int16_t* data, size_t n) { return fwht_host(data, n); }

int bmm_fwht_i32_dev(int32_t* d_data, size_t n, void* stream) {
    clear_error();
    int t = 0;
    BMM_TRY(fwht_size_log(n, &t));
    if (t == 0)
        return BMM_OK;
    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws)
        return st;
    if (t >= 14)
        return spectrum_dense_fwht(ws, d_data, t, (cudaStream_t)stream);
    return fwht_global_launch<int32_t>(ws, d_data, t, (cudaStream_t)stream);
}

// ---- window searches -------------------------------------------------------
int bmm_fwht_search(const uint64_t* words, size_t stride, size_t cols, const uint32_t* win,
                    size_t t, size_t max_rows, size_t k, bmm_candidate* out, size_t* out_count) {
    clear_error();
    if (!out_count)
        return fail(BMM_EINVAL, "FwhtSearch: null out_count");
    *out_count = 0;
    // src/search/fwht_search.cpp:36-46
    if (t == 0 || t > max_rows || k == 0)
        return BMM_OK;
    if (t > 64)
        return fail(BMM_EINVAL, "FwhtSearch: window_rows size must be <= 64");
    if (t > 33)
        return fail(BMM_EINVAL, "FwhtSearch: window_rows size %zu exceeds the 2^33-bucket device "
                                "spectrum limit", t);
    BMM_TRY(check_window(words, stride, cols, win, t, "FwhtSearch"));
    const size_t W = (cols + 63) / 64;
    if (W == 0)
        return BMM_OK;
    if (cols > 0x7fffffffull)
        return fail(BMM_EOVERFLOW, "FwhtSearch: total weight exceeds int32 range");
    const size_t n = (size_t)1 << t;
    size_t kk = k < n - 1 ? k : n - 1;
    if (kk > 1024)
        return fail(BMM_EINVAL, "FwhtSearch: max_candidates above 1024 is not supported on the "
                                "device (requested %zu)", k);
    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws)
        return st;
    const std::vector<uint64_t> packed = pack_window(words, stride, W, win, t);
    void *d_rows = nullptr, *d_out = nullptr;
    BMM_TRY(upload(ws, kSlotRows, packed.data(), packed.size() * 8, &d_rows));
    BMM_TRY(ws_buffer(ws, kSlotOut, kk * sizeof(bmm_candidate), &d_out));
    BMM_TRY(spectrum_topk_launch(ws, (const uint64_t*)d_rows, (int)t, (int)W, (long long)cols,
                                 (int)kk, (bmm_candidate*)d_out, ws->stream));
    return finish_candidates(ws, (bmm_candidate*)d_out, kk, out, out_count);
}

int bmm_mitm_search(const uint64_t* words, size_t stride, size_t cols, const uint32_t* win,
                    size_t t, size_t k, size_t low_bits, bmm_candidate* out, size_t* out_count) {
    clear_error();
    if (!out_count)
        return fail(BMM_EINVAL, "MitmFwhtSearch: null out_count");
    *out_count = 0;
    // src/search/mitm_fwht_search.cpp:270-289
    if (k == 0 || t == 0)
        return BMM_OK;
    if (t > 64)
        return fail(BMM_EINVAL, "MitmFwhtSearch: window_rows size must be <= 64");
    if (t > 40)
        return fail(BMM_EINVAL, "MitmFwhtSearch: 2^%zu combinations cannot be enumerated", t);
    if (low_bits != 0 && low_bits >= t)
        return fail(BMM_EINVAL, "MitmFwhtSearch: low_bits must be in [1, t - 1] or 0 for auto");
    BMM_TRY(check_window(words, stride, cols, win, t, "MitmFwhtSearch"));
    const size_t W = (cols + 63) / 64;
    if (W == 0)
        return BMM_OK;
    if (cols > 0x7fffffffull)
        return fail(BMM_EOVERFLOW, "build_compact_split_window: total weight exceeds int32 range");
    const size_t states = ((size_t)1 << t) - 1;
    const size_t kk = k < states ? k : states;
    if (kk > 1024)
        return fail(BMM_EINVAL, "MitmFwhtSearch: max_candidates above 1024 is not supported on "
                                "the device (requested %zu)", k);
    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws)
        return st;
    const std::vector<uint64_t> packed = pack_window(words, stride, W, win, t);
    void *d_rows = nullptr, *d_out = nullptr;
    BMM_TRY(upload(ws, kSlotRows, packed.data(), packed.size() * 8, &d_rows));
    BMM_TRY(ws_buffer(ws, kSlotOut, kk * sizeof(bmm_candidate), &d_out));
    BMM_TRY(spectrum_topk_launch(ws, (const uint64_t*)d_rows, (int)t, (int)W, (long long)cols,
                                 (int)kk, (bmm_candidate*)d_out, ws->stream));
    return finish_candidates(ws, (bmm_candidate*)d_out, kk, out, out_count);
}

int bmm_gray_search(const uint64_t* words, size_t stride, size_t cols, const uint32_t* win,
                    size_t t, size_t k, size_t chunk_bits, bmm_candidate* out,
                    size_t* out_count) {
    clear_error();
    if (!out_count)
        return fail(BMM_EINVAL, "BruteforceSearch: null out_count");
    *out_count = 0;
    // src/search/bruteforce_search.cpp:300-319
    if (k == 0 || t == 0)
        return BMM_OK;
    BMM_TRY(check_window(words, stride, cols, win, t, "BruteforceSearch"));
    const size_t W = (cols + 63) / 64;
    if (W == 0)
        return BMM_OK;
    if (cols > 0xffffffffull)
        return fail(BMM_EOVERFLOW, "BruteforceSearch: window width exceeds candidate weight range");
    size_t chunk = chunk_bits;
    if (chunk != 0 && (chunk > t || chunk >= 64))
        return fail(BMM_EINVAL,
                    "BruteforceSearch: chunk_bits must be in [1, min(t, 63)] or 0 for auto");
    if (t > 44)
        return fail(BMM_EINVAL, "BruteforceSearch: 2^%zu combinations cannot be enumerated", t);
    const size_t states = (t >= 63) ? ~(size_t)0 : (((size_t)1 << t) - 1);
    const size_t kk = k < states ? k : states;
    if (kk > 1024)
        return fail(BMM_EINVAL, "BruteforceSearch: max_candidates above 1024 is not supported on "
                                "the device (requested %zu)", k);
    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws)
        return st;
    int lanes = 1;
    {
        size_t G = 1;
        while (G * 64 < W)
            G *= 2;
        lanes = (int)G;
    }
    if (chunk == 0)
        chunk = (size_t)auto_chunk_bits((int)t, lanes, ws->sm_count, 1);
    if (chunk > 31)
        chunk = 31;  // a single lane sweeps at most 2^31 states; the rest become prefixes
    const std::vector<uint64_t> packed = pack_window(words, stride, W, win, t);
    void *d_rows = nullptr, *d_out = nullptr;
    BMM_TRY(upload(ws, kSlotRows, packed.data(), packed.size() * 8, &d_rows));
    BMM_TRY(ws_buffer(ws, kSlotOut, kk * sizeof(bmm_candidate), &d_out));
    BMM_TRY(gray_window_launch(ws, (const uint64_t*)d_rows, (int)t, (int)W, (int)chunk, (int)kk,
                               (bmm_candidate*)d_out, ws->stream));
    return finish_candidates(ws, (bmm_candidate*)d_out, kk, out, out_count);
}

// ---- per-target ------------------------------------------------------------
static int check_targets(size_t rows, size_t stride, size_t cols, const uint32_t* targets,
                         const uint32_t* others, size_t n_targets, size_t k, const char* who) {
    const size_t W = (cols + 63) / 64;
    if (W > stride)
        return fail(BMM_EINVAL, "%s: stride smaller than the row width", who);
    for (size_t i = 0; i < n_targets; ++i) {
        if (targets[i] >= rows)
            return fail(BMM_EINVAL, "%s: target row out of range", who);
        for (size_t j = 0; j < k; ++j) {
            const uint32_t o = others[i * k + j];
            if (o >= rows)
                return fail(BMM_EINVAL, "%s: other row out of range", who);
            if (o == targets[i])
                return fail(BMM_EINVAL, "%s: the target cannot be one of its own others", who);
        }
    }
    return BMM_OK;
}

static int gray_targets_common(Workspace* ws, const uint64_t* d_words, size_t rows, size_t stride,
                               size_t cols, const uint32_t* d_targets, const uint32_t* d_others,
                               size_t n_targets, size_t k, int tiebreak, uint64_t* d_best_mask,
                               uint32_t* d_best_weight, cudaStream_t stream) {
    if (k < 1 || k > 40)
        return fail(BMM_EINVAL, "gray targets: k must be in [1, 40]");
    if ((cols + 63) / 64 > stride)
        return fail(BMM_EINVAL, "gray targets: stride smaller than the row width");
    if (cols >= (1ull << 24))
        return fail(BMM_EINVAL, "gray targets: cols must be < 2^24");
    const size_t W = (cols + 63) / 64;
    int lanes = 1;
    {
        size_t G = 1;
        while (G * 64 < W)
            G *= 2;
        lanes = (int)G;
    }
    int chunk = targets_chunk_bits((int)k, lanes, ws->sm_count, (int)n_targets);
    const GrayTuning tune = gray_tuning_for(W, (int)k);
    if (tune.chunk_bits > 0)
        chunk = tune.chunk_bits;
    if (chunk > (int)k)
        chunk = (int)k;
    void* d_keys = nullptr;
    BMM_TRY(ws_buffer(ws, kSlotKeys, n_targets * 8, &d_keys));
    return gray_targets_launch(ws, d_words, (int)stride, (int)W, d_targets, d_others,
                               (int)n_targets, (int)k, tiebreak, chunk,
                               (unsigned long long*)d_keys, d_best_mask, d_best_weight, stream);
}

int bmm_gray_targets_dev(const uint64_t* d_words, size_t rows, size_t stride, size_t cols,
                         const uint32_t* d_targets, const uint32_t* d_others, size_t n_targets,
                         size_t k, int tiebreak, uint64_t* d_best_mask, uint32_t* d_best_weight,
                         void* stream) {
    clear_error();
    if (n_targets == 0)
        return BMM_OK;
    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws)
        return st;
    return gray_targets_common(ws, d_words, rows, stride, cols, d_targets, d_others, n_targets, k,
                               tiebreak, d_best_mask, d_best_weight, (cudaStream_t)stream);
}

int bmm_gray_targets(const uint64_t* words, size_t rows, size_t stride, size_t cols,
                     const uint32_t* targets, const uint32_t* others, size_t n_targets, size_t k,
                     int tiebreak, uint64_t* best_mask, uint32_t* best_weight) {
    clear_error();
    if (n_targets == 0)
        return BMM_OK;
    if (!words || !targets || (k && !others) || !best_mask || !best_weight)
        return fail(BMM_EINVAL, "gray targets: null argument");
    BMM_TRY(check_targets(rows, stride, cols, targets, others, n_targets, k, "gray targets"));
    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws)
        return st;
    void *d_words = nullptr, *d_t = nullptr, *d_o = nullptr, *d_m = nullptr, *d_w = nullptr;
    BMM_TRY(upload(ws, kSlotRows, words, rows * stride * 8, &d_words));
    BMM_TRY(upload(ws, kSlotIdx, targets, n_targets * 4, &d_t));
    BMM_TRY(upload(ws, kSlotAux, others, n_targets * k * 4, &d_o));
    BMM_TRY(ws_buffer(ws, kSlotOut, n_targets * 8, &d_m));
    BMM_TRY(ws_buffer(ws, kSlotExtra0, n_targets * 4, &d_w));
    BMM_TRY(gray_targets_common(ws, (const uint64_t*)d_words, rows, stride, cols,
                                (const uint32_t*)d_t, (const uint32_t*)d_o, n_targets, k, tiebreak,
                                (uint64_t*)d_m, (uint32_t*)d_w, ws->stream));
    BMM_CUDA_TRY(cudaMemcpyAsync(best_mask, d_m, n_targets * 8, cudaMemcpyDeviceToHost, ws->stream));
    BMM_CUDA_TRY(
        cudaMemcpyAsync(best_weight, d_w, n_targets * 4, cudaMemcpyDeviceToHost, ws->stream));
    BMM_CUDA_TRY(cudaStreamSynchronize(ws->stream));
    return BMM_OK;
}

static int fwht_targets_check(size_t cols, size_t k) {
    if (k > 16)
        return fail(BMM_EINVAL, "fwht targets: k must be <= 16");
    if (cols > 32767)
        return fail(BMM_EINVAL, "fwht targets: cols must be <= 32767");
    return BMM_OK;
}

int bmm_fwht_targets_dev(const uint64_t* d_words, size_t rows, size_t stride, size_t cols,
                         const uint32_t* d_targets, const uint32_t* d_others, size_t n_targets,
                         size_t k, uint64_t* d_best_mask, uint32_t* d_best_weight, void* stream) {
    clear_error();
    (void)rows;
    if (n_targets == 0)
        return BMM_OK;
    BMM_TRY(fwht_targets_check(cols, k));
    if ((cols + 63) / 64 > stride)
        return fail(BMM_EINVAL, "fwht targets: stride smaller than the row width");
    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws)
        return st;
    return fwht_targets_launch(ws, d_words, (int)stride, (int)cols, d_targets, d_others,
                               (int)n_targets, (int)k, d_best_mask, d_best_weight,
                               (cudaStream_t)stream);
}

int bmm_fwht_targets(const uint64_t* words, size_t rows, size_t stride, size_t cols,
                     const uint32_t* targets, const uint32_t* others, size_t n_targets, size_t k,
                     uint64_t* best_mask, uint32_t* best_weight) {
    clear_error();
    if (n_targets == 0)
        return BMM_OK;
    if (!words || !targets || (k && !others) || !best_mask || !best_weight)
        return fail(BMM_EINVAL, "fwht targets: null argument");
    BMM_TRY(fwht_targets_check(cols, k));
    BMM_TRY(check_targets(rows, stride, cols, targets, others, n_targets, k, "fwht targets"));
    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws)
        return st;
    void *d_words = nullptr, *d_t = nullptr, *d_o = nullptr, *d_m = nullptr, *d_w = nullptr;
    BMM_TRY(upload(ws, kSlotRows, words, rows * stride * 8, &d_words));
    BMM_TRY(upload(ws, kSlotIdx, targets, n_targets * 4, &d_t));
    BMM_TRY(upload(ws, kSlotAux, others, n_targets * k * 4, &d_o));
    BMM_TRY(ws_buffer(ws, kSlotOut, n_targets * 8, &d_m));
    BMM_TRY(ws_buffer(ws, kSlotExtra0, n_targets * 4, &d_w));
    BMM_TRY(fwht_targets_launch(ws, (const uint64_t*)d_words, (int)stride, (int)cols,
                                (const uint32_t*)d_t, (const uint32_t*)d_o, (int)n_targets, (int)k,
                                (uint64_t*)d_m, (uint32_t*)d_w, ws->stream));
    BMM_CUDA_TRY(cudaMemcpyAsync(best_mask, d_m, n_targets * 8, cudaMemcpyDeviceToHost, ws->stream));
    BMM_CUDA_TRY(
        cudaMemcpyAsync(best_weight, d_w, n_targets * 4, cudaMemcpyDeviceToHost, ws->stream));
    BMM_CUDA_TRY(cudaStreamSynchronize(ws->stream));
    return BMM_OK;
}

}  // extern "C"

// ---- spectrum slices (multi-GPU partition of one window's masks) ----------
int bmm_spectrum_tune(int low_bits) {
    clear_error();
    if (low_bits != -1 && (low_bits < 14 || low_bits > 33))
        return fail(BMM_EINVAL, "spectrum tuning: low_bits must be -1 or in [14, 33]");
    g_spectrum_low_bits = low_bits;
    return BMM_OK;
}

int bmm_spectrum_tune_last_pass(int double_buffered) {
    clear_error();
    if (double_buffered != 0 && double_buffered != 1)
        return fail(BMM_EINVAL, "spectrum tuning: double_buffered must be 0 or 1");
    g_spectrum_last_db = double_buffered;
    return BMM_OK;
}

int bmm_spectrum_tune_passes(int register_resident) {
    clear_error();
    if (register_resident < 0 || register_resident > 2)
        return fail(BMM_EINVAL, "spectrum tuning: register_resident must be 0, 1 or 2");
    g_spectrum_reg = register_resident;
    return BMM_OK;
}

int bmm_spectrum_low_bits(size_t t) { return t > 40 ? -1 : spectrum_low_bits((int)t); }

int bmm_spectrum_topk_slices_dev(const uint64_t* d_rows, size_t t, size_t W, size_t cols, size_t k,
                                 int low_bits, int64_t slice_begin, int64_t slice_end,
                                 bmm_candidate* d_out, void* stream) {
    clear_error();
    if (t == 0 || t > 40)
        return fail(BMM_EINVAL, "spectrum slices: t must be in [1, 40]");
    if (!d_rows || !d_out)
        return fail(BMM_EINVAL, "spectrum slices: null argument");
    if (W < (cols + 63) / 64 || W == 0)
        return fail(BMM_EINVAL, "spectrum slices: W smaller than the row width");
    if (cols > 0x7fffffffull)
        return fail(BMM_EOVERFLOW, "spectrum slices: total weight exceeds int32 range");
    const size_t states = ((size_t)1 << t) - 1;
    const size_t kk = k < states ? k : states;
    if (kk == 0 || kk > 1024)
        return fail(BMM_EINVAL, "spectrum slices: k must be in [1, 1024]");
    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws)
        return st;
    return spectrum_topk_slices(ws, d_rows, (int)t, (int)W, (long long)cols, (int)kk, low_bits,
                                (long long)slice_begin, (long long)slice_end, d_out,
                                (cudaStream_t)stream);
}
