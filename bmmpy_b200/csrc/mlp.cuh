// Proposal network state and the device-side entry points used by the GA
// (mlp.cu).
#pragma once

#include "common.cuh"

#include <cuda_bf16.h>

namespace bmm {
namespace mlp {

constexpr int kIn = 512, kHid = 256, kOut = 256;
constexpr size_t kW1 = 0, kB1 = kW1 + (size_t)kHid * kIn, kW2 = kB1 + kHid,
                 kB2 = kW2 + (size_t)kHid * kHid, kW3 = kB2 + kHid,
                 kB3 = kW3 + (size_t)kOut * kHid, kParams = kB3 + kOut;

}  // namespace mlp
}  // namespace bmm

// Parameters, Adam moments, gradients and activation scratch for up to `cap`
// rows, all device-resident.
struct bmm_mlp {
    int device = -1;
    cudaStream_t stream = nullptr;
    bool owns_stream = true;
    float* w = nullptr;  // kParams
    __nv_bfloat16* wb = nullptr;  // kParams: w rounded to BF16, rewritten whenever w changes
    float* m = nullptr;
    float* v = nullptr;
    float* g = nullptr;
    long long step = 0;
    float lr = 1e-3f, b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    size_t cap = 0;
    float* z1 = nullptr;  // [cap][256] pre-activations
    float* z2 = nullptr;
    float* z3 = nullptr;  // logits
    __nv_bfloat16* h1 = nullptr;
    __nv_bfloat16* h2 = nullptr;
    float* dz3 = nullptr;
    float* dz2 = nullptr;
    float* dz1 = nullptr;
    float* x = nullptr;  // [cap][512] staging for host inputs
    float* t = nullptr;  // [cap][256] targets
    float* loss = nullptr;
    float* row_loss = nullptr;  // [cap]
    float* part = nullptr;  // split-K partials of the weight gradients (16 x 256 x 512)
    int* err = nullptr;
};

namespace bmm {
namespace mlp {

// A network on `stream` (nullptr: its own stream).
int create(uint64_t seed, float learning_rate, cudaStream_t stream, bmm_mlp** out);
void destroy(bmm_mlp* h);
// rows inputs X [rows][512] (BF16 if x_bf16, else FP32) -> logits [rows][256]
// (h->z3 when logits is null); asynchronous on h->stream.
int forward_dev(bmm_mlp* h, const void* X, int x_bf16, int rows, float* logits,
                bool keep_pre = true);
// One Adam step on targets T [rows][256]; the loss goes to *h->loss.
int train_step_dev(bmm_mlp* h, const void* X, int x_bf16, const float* T, int rows);
int ensure_cap(bmm_mlp* h, size_t rows);

}  // namespace mlp
}  // namespace bmm
