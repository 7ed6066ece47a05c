// Shared host/device plumbing for the sm_100a kernels: status codes, the
// per-thread error message, the per-thread per-device workspace (stream and
// grow-only device buffers), and small device helpers.
#pragma once

#include "../../include/bmm_b200.h"

#include <cstdarg>
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace bmm {

constexpr unsigned kFull = 0xffffffffu;

// ---- host: error reporting -------------------------------------------------
int fail(int code, const char* fmt, ...);  // records the message, returns code
void clear_error();

#define BMM_CUDA_TRY(expr)                                                                        \
    do {                                                                                          \
        cudaError_t bmm_e_ = (expr);                                                              \
        if (bmm_e_ != cudaSuccess)                                                                \
            return ::bmm::fail(BMM_ECUDA, "%s failed: %s", #expr, cudaGetErrorString(bmm_e_));    \
    } while (0)

#define BMM_TRY(expr)                                                                             \
    do {                                                                                          \
        int bmm_rc_ = (expr);                                                                     \
        if (bmm_rc_ != BMM_OK)                                                                    \
            return bmm_rc_;                                                                       \
    } while (0)

// ---- host: per-thread, per-device workspace --------------------------------
// Slots name the device buffers an entry point needs; each grows on demand and
// is reused by later calls from the same host thread on the same device.
enum Slot : int {
    kSlotRows = 0,
    kSlotAux,
    kSlotIdx,
    kSlotSpec,
    kSlotCand,
    kSlotOut,
    kSlotKeys,
    kSlotCounter,
    kSlotExtra0,
    kSlotExtra1,
    kSlotSlices,
    kSlotSweepWin,    // search -> apply sweeps: window lists, new rows, states, order
    kSlotSweepNew,
    kSlotSweepState,
    kSlotSweepOrder,
    kSlotEmptyBits,   // spectrum: one bit per pass-A tile without patterns
    kSlotCount
};

struct Workspace {
    int device = -1;
    int sm_count = 0;
    int smem_optin = 0;
    cudaStream_t stream = nullptr;
    void* buf[kSlotCount] = {};
    size_t cap[kSlotCount] = {};
    void* pinned = nullptr;  // pinned host staging
    size_t pinned_cap = 0;
};

// Returns the calling thread's workspace for the current device (created and
// queried on first use).  Sets *ok = BMM_OK or an error status.
Workspace* workspace(int* status);
int ws_buffer(Workspace* ws, int slot, size_t bytes, void** out);
int ws_pinned(Workspace* ws, size_t bytes, void** out);

// ---- device helpers --------------------------------------------------------
__device__ __forceinline__ bool pair_less(uint32_t wa, uint64_t ma, uint32_t wb, uint64_t mb) {
    return wa < wb || (wa == wb && ma < mb);
}

__host__ __device__ __forceinline__ uint64_t inverse_gray64(uint64_t s) {
    s ^= s >> 1;
    s ^= s >> 2;
    s ^= s >> 4;
    s ^= s >> 8;
    s ^= s >> 16;
    s ^= s >> 32;
    return s;
}

}  // namespace bmm
