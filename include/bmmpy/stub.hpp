// bmmpy::RuntimeFeatures / get_runtime_features / get_version (reference:
// include/bmmpy/stub.hpp:7-21) for the B200 build: the CUDA path is always
// compiled; AVX2 / OpenMP CPU backends do not exist here.
#pragma once

#include "b200_status.hpp"

#include <string>

namespace bmmpy {

struct RuntimeFeatures {
    bool avx2_compiled = false;
    bool avx2_available = false;
    bool cuda_compiled = true;
    bool cuda_available = false;
    bool parallel_compiled = false;
    bool parallel_enabled = false;
    int max_threads = 1;
    std::string bit_ops_backend = "cuda";
    std::string fwht_backend = "cuda";
};

inline std::string get_version() { return bmm_version(); }

inline RuntimeFeatures get_runtime_features() {
    RuntimeFeatures out;
    bmm_features f{};
    if (bmm_runtime_features(&f) == BMM_OK) {
        out.cuda_compiled = f.cuda_compiled != 0;
        out.cuda_available = f.cuda_available != 0;
    }
    return out;
}

}  // namespace bmmpy
