// bmmpy::CudaBruteforceSearch (reference:
// include/bmmpy/search/cuda_bruteforce_search.hpp,
// src/search/cuda_bruteforce_search.cpp:38-103): the reference's argument
// checks and messages, then the B200 Gray-code kernel (bmm_gray_search).
#pragma once

#include "searcher.hpp"

#include <stdexcept>

namespace bmmpy {

struct CudaBruteforceSearchConfig {
    std::size_t max_candidates = 128;
    std::size_t chunk_bits = 0;  // 0 = auto
};

class CudaBruteforceSearch final : public Searcher {
public:
    explicit CudaBruteforceSearch(CudaBruteforceSearchConfig config = {}) : _config(config) {}

    std::vector<Candidate> search(const RowWindow& window) override {
        if (_config.max_candidates == 0)
            return {};
        const std::size_t t = window.size();
        if (t == 0)
            return {};
        if (t > Candidate::k_word_bits)
            throw std::invalid_argument(
                "CudaBruteforceSearch: too many rows in the window (must be <= 64)");
        if (t < k_min_rows || t > k_max_rows)
            throw std::invalid_argument(
                "CudaBruteforceSearch: window_rows size is outside the supported GPU range");
        if (_config.max_candidates > 128)
            throw std::invalid_argument("CudaBruteforceSearch: max_candidates must be <= 128");
        const std::size_t wpr = window.words_per_row();
        if (wpr == 0)
            return {};
        if (wpr != 8 && wpr != 16 && wpr != 64)
            throw std::invalid_argument("CudaBruteforceSearch: only widths 512, 1024, and 4096 "
                                        "are supported in the current GPU path");
        if (_config.chunk_bits != 0 &&
            (_config.chunk_bits >= t || _config.chunk_bits >= Candidate::k_word_bits))
            throw std::invalid_argument(
                "CudaBruteforceSearch: chunk_bits must be in [1, t - 1] or 0 for auto");
        return b200::window_search(bmm_gray_search, window, _config.max_candidates,
                                   _config.max_candidates, _config.chunk_bits);
    }
    const char* name() const noexcept override { return "cuda_bruteforce"; }

private:
    static constexpr std::size_t k_min_rows = 16;
    static constexpr std::size_t k_max_rows = 64;
    CudaBruteforceSearchConfig _config;
};

}  // namespace bmmpy
