// bmmpy::CudaMitmFwhtSearch (reference:
// include/bmmpy/search/cuda_mitm_fwht_search.hpp,
// src/search/cuda_mitm_fwht_search.cpp:123-180): the reference's checks,
// including its int16 total-weight guard, then the B200 spectrum search
// (bmm_mitm_search, exact in int32).
#pragma once

#include "searcher.hpp"

#include <stdexcept>

namespace bmmpy {

struct CudaMitmFwhtSearchConfig {
    std::size_t max_candidates = 64;
    std::size_t low_bits = 0;  // auto
};

class CudaMitmFwhtSearch final : public Searcher {
public:
    explicit CudaMitmFwhtSearch(CudaMitmFwhtSearchConfig config = {}) : _config(config) {}

    std::vector<Candidate> search(const RowWindow& window) override {
        if (_config.max_candidates == 0)
            return {};
        const std::size_t t = window.size();
        if (t == 0)
            return {};
        if (t > Candidate::k_word_bits)
            throw std::invalid_argument(
                "CudaMitmFwhtSearch: too many rows in the window (must be <= 64)");
        if (t < k_min_rows || t > k_max_rows)
            throw std::invalid_argument(
                "CudaMitmFwhtSearch: window_rows size is outside the supported GPU range");
        if (_config.low_bits != 0 && _config.low_bits >= t)
            throw std::invalid_argument(
                "CudaMitmFwhtSearch: low_bits must be in [1, t - 1] or 0 for auto");
        if (_config.low_bits > k_max_low_bits)
            throw std::invalid_argument(
                "CudaMitmFwhtSearch: low_bits exceeds the specialized CUDA template range");
        if (window.words_per_row() == 0)
            return {};
        const std::uint64_t active = window.total_weight();
        if (active == 0)
            return {};
        if (active > 32767)
            throw std::invalid_argument(
                "CudaMitmFwhtSearch: total_weight must be <= 32767 for int16-safe GPU mode");
        if (_config.max_candidates > 128)
            throw std::invalid_argument("run_cuda_mitm_fwht_search: max_candidates must be <= 128");
        return b200::window_search(bmm_mitm_search, window, _config.max_candidates,
                                   _config.max_candidates, _config.low_bits);
    }
    const char* name() const noexcept override { return "cuda_mitm_fwht"; }

private:
    static constexpr std::size_t k_min_rows = 16;
    static constexpr std::size_t k_max_rows = 64;
    static constexpr std::size_t k_max_low_bits = 15;
    CudaMitmFwhtSearchConfig _config;
};

}  // namespace bmmpy
