// bmmpy::BruteforceSearch (reference: include/bmmpy/search/bruteforce_search.hpp,
// src/search/bruteforce_search.cpp:300-329) over bmm_gray_search.
#pragma once

#include "searcher.hpp"

namespace bmmpy {

struct BruteforceSearchConfig {
    std::size_t max_candidates = 128;
    std::size_t chunk_bits = 0;  // 0 = auto
};

class BruteforceSearch final : public Searcher {
public:
    explicit BruteforceSearch(BruteforceSearchConfig config = {}) : _config(config) {}
    std::vector<Candidate> search(const RowWindow& window) override {
        if (_config.max_candidates == 0 || window.size() == 0)
            return {};
        return b200::window_search(bmm_gray_search, window, _config.max_candidates,
                                   _config.max_candidates, _config.chunk_bits);
    }
    const char* name() const noexcept override { return "bruteforce"; }

private:
    BruteforceSearchConfig _config;
};

}  // namespace bmmpy
