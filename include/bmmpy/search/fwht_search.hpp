// bmmpy::FwhtSearch (reference: include/bmmpy/search/fwht_search.hpp,
// src/search/fwht_search.cpp:34-132) over bmm_fwht_search.
#pragma once

#include "searcher.hpp"

namespace bmmpy {

struct FwhtSearchConfig {
    std::size_t max_rows = 16;
    std::size_t max_candidates = 64;
};

class FwhtSearch final : public Searcher {
public:
    explicit FwhtSearch(FwhtSearchConfig config = {}) : _config(config) {}
    std::vector<Candidate> search(const RowWindow& window) override {
        if (_config.max_candidates == 0 || window.size() == 0 ||
            window.size() > _config.max_rows)
            return {};
        return b200::window_search(bmm_fwht_search, window, _config.max_candidates,
                                   _config.max_rows, _config.max_candidates);
    }
    const char* name() const noexcept override { return "fwht"; }
    const FwhtSearchConfig& config() const noexcept { return _config; }

private:
    FwhtSearchConfig _config;
};

}  // namespace bmmpy
