// bmmpy::MitmFwhtSearch (reference: include/bmmpy/search/mitm_fwht_search.hpp,
// src/search/mitm_fwht_search.cpp:267-322) over bmm_mitm_search.  The
// reserve_* fields size the reference's CPU scratch; they are accepted and
// have no effect here.
#pragma once

#include "searcher.hpp"

namespace bmmpy {

struct MitmFwhtSearchConfig {
    std::size_t reserve_unique_patterns = 1024;
    std::size_t reserve_left_rows = 20;
    std::size_t reserve_right_states = std::size_t{1} << 16;
    std::size_t max_candidates = 64;
};

class MitmFwhtSearch final : public Searcher {
public:
    explicit MitmFwhtSearch(MitmFwhtSearchConfig config = {}) : _config(config) {}
    std::vector<Candidate> search(const RowWindow& window) override {
        if (_config.max_candidates == 0 || window.size() == 0)
            return {};
        return b200::window_search(bmm_mitm_search, window, _config.max_candidates,
                                   _config.max_candidates, std::size_t{0});
    }
    const char* name() const noexcept override { return "mitm_fwht"; }

private:
    MitmFwhtSearchConfig _config;
};

}  // namespace bmmpy
