// bmmpy::Searcher (reference: include/bmmpy/search/searcher.hpp:11-19) and the
// B200 searchers behind it.  Every search runs on the GPU through the C ABI
// (bmm_b200.h) and returns candidates ordered by (weight, mask); exceptions
// follow the reference's types (see b200_status.hpp).
#pragma once

#include "../core/bit_matrix.hpp"
#include "../types/candidate.hpp"

#include <vector>

namespace bmmpy {

class Searcher {
public:
    virtual ~Searcher() = default;
    virtual std::vector<Candidate> search(const RowWindow& window) = 0;
    virtual const char* name() const noexcept = 0;
};

namespace b200 {

// Runs one of the C ABI window searches on the window's rows in place.
template <typename Fn, typename... Extra>
std::vector<Candidate> window_search(Fn fn, const RowWindow& w, std::size_t k, Extra... extra) {
    const std::size_t t = w.size();
    const std::size_t states = t >= 64 ? ~std::size_t{0} : ((std::size_t{1} << t) - 1);
    const std::size_t cap = std::max<std::size_t>(1, std::min(k, states));
    std::vector<bmm_candidate> out(cap);
    std::size_t n = 0;
    const std::vector<std::uint32_t> win = w.index_u32();
    check(fn(w.matrix().data(), w.stride_words(), w.cols(), win.data(), t, extra...,
             out.data(), &n));
    std::vector<Candidate> res;
    res.reserve(n);
    for (std::size_t i = 0; i < n; ++i)
        res.push_back(Candidate::from_u64(out[i].mask, out[i].weight));
    return res;
}

}  // namespace b200
}  // namespace bmmpy
