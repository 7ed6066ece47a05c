// The reference's MITM launch seam (include/bmmpy/search/cuda_mitm_fwht_launch.hpp:15-16,
// src/search/cuda_mitm_fwht_launch.cu:453-496) on the B200 spectrum search:
// the split window's patterns, each repeated by its multiplicity, are the
// columns of a (low_bits + high_bits)-row window whose exact top-k
// bmm_mitm_search returns -- the same (mask, weight) list the reference's
// kernel returns, with no int16 or multiplicity limit.
#pragma once

#include "split_window_prep.hpp"
#include "../b200_status.hpp"

#include <vector>

namespace bmmpy {

struct CudaMitmFwhtResult {
    std::uint64_t mask;
    std::uint32_t weight;
};

inline std::vector<CudaMitmFwhtResult> run_cuda_mitm_fwht_search(const CompactSplitWindow& prep,
                                                                 std::size_t max_candidates) {
    if (max_candidates == 0 || prep.multiplicity.empty())
        return {};
    if (max_candidates > 128)
        throw std::invalid_argument("run_cuda_mitm_fwht_search: max_candidates must be <= 128");
    const std::size_t t = prep.low_bits + prep.high_bits;
    std::size_t cols = 0;
    for (std::int32_t m : prep.multiplicity) {
        if (m <= 0)
            throw std::invalid_argument(
                "run_cuda_mitm_fwht_search: multiplicity must be positive");
        cols += static_cast<std::size_t>(m);
    }
    const std::size_t W = (cols + 63) / 64;
    std::vector<std::uint64_t> words(t * W, 0);
    std::size_t c = 0;
    for (std::size_t i = 0; i < prep.multiplicity.size(); ++i) {
        const std::uint64_t p = (prep.q[i] << prep.low_bits) | prep.r[i];
        for (std::int32_t rep = 0; rep < prep.multiplicity[i]; ++rep, ++c)
            for (std::size_t row = 0; row < t; ++row)
                if ((p >> row) & 1u)
                    words[row * W + c / 64] |= std::uint64_t{1} << (c % 64);
    }
    std::vector<std::uint32_t> win(t);
    for (std::size_t i = 0; i < t; ++i)
        win[i] = static_cast<std::uint32_t>(i);
    std::vector<bmm_candidate> out(max_candidates);
    std::size_t n = 0;
    b200::check(bmm_mitm_search(words.data(), W, cols, win.data(), t, max_candidates, 0,
                                out.data(), &n));
    std::vector<CudaMitmFwhtResult> res(n);
    for (std::size_t i = 0; i < n; ++i)
        res[i] = {out[i].mask, out[i].weight};
    return res;
}

}  // namespace bmmpy
