// bmmpy::CompactSplitWindow / build_compact_split_window (reference:
// include/bmmpy/search/split_window_prep.hpp:10-19,
// src/search/split_window_prep.cpp:42-137): the window's distinct column
// patterns (bit r = row r) in ascending order with their multiplicities,
// split into q = pattern >> low_bits and r = pattern & (2^low_bits - 1);
// total_weight = the number of active columns.  Same checks and messages.
#pragma once

#include "../core/bit_matrix.hpp"

#include <algorithm>
#include <cstdint>
#include <limits>
#include <stdexcept>
#include <utility>
#include <vector>

namespace bmmpy {

struct CompactSplitWindow {
    std::size_t t = 0;
    std::size_t low_bits = 0;
    std::size_t high_bits = 0;
    std::int32_t total_weight = 0;
    std::vector<std::uint64_t> q;
    std::vector<std::uint64_t> r;
    std::vector<std::int32_t> multiplicity;
};

inline CompactSplitWindow build_compact_split_window(const std::vector<const std::uint64_t*>& rows,
                                                     std::size_t words_per_row, std::size_t cols,
                                                     std::size_t low_bits) {
    CompactSplitWindow out;
    out.t = rows.size();
    out.low_bits = low_bits;
    if (low_bits > out.t)
        throw std::invalid_argument(
            "build_compact_split_window: low_bits must be <= number of rows");
    if (out.t > 64)
        throw std::invalid_argument("build_compact_split_window: row count must be <= 64");
    out.high_bits = out.t - low_bits;
    if (rows.empty() || words_per_row == 0)
        return out;
    // column patterns, then sort + run lengths (the same multiset as the
    // reference's hash map, in the same ascending order)
    std::vector<std::uint64_t> pats;
    pats.reserve(cols);
    for (std::size_t c = 0; c < cols; ++c) {
        std::uint64_t p = 0;
        for (std::size_t i = 0; i < rows.size(); ++i)
            p |= ((rows[i][c / 64] >> (c % 64)) & 1u) << i;
        if (p)
            pats.push_back(p);
    }
    if (pats.size() > static_cast<std::size_t>(std::numeric_limits<std::int32_t>::max()))
        throw std::overflow_error("build_compact_split_window: total weight exceeds int32 range");
    std::sort(pats.begin(), pats.end());
    out.total_weight = static_cast<std::int32_t>(pats.size());
    const std::uint64_t low_mask = low_bits >= 64 ? ~std::uint64_t{0}
                                                  : ((std::uint64_t{1} << low_bits) - 1);
    for (std::size_t i = 0; i < pats.size();) {
        std::size_t j = i;
        while (j < pats.size() && pats[j] == pats[i])
            ++j;
        out.q.push_back(low_bits >= 64 ? 0 : (pats[i] >> low_bits));
        out.r.push_back(pats[i] & low_mask);
        out.multiplicity.push_back(static_cast<std::int32_t>(j - i));
        i = j;
    }
    return out;
}

inline CompactSplitWindow build_compact_split_window(const RowWindow& window,
                                                     std::size_t low_bits) {
    return build_compact_split_window(window.row_ptrs(), window.words_per_row(), window.cols(),
                                      low_bits);
}

}  // namespace bmmpy
