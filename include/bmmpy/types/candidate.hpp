// bmmpy::Candidate (reference: include/bmmpy/types/candidate.hpp): one row
// combination of a window -- the mask over the window's local rows as 64-bit
// words, and the weight of the combined row.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

namespace bmmpy {

struct Candidate {
    using word_type = std::uint64_t;
    using mask_type = std::vector<word_type>;
    static constexpr std::size_t k_word_bits = 64;

    mask_type mask;
    std::uint32_t weight = 0;

    static Candidate from_u64(std::uint64_t m, std::uint32_t w) {
        Candidate c;
        if (m != 0)
            c.mask.push_back(m);
        c.weight = w;
        return c;
    }

    // First mask word (windows of at most 64 rows use only this one).
    std::uint64_t mask_u64() const noexcept { return mask.empty() ? 0 : mask[0]; }

    bool empty() const noexcept {
        for (word_type w : mask)
            if (w)
                return false;
        return true;
    }

    // Local row indices selected by the mask, ascending.
    std::vector<std::size_t> selected_rows() const {
        std::vector<std::size_t> out;
        for (std::size_t i = 0; i < mask.size(); ++i)
            for (word_type w = mask[i]; w; w &= w - 1)
                out.push_back(i * k_word_bits + static_cast<std::size_t>(__builtin_ctzll(w)));
        return out;
    }

    std::size_t popcount() const noexcept {
        std::size_t n = 0;
        for (word_type w : mask)
            n += static_cast<std::size_t>(__builtin_popcountll(w));
        return n;
    }
};

// The reference's candidate order: weight, then mask value.
inline bool candidate_less(const Candidate& a, const Candidate& b) noexcept {
    if (a.weight != b.weight)
        return a.weight < b.weight;
    return a.mask_u64() < b.mask_u64();
}

}  // namespace bmmpy
