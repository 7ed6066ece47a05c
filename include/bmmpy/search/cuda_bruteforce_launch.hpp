// The reference's brute-force launch seam
// (include/bmmpy/search/cuda_bruteforce_launch.hpp:9-23,
// src/search/cuda_bruteforce_launch.cu:406-458) on the B200 Gray-code kernel
// (bmm_gray_search): the plan's packed rows are searched in place.
#pragma once

#include "../b200_status.hpp"

#include <cstdint>
#include <stdexcept>
#include <vector>

namespace bmmpy {

struct CudaBruteforcePlan {
    std::size_t rows = 0;
    std::size_t cols = 0;
    std::size_t words_per_row = 0;
    std::size_t chunk_bits = 0;  // 0 = auto
    std::vector<std::uint64_t> row_words;
};

struct CudaBruteforceResult {
    std::uint64_t mask;
    std::uint32_t weight;
};

inline std::vector<CudaBruteforceResult> run_cuda_bruteforce_search(const CudaBruteforcePlan& plan,
                                                                   std::size_t max_candidates) {
    if (max_candidates == 0 || plan.rows == 0 || plan.words_per_row == 0)
        return {};
    if (max_candidates > 128)
        throw std::invalid_argument("run_cuda_bruteforce_search: max_candidates must be <= 128");
    if (plan.rows > 64)
        throw std::invalid_argument("run_cuda_bruteforce_search: row count must be <= 64");
    if (plan.row_words.size() != plan.rows * plan.words_per_row)
        throw std::invalid_argument(
            "run_cuda_bruteforce_search: row_words size does not match rows * words_per_row");
    if (plan.chunk_bits != 0 && plan.chunk_bits >= plan.rows)
        throw std::invalid_argument(
            "run_cuda_bruteforce_search: chunk_bits must be in [1, rows - 1] or 0 for auto");
    std::vector<std::uint32_t> win(plan.rows);
    for (std::size_t i = 0; i < plan.rows; ++i)
        win[i] = static_cast<std::uint32_t>(i);
    const std::size_t cols =
        plan.cols ? plan.cols : plan.words_per_row * 64;  // padding bits are zero
    std::vector<bmm_candidate> out(max_candidates);
    std::size_t n = 0;
    b200::check(bmm_gray_search(plan.row_words.data(), plan.words_per_row, cols, win.data(),
                                plan.rows, max_candidates, plan.chunk_bits, out.data(), &n));
    std::vector<CudaBruteforceResult> res(n);
    for (std::size_t i = 0; i < n; ++i)
        res[i] = {out[i].mask, out[i].weight};
    return res;
}

}  // namespace bmmpy
