// Test-infrastructure harness around the UNMODIFIED reference CUDA search path.
//
// Linked (by `make -C oracle ref-cuda`) against the reference's own
// translation units compiled in place with its CUDA backend on
// (BMMPY_HAS_CUDA_BACKEND; src/search/cuda_bruteforce_launch.cu and
// src/search/cuda_mitm_fwht_launch.cu built by nvcc for sm_100a), so that
// bench.py's `--impl reference-gpu` arm and the tests can time and check the
// reference's GPU kernels on the same B200.  Nothing in the product links it.
//
// Rows are a packed row-major uint64 buffer (bit c of a row in word c/64,
// `stride` words per row), as in ref_harness.cpp.  Return convention: >= 0 the
// number of candidates the reference returned (at most `cap` are written),
// -1 std::invalid_argument, -4 std::runtime_error, -5 other std::exception.

#include "bmmpy/core/bit_matrix.hpp"
#include "bmmpy/core/row_window.hpp"
#include "bmmpy/search/cuda_bruteforce_search.hpp"
#include "bmmpy/search/cuda_mitm_fwht_search.hpp"

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

bmmpy::BitMatrix make_matrix(const std::uint64_t* words, std::size_t rows, std::size_t cols,
                             std::size_t stride) {
    bmmpy::BitMatrix m(rows, cols);
    const std::size_t wpr = m.words_per_row();
    for (std::size_t r = 0; r < rows; ++r) {
        std::uint64_t* dst = m.row_words(r);
        for (std::size_t w = 0; w < wpr; ++w)
            dst[w] = words[r * stride + w];
        const std::size_t tail = cols % 64;
        if (tail != 0 && wpr != 0)
            dst[wpr - 1] &= (std::uint64_t{1} << tail) - 1;
    }
    return m;
}

template <typename Fn> long guarded(Fn&& fn) {
    try {
        g_err.clear();
        return fn();
    } catch (const std::invalid_argument& e) {
        g_err = e.what();
        return -1;
    } catch (const std::runtime_error& e) {
        g_err = e.what();
        return -4;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -5;
    }
}

long emit(const std::vector<bmmpy::Candidate>& cands, std::size_t cap, std::uint64_t* out_mask,
          std::uint32_t* out_weight) {
    for (std::size_t i = 0; i < cands.size() && i < cap; ++i) {
        out_mask[i] = cands[i].mask_u64();
        out_weight[i] = cands[i].weight;
    }
    return static_cast<long>(cands.size());
}

}  // namespace

extern "C" {

const char* refc_last_error() { return g_err.c_str(); }

// bmmpy::CudaBruteforceSearch{k, chunk_bits}.search(window)
// (src/search/cuda_bruteforce_search.cpp:38-103 -> run_cuda_bruteforce_search,
// src/search/cuda_bruteforce_launch.cu:406-458)
long refc_cuda_bruteforce_search(const std::uint64_t* words, std::size_t rows, std::size_t cols,
                                 std::size_t stride, const std::size_t* win, std::size_t t,
                                 std::size_t k, std::size_t chunk_bits, std::uint64_t* out_mask,
                                 std::uint32_t* out_weight, std::size_t cap) {
    return guarded([&] {
        const auto m = make_matrix(words, rows, cols, stride);
        const auto w = m.row_window(std::vector<std::size_t>(win, win + t));
        bmmpy::CudaBruteforceSearch s(bmmpy::CudaBruteforceSearchConfig{k, chunk_bits});
        return emit(s.search(w), cap, out_mask, out_weight);
    });
}

// bmmpy::CudaMitmFwhtSearch{k, low_bits}.search(window)
// (src/search/cuda_mitm_fwht_search.cpp:123-180 -> run_cuda_mitm_fwht_search,
// src/search/cuda_mitm_fwht_launch.cu:453-496)
long refc_cuda_mitm_search(const std::uint64_t* words, std::size_t rows, std::size_t cols,
                           std::size_t stride, const std::size_t* win, std::size_t t,
                           std::size_t k, std::size_t low_bits, std::uint64_t* out_mask,
                           std::uint32_t* out_weight, std::size_t cap) {
    return guarded([&] {
        const auto m = make_matrix(words, rows, cols, stride);
        const auto w = m.row_window(std::vector<std::size_t>(win, win + t));
        bmmpy::CudaMitmFwhtSearch s(bmmpy::CudaMitmFwhtSearchConfig{k, low_bits});
        return emit(s.search(w), cap, out_mask, out_weight);
    });
}

}  // extern "C"
