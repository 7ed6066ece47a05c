// bmmpy::ExactBasisSolver (reference: include/bmmpy/solver/exact_basis_solver.hpp:12-43,
// src/solver/exact_basis_solver.cpp:58-157) over bmm_exact_basis: the
// minimum-weight basis of the window's row space the reference's greedy
// picks, with its transform and basis matrices.
#pragma once

#include "../core/bit_matrix.hpp"

#include <vector>

namespace bmmpy {

struct ExactBasisSolverConfig {
    std::size_t max_rows = 24;
    std::uint64_t max_states = (std::uint64_t{1} << 24) - 1;
    std::size_t max_storage_bytes = 128u * 1024u * 1024u;
};

struct ExactBasisResult {
    std::size_t input_rows = 0;
    std::size_t cols = 0;
    std::size_t rank = 0;
    std::uint64_t enumerated_states = 0;
    std::uint64_t total_weight = 0;
    std::vector<std::uint32_t> basis_masks;
    std::vector<std::uint32_t> basis_weights;
    BitMatrix transform_matrix;
    BitMatrix basis_matrix;
};

class ExactBasisSolver final {
public:
    explicit ExactBasisSolver(ExactBasisSolverConfig config = {}) : _config(config) {}
    const char* name() const noexcept { return "exact_basis"; }

    ExactBasisResult solve(const RowWindow& window) const {
        const std::size_t t = window.size();
        const bmm_exact_basis_config cfg{_config.max_rows, _config.max_states,
                                         _config.max_storage_bytes};
        bmm_exact_basis_result r{};
        const std::size_t room = std::max<std::size_t>(1, std::min(t, window.cols()));
        std::vector<std::uint32_t> masks(room), weights(room);
        const std::vector<std::uint32_t> win = window.index_u32();
        b200::check(bmm_exact_basis(window.matrix().data(), window.stride_words(), window.cols(),
                                    win.data(), t, &cfg, &r, masks.data(), weights.data()));
        ExactBasisResult out;
        out.input_rows = r.input_rows;
        out.cols = r.cols;
        out.rank = r.rank;
        out.enumerated_states = r.enumerated_states;
        out.total_weight = r.total_weight;
        out.basis_masks.assign(masks.begin(), masks.begin() + r.rank);
        out.basis_weights.assign(weights.begin(), weights.begin() + r.rank);
        // transform row k = basis mask k over the t rows; basis row k = that
        // combination of the window rows
        out.transform_matrix = BitMatrix(r.rank, t);
        out.basis_matrix = BitMatrix(r.rank, window.cols());
        for (std::size_t k = 0; k < r.rank; ++k)
            for (std::size_t i = 0; i < t; ++i)
                if ((out.basis_masks[k] >> i) & 1u) {
                    out.transform_matrix.set(k, i, true);
                    std::uint64_t* dst = out.basis_matrix.row_words(k);
                    const std::uint64_t* src = window.row_words(i);
                    for (std::size_t w = 0; w < window.words_per_row(); ++w)
                        dst[w] ^= src[w];
                }
        return out;
    }

private:
    ExactBasisSolverConfig _config;
};

}  // namespace bmmpy
