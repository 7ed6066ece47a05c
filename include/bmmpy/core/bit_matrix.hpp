// bmmpy::BitMatrix and bmmpy::RowWindow for the B200 build (reference:
// include/bmmpy/core/bit_matrix.hpp, include/bmmpy/core/row_window.hpp).
//
// Same storage as the reference: row-major uint64 words, bit c of a row in
// word c / 64 at bit c % 64, each row padded to a stride that is a multiple of
// four words, bits past cols always zero (src/core/bit_matrix.cpp:67-72).  A
// RowWindow borrows row pointers of one matrix (a mutable one when built from
// a non-const matrix).  The searches read these buffers directly through the
// C ABI, so a BitMatrix here is what bmm_*_search expects.
#pragma once

#include "../b200_status.hpp"

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace bmmpy {

class RowWindow;

class BitMatrix {
public:
    static constexpr std::size_t k_word_bits = 64;

    BitMatrix() noexcept = default;
    BitMatrix(std::size_t rows, std::size_t cols)
        : _rows(rows), _cols(cols), _stride(((cols + 63) / 64 + 3) / 4 * 4),
          _words(rows * _stride, 0) {}

    std::size_t rows() const noexcept { return _rows; }
    std::size_t cols() const noexcept { return _cols; }
    std::size_t stride_words() const noexcept { return _stride; }
    std::size_t words_per_row() const noexcept { return (_cols + 63) / 64; }
    std::size_t total_words() const noexcept { return _words.size(); }
    const std::uint64_t* data() const noexcept { return _words.data(); }
    std::uint64_t* data() noexcept { return _words.data(); }

    const std::uint64_t* row_words(std::size_t r) const {
        check_row(r);
        return _words.data() + r * _stride;
    }
    std::uint64_t* row_words(std::size_t r) {
        check_row(r);
        return _words.data() + r * _stride;
    }

    bool get(std::size_t r, std::size_t c) const {
        check_cell(r, c);
        return (row_words(r)[c / 64] >> (c % 64)) & 1u;
    }
    void set(std::size_t r, std::size_t c, bool v) {
        check_cell(r, c);
        std::uint64_t& w = row_words(r)[c / 64];
        const std::uint64_t bit = std::uint64_t{1} << (c % 64);
        w = v ? (w | bit) : (w & ~bit);
    }

    void row_xor(std::size_t target, std::size_t source) {
        std::uint64_t* t = row_words(target);
        const std::uint64_t* s = row_words(source);
        for (std::size_t i = 0; i < words_per_row(); ++i)
            t[i] ^= s[i];
    }

    std::uint64_t row_popcount(std::size_t r) const {
        const std::uint64_t* p = row_words(r);
        std::uint64_t n = 0;
        for (std::size_t i = 0; i < words_per_row(); ++i)
            n += static_cast<std::uint64_t>(__builtin_popcountll(p[i]));
        return n;
    }
    std::uint64_t weight() const {
        std::uint64_t n = 0;
        for (std::size_t r = 0; r < _rows; ++r)
            n += row_popcount(r);
        return n;
    }

    static BitMatrix identity(std::size_t n) {
        BitMatrix m(n, n);
        for (std::size_t i = 0; i < n; ++i)
            m.set(i, i, true);
        return m;
    }

    // Rows given as strings of '0' / '1' of equal length.
    static BitMatrix from_rows(const std::vector<std::string>& rows) {
        const std::size_t cols = rows.empty() ? 0 : rows[0].size();
        BitMatrix m(rows.size(), cols);
        for (std::size_t r = 0; r < rows.size(); ++r) {
            if (rows[r].size() != cols)
                throw std::invalid_argument("matrix_from_rows: rows must have equal length");
            for (std::size_t c = 0; c < cols; ++c) {
                if (rows[r][c] != '0' && rows[r][c] != '1')
                    throw std::invalid_argument("matrix_from_rows: rows may hold only 0 and 1");
                m.set(r, c, rows[r][c] == '1');
            }
        }
        return m;
    }
    std::vector<std::string> to_rows() const {
        std::vector<std::string> out(_rows, std::string(_cols, '0'));
        for (std::size_t r = 0; r < _rows; ++r)
            for (std::size_t c = 0; c < _cols; ++c)
                if (get(r, c))
                    out[r][c] = '1';
        return out;
    }

    RowWindow row_window(const std::vector<std::size_t>& rows);
    RowWindow row_window(const std::vector<std::size_t>& rows) const;

    bool operator==(const BitMatrix& o) const noexcept {
        return _rows == o._rows && _cols == o._cols && _words == o._words;
    }

private:
    void check_row(std::size_t r) const {
        if (r >= _rows)
            throw std::out_of_range("BitMatrix: row index out of bounds");
    }
    void check_cell(std::size_t r, std::size_t c) const {
        check_row(r);
        if (c >= _cols)
            throw std::out_of_range("BitMatrix: column index out of bounds");
    }

    std::size_t _rows = 0, _cols = 0, _stride = 0;
    std::vector<std::uint64_t> _words;
};

inline BitMatrix matrix_from_rows(const std::vector<std::string>& rows) {
    return BitMatrix::from_rows(rows);
}

class RowWindow {
public:
    RowWindow(BitMatrix& m, std::vector<std::size_t> rows)
        : _matrix(&m), _mutable(&m), _rows(std::move(rows)) {
        init();
    }
    RowWindow(const BitMatrix& m, std::vector<std::size_t> rows)
        : _matrix(&m), _rows(std::move(rows)) {
        init();
    }

    const BitMatrix& matrix() const noexcept { return *_matrix; }
    bool is_mutable() const noexcept { return _mutable != nullptr; }
    std::size_t size() const noexcept { return _rows.size(); }
    std::size_t cols() const noexcept { return _matrix->cols(); }
    std::size_t words_per_row() const noexcept { return _matrix->words_per_row(); }
    std::size_t stride_words() const noexcept { return _matrix->stride_words(); }
    const std::vector<std::size_t>& global_rows() const noexcept { return _rows; }
    std::size_t global_row(std::size_t i) const { return _rows.at(i); }
    const std::vector<const std::uint64_t*>& row_ptrs() const noexcept { return _ptrs; }
    const std::uint64_t* row_words(std::size_t i) const { return _ptrs.at(i); }
    std::uint64_t row_popcount(std::size_t i) const { return _matrix->row_popcount(_rows.at(i)); }
    std::uint64_t weight() const {
        std::uint64_t n = 0;
        for (std::size_t r : _rows)
            n += _matrix->row_popcount(r);
        return n;
    }
    // Columns active in any window row (the total weight the spectrum
    // searches split over their column patterns).
    std::uint64_t total_weight() const {
        std::uint64_t n = 0;
        for (std::size_t w = 0; w < words_per_row(); ++w) {
            std::uint64_t acc = 0;
            for (const std::uint64_t* p : _ptrs)
                acc |= p[w];
            n += static_cast<std::uint64_t>(__builtin_popcountll(acc));
        }
        return n;
    }
    bool get(std::size_t i, std::size_t c) const { return _matrix->get(_rows.at(i), c); }
    void set(std::size_t i, std::size_t c, bool v) { require_mutable().set(_rows.at(i), c, v); }
    void row_xor(std::size_t target, std::size_t source) {
        require_mutable().row_xor(_rows.at(target), _rows.at(source));
    }

    BitMatrix materialize() const {
        BitMatrix out(size(), cols());
        for (std::size_t i = 0; i < size(); ++i)
            std::copy_n(_ptrs[i], words_per_row(), out.row_words(i));
        return out;
    }
    void assign_materialized(const BitMatrix& rows) {
        if (rows.rows() != size() || rows.cols() != cols())
            throw MatrixError(MatrixErr::DimensionMismatch, "RowWindow: dimension mismatch");
        BitMatrix& m = require_mutable();
        for (std::size_t i = 0; i < size(); ++i)
            std::copy_n(rows.row_words(i), words_per_row(), m.row_words(_rows[i]));
    }

    // Local row list as the 32-bit indices the C ABI takes, with the matrix
    // buffer it indexes (the window borrows the matrix's rows in place).
    std::vector<std::uint32_t> index_u32() const {
        std::vector<std::uint32_t> out(_rows.size());
        for (std::size_t i = 0; i < _rows.size(); ++i) {
            if (_rows[i] > 0xfffffffeu)
                throw std::invalid_argument("RowWindow: row index exceeds the 32-bit range");
            out[i] = static_cast<std::uint32_t>(_rows[i]);
        }
        return out;
    }

private:
    void init() {
        _ptrs.reserve(_rows.size());
        for (std::size_t r : _rows) {
            if (r >= _matrix->rows())
                throw std::out_of_range("row window row out of bounds");
            _ptrs.push_back(_matrix->row_words(r));
        }
    }
    BitMatrix& require_mutable() {
        if (!_mutable)
            throw std::logic_error("RowWindow: the window was built from a const matrix");
        return *_mutable;
    }

    const BitMatrix* _matrix = nullptr;
    BitMatrix* _mutable = nullptr;
    std::vector<std::size_t> _rows;
    std::vector<const std::uint64_t*> _ptrs;
};

inline RowWindow BitMatrix::row_window(const std::vector<std::size_t>& rows) {
    return RowWindow(*this, rows);
}
inline RowWindow BitMatrix::row_window(const std::vector<std::size_t>& rows) const {
    return RowWindow(*this, rows);
}

}  // namespace bmmpy
