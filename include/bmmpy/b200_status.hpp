// Status translation for the C++ layer over the C ABI (bmm_b200.h).
//
// The C ABI never throws; this layer turns its status codes into the
// exception types the reference's C++ API throws, so code and tests written
// against bmmpy (include/bmmpy/...) see the same types:
//   BMM_EINVAL -> std::invalid_argument, BMM_EOVERFLOW -> std::overflow_error,
//   BMM_EMATRIX -> bmmpy::MatrixError, everything else -> std::runtime_error.
#pragma once

#include "../bmm_b200.h"

#include <stdexcept>
#include <string>

namespace bmmpy {

enum class MatrixErr { SizeTooLarge, AllocationFailed, DimensionMismatch };

class MatrixError : public std::runtime_error {
public:
    explicit MatrixError(MatrixErr code, const std::string& what = "matrix error")
        : std::runtime_error(what), _code(code) {}
    MatrixErr code() const noexcept { return _code; }

private:
    MatrixErr _code;
};

namespace b200 {

inline std::string last_error() {
    const char* e = bmm_last_error();
    return e ? std::string(e) : std::string();
}

// Throws the reference's exception type for a non-OK status.
inline void check(int rc) {
    if (rc == BMM_OK)
        return;
    const std::string msg = last_error();
    switch (rc) {
    case BMM_EINVAL:
        throw std::invalid_argument(msg);
    case BMM_EOVERFLOW:
        throw std::overflow_error(msg);
    case BMM_EMATRIX:
        throw MatrixError(MatrixErr::DimensionMismatch, msg);
    default:
        throw std::runtime_error(msg);
    }
}

}  // namespace b200
}  // namespace bmmpy
