// bmmpy::fwht_inplace (reference: include/bmmpy/math/fwht.hpp:8-9): the
// unnormalised Walsh-Hadamard transform in natural order, wrapping
// two's-complement, on the GPU (bmm_fwht_i16 / bmm_fwht_i32).  Throws
// std::invalid_argument for a size that is not a power of two.
#pragma once

#include "../b200_status.hpp"

#include <cstdint>

namespace bmmpy {

inline void fwht_inplace(std::int16_t* data, std::size_t size) {
    b200::check(bmm_fwht_i16(data, size));
}

inline void fwht_inplace(std::int32_t* data, std::size_t size) {
    b200::check(bmm_fwht_i32(data, size));
}

}  // namespace bmmpy
