// bmmpy::RowWindow (reference: include/bmmpy/core/row_window.hpp); defined
// with BitMatrix in bit_matrix.hpp.
#pragma once

#include "bit_matrix.hpp"
