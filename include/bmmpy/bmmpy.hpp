// The C++ API of bmmpy's search / solver path for the B200 build: the
// reference's class names and signatures (include/bmmpy/...), header-only
// over the C ABI of bmm_b200.h (link with libbmm_b200.so).  The GA classes are
// reached through the C ABI (bmm_ga_*) and the Python package.
#pragma once

#include "core/bit_matrix.hpp"
#include "core/row_window.hpp"
#include "math/fwht.hpp"
#include "search/bruteforce_search.hpp"
#include "search/cuda_bruteforce_launch.hpp"
#include "search/cuda_bruteforce_search.hpp"
#include "search/cuda_mitm_fwht_launch.hpp"
#include "search/cuda_mitm_fwht_search.hpp"
#include "search/fwht_search.hpp"
#include "search/mitm_fwht_search.hpp"
#include "search/searcher.hpp"
#include "search/split_window_prep.hpp"
#include "solver/exact_basis_solver.hpp"
#include "stub.hpp"
#include "types/candidate.hpp"
