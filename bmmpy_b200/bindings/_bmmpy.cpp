// _bmmpy: the reference's native Python module name (python/bindings/*.cpp,
// bmmpy/_bmmpy.pyi) for the search / solver path, bound with pybind11 over
// the C++ API of include/bmmpy/ (itself over the C ABI of libbmm_b200.so).
// Classes, constructor keywords, method names and exception types follow the
// reference's module; everything runs on the GPU.
#include "bmmpy/bmmpy.hpp"

#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <sstream>

namespace py = pybind11;
using namespace bmmpy;

namespace {

std::pair<std::size_t, std::size_t> cell(const py::tuple& idx) {
    if (idx.size() != 2)
        throw py::index_error("BitMatrix index must be (row, col)");
    return {idx[0].cast<std::size_t>(), idx[1].cast<std::size_t>()};
}

template <typename T>
void fwht_array(py::array_t<T, py::array::c_style> a) {
    py::buffer_info b = a.request(true);
    fwht_inplace(static_cast<T*>(b.ptr), static_cast<std::size_t>(b.size));
}

}  // namespace

PYBIND11_MODULE(_bmmpy, m) {
    m.doc() = "bmmpy native module (B200 build): search and solver path on sm_100a";
    py::register_exception<MatrixError>(m, "MatrixError", PyExc_RuntimeError);

    py::class_<BitMatrix>(m, "BitMatrix")
        .def(py::init<>())
        .def(py::init<std::size_t, std::size_t>(), py::arg("rows"), py::arg("cols"))
        .def_property_readonly("rows", &BitMatrix::rows)
        .def_property_readonly("cols", &BitMatrix::cols)
        .def_property_readonly("shape",
                               [](const BitMatrix& b) { return py::make_tuple(b.rows(), b.cols()); })
        .def_property_readonly("stride_words", &BitMatrix::stride_words)
        .def_property_readonly("words_per_row", &BitMatrix::words_per_row)
        .def_property_readonly("total_words", &BitMatrix::total_words)
        .def("__len__", &BitMatrix::rows)
        .def("copy", [](const BitMatrix& b) { return BitMatrix(b); })
        .def("__getitem__",
             [](const BitMatrix& b, const py::tuple& i) {
                 const auto [r, c] = cell(i);
                 return b.get(r, c);
             })
        .def("__setitem__",
             [](BitMatrix& b, const py::tuple& i, bool v) {
                 const auto [r, c] = cell(i);
                 b.set(r, c, v);
             })
        .def("get", &BitMatrix::get, py::arg("row"), py::arg("col"))
        .def("set", &BitMatrix::set, py::arg("row"), py::arg("col"), py::arg("value"))
        .def("row_xor", &BitMatrix::row_xor, py::arg("target_row"), py::arg("source_row"))
        .def("row_popcount", &BitMatrix::row_popcount, py::arg("row"))
        .def("weight", &BitMatrix::weight)
        .def("row_window",
             [](BitMatrix& b, const std::vector<std::size_t>& rows) { return b.row_window(rows); },
             py::arg("rows"), py::keep_alive<0, 1>())
        .def("to_rows", &BitMatrix::to_rows)
        .def("__eq__", &BitMatrix::operator==)
        .def("__repr__",
             [](const BitMatrix& b) {
                 std::ostringstream s;
                 s << "BitMatrix(rows=" << b.rows() << ", cols=" << b.cols() << ")";
                 return s.str();
             })
        .def_static("from_rows", &BitMatrix::from_rows, py::arg("rows"))
        .def_static("identity", &BitMatrix::identity, py::arg("n"));

    py::class_<RowWindow>(m, "RowWindow")
        .def("__len__", &RowWindow::size)
        .def_property_readonly("size", &RowWindow::size)
        .def_property_readonly("cols", &RowWindow::cols)
        .def_property_readonly("shape",
                               [](const RowWindow& w) { return py::make_tuple(w.size(), w.cols()); })
        .def_property_readonly("rows", &RowWindow::global_rows)
        .def("row_popcount", &RowWindow::row_popcount, py::arg("local_row"))
        .def_property_readonly("total_weight", &RowWindow::total_weight)
        .def("assign_materialized", &RowWindow::assign_materialized, py::arg("rows"))
        .def("materialize", &RowWindow::materialize)
        .def("__repr__", [](const RowWindow& w) {
            std::ostringstream s;
            s << "RowWindow(size=" << w.size() << ", cols=" << w.cols() << ")";
            return s.str();
        });

    py::class_<Candidate>(m, "Candidate")
        .def(py::init<>())
        .def(py::init([](std::vector<std::uint64_t> mask, std::uint32_t weight) {
                 Candidate c;
                 c.mask = std::move(mask);
                 c.weight = weight;
                 return c;
             }),
             py::arg("mask"), py::arg("weight"))
        .def_readwrite("mask", &Candidate::mask)
        .def_readwrite("weight", &Candidate::weight)
        .def("__len__", &Candidate::popcount)
        .def("mask_u64", &Candidate::mask_u64)
        .def("mask_popcount", &Candidate::popcount)
        .def("selected_rows", &Candidate::selected_rows)
        .def_property_readonly("rows", &Candidate::selected_rows)
        .def("has_row",
             [](const Candidate& c, std::size_t r) {
                 return r / 64 < c.mask.size() && ((c.mask[r / 64] >> (r % 64)) & 1u);
             })
        .def("__contains__",
             [](const Candidate& c, std::size_t r) {
                 return r / 64 < c.mask.size() && ((c.mask[r / 64] >> (r % 64)) & 1u);
             })
        .def("__iter__",
             [](const Candidate& c) { return py::iter(py::cast(c.selected_rows())); })
        .def("__repr__",
             [](const Candidate& c) {
                 std::ostringstream s;
                 s << "Candidate(mask=0x" << std::hex << c.mask_u64() << std::dec
                   << ", weight=" << c.weight << ")";
                 return s.str();
             })
        .def_static("from_u64", &Candidate::from_u64, py::arg("mask"), py::arg("weight"));

    py::class_<FwhtSearch>(m, "FwhtSearch")
        .def(py::init([](std::size_t max_rows, std::size_t max_candidates) {
                 return FwhtSearch(FwhtSearchConfig{max_rows, max_candidates});
             }),
             py::kw_only(), py::arg("max_rows") = 16, py::arg("max_candidates") = 64)
        .def("search", &FwhtSearch::search, py::arg("window"))
        .def("name", &FwhtSearch::name);
    py::class_<MitmFwhtSearch>(m, "MitmFwhtSearch")
        .def(py::init([](std::size_t max_candidates) {
                 MitmFwhtSearchConfig c;
                 c.max_candidates = max_candidates;
                 return MitmFwhtSearch(c);
             }),
             py::kw_only(), py::arg("max_candidates") = 64)
        .def("search", &MitmFwhtSearch::search, py::arg("window"))
        .def("name", &MitmFwhtSearch::name);
    py::class_<BruteforceSearch>(m, "BruteforceSearch")
        .def(py::init([](std::size_t max_candidates, std::size_t chunk_bits) {
                 return BruteforceSearch(BruteforceSearchConfig{max_candidates, chunk_bits});
             }),
             py::kw_only(), py::arg("max_candidates") = 128, py::arg("chunk_bits") = 0)
        .def("search", &BruteforceSearch::search, py::arg("window"))
        .def("name", &BruteforceSearch::name);
    py::class_<CudaMitmFwhtSearch>(m, "CudaMitmFwhtSearch")
        .def(py::init([](std::size_t max_candidates, std::size_t low_bits) {
                 return CudaMitmFwhtSearch(CudaMitmFwhtSearchConfig{max_candidates, low_bits});
             }),
             py::kw_only(), py::arg("max_candidates") = 64, py::arg("low_bits") = 0)
        .def("search", &CudaMitmFwhtSearch::search, py::arg("window"))
        .def("name", &CudaMitmFwhtSearch::name);
    py::class_<CudaBruteforceSearch>(m, "CudaBruteforceSearch")
        .def(py::init([](std::size_t max_candidates, std::size_t chunk_bits) {
                 return CudaBruteforceSearch(CudaBruteforceSearchConfig{max_candidates, chunk_bits});
             }),
             py::kw_only(), py::arg("max_candidates") = 128, py::arg("chunk_bits") = 0)
        .def("search", &CudaBruteforceSearch::search, py::arg("window"))
        .def("name", &CudaBruteforceSearch::name);

    py::class_<CompactSplitWindow>(m, "CompactSplitWindow")
        .def_readonly("t", &CompactSplitWindow::t)
        .def_readonly("low_bits", &CompactSplitWindow::low_bits)
        .def_readonly("high_bits", &CompactSplitWindow::high_bits)
        .def_readonly("total_weight", &CompactSplitWindow::total_weight)
        .def_readonly("q", &CompactSplitWindow::q)
        .def_readonly("r", &CompactSplitWindow::r)
        .def_readonly("multiplicity", &CompactSplitWindow::multiplicity);
    m.def("build_compact_split_window",
          [](const RowWindow& w, std::size_t low_bits) {
              return build_compact_split_window(w, low_bits);
          },
          py::arg("window"), py::arg("low_bits"));
    m.def("run_cuda_mitm_fwht_search",
          [](const CompactSplitWindow& p, std::size_t k) {
              std::vector<std::pair<std::uint64_t, std::uint32_t>> out;
              for (const auto& r : run_cuda_mitm_fwht_search(p, k))
                  out.emplace_back(r.mask, r.weight);
              return out;
          },
          py::arg("prep"), py::arg("max_candidates"));

    py::class_<ExactBasisResult>(m, "ExactBasisResult")
        .def_readonly("input_rows", &ExactBasisResult::input_rows)
        .def_readonly("cols", &ExactBasisResult::cols)
        .def_readonly("rank", &ExactBasisResult::rank)
        .def_readonly("enumerated_states", &ExactBasisResult::enumerated_states)
        .def_readonly("total_weight", &ExactBasisResult::total_weight)
        .def_readonly("basis_masks", &ExactBasisResult::basis_masks)
        .def_readonly("basis_weights", &ExactBasisResult::basis_weights)
        .def_readonly("transform_matrix", &ExactBasisResult::transform_matrix)
        .def_readonly("basis_matrix", &ExactBasisResult::basis_matrix);
    py::class_<ExactBasisSolver>(m, "ExactBasisSolver")
        .def(py::init([](std::size_t max_rows, std::uint64_t max_states, std::size_t storage) {
                 return ExactBasisSolver(ExactBasisSolverConfig{max_rows, max_states, storage});
             }),
             py::kw_only(), py::arg("max_rows") = 24,
             py::arg("max_states") = (std::uint64_t{1} << 24) - 1,
             py::arg("max_storage_bytes") = std::size_t{128} << 20)
        .def("solve", &ExactBasisSolver::solve, py::arg("window"))
        .def("name", &ExactBasisSolver::name);

    m.def("fwht_inplace", &fwht_array<std::int32_t>, py::arg("data"));
    m.def("fwht_inplace", &fwht_array<std::int16_t>, py::arg("data"));

    py::class_<RuntimeFeatures>(m, "RuntimeFeatures")
        .def_readonly("avx2_compiled", &RuntimeFeatures::avx2_compiled)
        .def_readonly("avx2_available", &RuntimeFeatures::avx2_available)
        .def_readonly("cuda_compiled", &RuntimeFeatures::cuda_compiled)
        .def_readonly("cuda_available", &RuntimeFeatures::cuda_available)
        .def_readonly("parallel_compiled", &RuntimeFeatures::parallel_compiled)
        .def_readonly("parallel_enabled", &RuntimeFeatures::parallel_enabled)
        .def_readonly("max_threads", &RuntimeFeatures::max_threads)
        .def_readonly("bit_ops_backend", &RuntimeFeatures::bit_ops_backend)
        .def_readonly("fwht_backend", &RuntimeFeatures::fwht_backend);
    m.def("get_runtime_features", &get_runtime_features);
    m.def("get_version", &get_version);
}
