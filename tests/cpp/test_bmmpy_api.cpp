// C++ API test: the reference's class names and signatures (include/bmmpy/)
// over the B200 C ABI.  `host` mode runs everything that needs no GPU (layout,
// argument checks and the exception types the reference throws); `device`
// mode runs the searches and checks them against each other and against
// known answers.  Prints "ok" and exits 0 on success.
#include "bmmpy/bmmpy.hpp"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

int g_fail = 0;

#define EXPECT(cond)                                                                              \
    do {                                                                                          \
        if (!(cond)) {                                                                            \
            std::fprintf(stderr, "%s:%d: expected %s\n", __FILE__, __LINE__, #cond);              \
            ++g_fail;                                                                             \
        }                                                                                         \
    } while (0)

template <typename E, typename F>
bool throws(F&& f) {
    try {
        f();
    } catch (const E&) {
        return true;
    } catch (...) {
        return false;
    }
    return false;
}

bmmpy::BitMatrix random_matrix(std::size_t rows, std::size_t cols, double p, unsigned seed) {
    std::mt19937_64 rng(seed);
    std::bernoulli_distribution bit(p);
    bmmpy::BitMatrix m(rows, cols);
    for (std::size_t r = 0; r < rows; ++r)
        for (std::size_t c = 0; c < cols; ++c)
            m.set(r, c, bit(rng));
    return m;
}

std::vector<std::pair<std::uint64_t, std::uint32_t>> pairs(const std::vector<bmmpy::Candidate>& v) {
    std::vector<std::pair<std::uint64_t, std::uint32_t>> out;
    for (const auto& c : v)
        out.emplace_back(c.mask_u64(), c.weight);
    return out;
}

std::vector<std::size_t> iota(std::size_t a, std::size_t n) {
    std::vector<std::size_t> v(n);
    for (std::size_t i = 0; i < n; ++i)
        v[i] = a + i;
    return v;
}

void host_tests() {
    using namespace bmmpy;
    // layout: stride padded to 4 words, bits past cols stay zero
    BitMatrix m(3, 130);
    EXPECT(m.words_per_row() == 3 && m.stride_words() == 4);
    m.set(1, 129, true);
    m.set(2, 0, true);
    EXPECT(m.get(1, 129) && !m.get(1, 128) && m.weight() == 2);
    EXPECT(m.row_words(1)[2] == (std::uint64_t{1} << 1));
    EXPECT(throws<std::out_of_range>([&] { m.get(3, 0); }));
    EXPECT(throws<std::out_of_range>([&] { m.set(0, 130, true); }));
    EXPECT(throws<std::out_of_range>([&] { m.row_window({0, 3}); }));
    BitMatrix r = matrix_from_rows({"1100", "0110", "0011"});
    EXPECT(r.to_rows() == (std::vector<std::string>{"1100", "0110", "0011"}));
    EXPECT(BitMatrix::identity(5).weight() == 5);
    EXPECT(throws<std::invalid_argument>([] { matrix_from_rows({"10", "1"}); }));

    // window: borrowed rows, active-column total weight, materialize
    RowWindow w = r.row_window({0, 2});
    EXPECT(w.size() == 2 && w.total_weight() == 4 && w.weight() == 4);
    EXPECT(w.materialize().to_rows() == (std::vector<std::string>{"1100", "0011"}));
    const BitMatrix& cr = r;
    RowWindow cw = cr.row_window({1});
    EXPECT(!cw.is_mutable() && throws<std::logic_error>([&] { cw.row_xor(0, 0); }));

    // candidates
    const Candidate c = Candidate::from_u64(0b10110, 7);
    EXPECT(c.mask_u64() == 0b10110 && c.popcount() == 3);
    EXPECT(c.selected_rows() == (std::vector<std::size_t>{1, 2, 4}));
    EXPECT(candidate_less(Candidate::from_u64(9, 1), Candidate::from_u64(3, 2)));
    EXPECT(candidate_less(Candidate::from_u64(3, 2), Candidate::from_u64(9, 2)));

    // split-window prep: distinct patterns ascending with multiplicities
    const BitMatrix sp = matrix_from_rows({"1101", "0111", "1001"});
    const CompactSplitWindow prep = build_compact_split_window(sp.row_window({0, 1, 2}), 1);
    // columns: 0 -> 0b101, 1 -> 0b011, 2 -> 0b010, 3 -> 0b111
    EXPECT(prep.total_weight == 4 && prep.high_bits == 2);
    EXPECT(prep.q == (std::vector<std::uint64_t>{1, 1, 2, 3}));
    EXPECT(prep.r == (std::vector<std::uint64_t>{0, 1, 1, 1}));
    EXPECT(prep.multiplicity == (std::vector<std::int32_t>{1, 1, 1, 1}));
    EXPECT(throws<std::invalid_argument>([&] { build_compact_split_window(sp.row_window({0}), 2); }));

    // checks that precede any device work
    BitMatrix big = random_matrix(70, 512, 0.5, 1);
    FwhtSearch fw(FwhtSearchConfig{4, 8});
    EXPECT(fw.search(big.row_window(iota(0, 5))).empty());  // t > max_rows: no result
    EXPECT(std::string(fw.name()) == "fwht");
    CudaBruteforceSearch cb;
    EXPECT(throws<std::invalid_argument>([&] { cb.search(big.row_window(iota(0, 10))); }));
    EXPECT(throws<std::invalid_argument>([&] { cb.search(big.row_window(iota(0, 65))); }));
    CudaBruteforceSearch cb200(CudaBruteforceSearchConfig{200, 0});
    EXPECT(throws<std::invalid_argument>([&] { cb200.search(big.row_window(iota(0, 16))); }));
    BitMatrix narrow = random_matrix(20, 100, 0.5, 2);
    EXPECT(throws<std::invalid_argument>([&] { cb.search(narrow.row_window(iota(0, 16))); }));
    CudaMitmFwhtSearch cm;
    BitMatrix heavy = random_matrix(20, 40000, 0.5, 3);
    EXPECT(throws<std::invalid_argument>([&] { cm.search(heavy.row_window(iota(0, 16))); }));
    CudaMitmFwhtSearch cm_low(CudaMitmFwhtSearchConfig{64, 16});
    EXPECT(throws<std::invalid_argument>([&] { cm_low.search(heavy.row_window(iota(0, 17))); }));
    std::int32_t three[3] = {1, 2, 3};
    EXPECT(throws<std::invalid_argument>([&] { fwht_inplace(three, 3); }));
    EXPECT(throws<std::invalid_argument>(
        [] { run_cuda_mitm_fwht_search(CompactSplitWindow{3, 1, 2, 1, {1}, {0}, {1}}, 200); }));
    EXPECT(get_runtime_features().cuda_compiled);
}

void device_tests() {
    using namespace bmmpy;
    std::int32_t a[4] = {1, 2, 3, 4};
    fwht_inplace(a, 4);
    EXPECT(a[0] == 10 && a[1] == -2 && a[2] == -4 && a[3] == 0);
    std::int16_t b[2] = {32767, 1};
    fwht_inplace(b, 2);  // wrapping two's complement
    EXPECT(b[0] == -32768 && b[1] == 32766);

    BitMatrix m = random_matrix(40, 600, 0.3, 11);
    const RowWindow w = m.row_window(iota(5, 18));
    const auto want = pairs(BruteforceSearch(BruteforceSearchConfig{40, 0}).search(w));
    EXPECT(want.size() == 40);
    EXPECT(pairs(FwhtSearch(FwhtSearchConfig{18, 40}).search(w)) == want);
    MitmFwhtSearchConfig mc;
    mc.max_candidates = 40;
    EXPECT(pairs(MitmFwhtSearch(mc).search(w)) == want);
    std::vector<Searcher*> all;
    FwhtSearch s1(FwhtSearchConfig{18, 40});
    MitmFwhtSearch s2(mc);
    all.push_back(&s1);
    all.push_back(&s2);
    for (Searcher* s : all)
        EXPECT(pairs(s->search(w)) == want);

    // the reference's launch seams
    const CompactSplitWindow prep = build_compact_split_window(w, 8);
    const auto seam = run_cuda_mitm_fwht_search(prep, 40);
    EXPECT(seam.size() == want.size());
    for (std::size_t i = 0; i < seam.size() && i < want.size(); ++i)
        EXPECT(seam[i].mask == want[i].first && seam[i].weight == want[i].second);
    BitMatrix m512 = random_matrix(24, 512, 0.4, 12);
    const RowWindow w16 = m512.row_window(iota(2, 16));
    CudaBruteforcePlan plan;
    plan.rows = 16;
    plan.cols = 512;
    plan.words_per_row = 8;
    for (std::size_t i = 0; i < 16; ++i)
        plan.row_words.insert(plan.row_words.end(), w16.row_words(i), w16.row_words(i) + 8);
    const auto bf = run_cuda_bruteforce_search(plan, 32);
    const auto bf_want = pairs(BruteforceSearch(BruteforceSearchConfig{32, 0}).search(w16));
    EXPECT(bf.size() == bf_want.size());
    for (std::size_t i = 0; i < bf.size() && i < bf_want.size(); ++i)
        EXPECT(bf[i].mask == bf_want[i].first && bf[i].weight == bf_want[i].second);
    EXPECT(pairs(CudaBruteforceSearch(CudaBruteforceSearchConfig{32, 0}).search(w16)) == bf_want);
    EXPECT(pairs(CudaMitmFwhtSearch(CudaMitmFwhtSearchConfig{32, 0}).search(w16)) == bf_want);

    // exact basis: the identity's basis is its rows, weight 1 each
    const BitMatrix id = BitMatrix::identity(6);
    const ExactBasisResult eb = ExactBasisSolver().solve(id.row_window(iota(0, 6)));
    EXPECT(eb.rank == 6 && eb.total_weight == 6 && eb.basis_matrix.weight() == 6);
    EXPECT(get_runtime_features().cuda_available);
}

}  // namespace

int main(int argc, char** argv) {
    const std::string mode = argc > 1 ? argv[1] : "host";
    host_tests();
    if (mode == "device")
        device_tests();
    if (g_fail) {
        std::fprintf(stderr, "%d failure(s)\n", g_fail);
        return 1;
    }
    std::printf("ok\n");
    return 0;
}
