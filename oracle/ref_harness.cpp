// Test-infrastructure harness around the UNMODIFIED reference C++ sources.
//
// This file is part of the oracle: it is linked against the reference's own
// translation units (compiled in place by oracle/Makefile into oracle/_ref/)
// and exposes a handful of extern "C" shims so that the Python tests, the
// golden-fixture generator and bench.py's reference arm can call the
// reference implementation directly.  Nothing in the product links it.
//
// Every shim builds a reference `bmmpy::BitMatrix` from a packed row-major
// uint64 buffer (bit c of a row in word c/64, bit c%64; `stride` words per
// row) and calls the reference class named in its comment.
//
// Return convention: >= 0 on success (count of results written), negative on
// a reference exception: -1 std::invalid_argument, -2 std::overflow_error,
// -3 std::out_of_range, -4 std::logic_error, -5 other std::exception.

#include "bmmpy/apply/global_greedy_applier.hpp"
#include "bmmpy/apply/greedy_applier.hpp"
#include "bmmpy/core/bit_matrix.hpp"
#include "bmmpy/core/row_window.hpp"
#include "bmmpy/ga/genetic_algorithm.hpp"
#include "bmmpy/ga/island_model.hpp"
#include "bmmpy/ga/migration/bounded_channel.hpp"
#include "bmmpy/math/fwht.hpp"
#include "bmmpy/search/bruteforce_search.hpp"
#include "bmmpy/search/fwht_search.hpp"
#include "bmmpy/search/mitm_fwht_search.hpp"
#include "bmmpy/search/sa_selector.hpp"
#include "bmmpy/search/split_window_prep.hpp"
#include "bmmpy/solver/exact_basis_solver.hpp"

#include <chrono>
#include <sstream>
#include <string>
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <thread>
#include <vector>

namespace {

bmmpy::BitMatrix make_matrix(const std::uint64_t* words, std::size_t rows, std::size_t cols,
                             std::size_t stride) {
    bmmpy::BitMatrix m(rows, cols);
    const std::size_t wpr = m.words_per_row();
    for (std::size_t r = 0; r < rows; ++r) {
        std::uint64_t* dst = m.row_words(r);
        for (std::size_t w = 0; w < wpr; ++w)
            dst[w] = words[r * stride + w];
        // keep the reference's invariant: bits past `cols` are zero
        const std::size_t tail = cols % 64;
        if (tail != 0 && wpr != 0)
            dst[wpr - 1] &= (std::uint64_t{1} << tail) - 1;
    }
    return m;
}

thread_local std::string g_last_error;

template <typename Fn> long guarded(Fn&& fn) {
    try {
        g_last_error.clear();
        return fn();
    } catch (const std::invalid_argument& e) {
        g_last_error = e.what();
        return -1;
    } catch (const std::overflow_error& e) {
        g_last_error = e.what();
        return -2;
    } catch (const std::out_of_range& e) {
        g_last_error = e.what();
        return -3;
    } catch (const std::logic_error& e) {
        g_last_error = e.what();
        return -4;
    } catch (const bmmpy::MatrixError& e) {
        g_last_error = e.what();
        return -6;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -5;
    }
}

void copy_words(const bmmpy::BitMatrix& m, std::uint64_t* out, std::size_t stride) {
    const std::size_t wpr = m.words_per_row();
    for (std::size_t r = 0; r < m.rows(); ++r)
        for (std::size_t q = 0; q < stride; ++q)
            out[r * stride + q] = q < wpr ? m.row_words(r)[q] : 0;
}

long emit(const std::vector<bmmpy::Candidate>& cands, std::size_t cap, std::uint64_t* out_mask,
          std::uint32_t* out_weight) {
    const std::size_t n = cands.size() < cap ? cands.size() : cap;
    for (std::size_t i = 0; i < n; ++i) {
        out_mask[i] = cands[i].mask_u64();
        out_weight[i] = cands[i].weight;
    }
    return static_cast<long>(cands.size());
}

std::vector<std::size_t> to_rows(const std::size_t* win, std::size_t t) {
    return std::vector<std::size_t>(win, win + t);
}

} // namespace

extern "C" {

// bmmpy::fwht_inplace(int32_t*, size_t)
long refh_fwht_i32(std::int32_t* data, std::size_t n) {
    return guarded([&] {
        bmmpy::fwht_inplace(data, n);
        return 0L;
    });
}

// bmmpy::fwht_inplace(int16_t*, size_t)
long refh_fwht_i16(std::int16_t* data, std::size_t n) {
    return guarded([&] {
        bmmpy::fwht_inplace(data, n);
        return 0L;
    });
}

// bmmpy::FwhtSearch{max_rows, k}.search(window)
long refh_fwht_search(const std::uint64_t* words, std::size_t rows, std::size_t cols,
                      std::size_t stride, const std::size_t* win, std::size_t t,
                      std::size_t max_rows, std::size_t k, std::uint64_t* out_mask,
                      std::uint32_t* out_weight, std::size_t cap) {
    return guarded([&] {
        const auto m = make_matrix(words, rows, cols, stride);
        const auto w = m.row_window(to_rows(win, t));
        bmmpy::FwhtSearch s(bmmpy::FwhtSearchConfig{max_rows, k});
        return emit(s.search(w), cap, out_mask, out_weight);
    });
}

// bmmpy::MitmFwhtSearch{..., k}.search(window)
long refh_mitm_search(const std::uint64_t* words, std::size_t rows, std::size_t cols,
                      std::size_t stride, const std::size_t* win, std::size_t t, std::size_t k,
                      std::uint64_t* out_mask, std::uint32_t* out_weight, std::size_t cap) {
    return guarded([&] {
        const auto m = make_matrix(words, rows, cols, stride);
        const auto w = m.row_window(to_rows(win, t));
        bmmpy::MitmFwhtSearchConfig cfg;
        cfg.max_candidates = k;
        bmmpy::MitmFwhtSearch s(cfg);
        return emit(s.search(w), cap, out_mask, out_weight);
    });
}

// bmmpy::BruteforceSearch{k, chunk_bits}.search(window)
long refh_bruteforce_search(const std::uint64_t* words, std::size_t rows, std::size_t cols,
                            std::size_t stride, const std::size_t* win, std::size_t t,
                            std::size_t k, std::size_t chunk_bits, std::uint64_t* out_mask,
                            std::uint32_t* out_weight, std::size_t cap) {
    return guarded([&] {
        const auto m = make_matrix(words, rows, cols, stride);
        const auto w = m.row_window(to_rows(win, t));
        bmmpy::BruteforceSearch s(bmmpy::BruteforceSearchConfig{k, chunk_bits});
        return emit(s.search(w), cap, out_mask, out_weight);
    });
}

// bmmpy::build_compact_split_window(window, low_bits)
long refh_split_window(const std::uint64_t* words, std::size_t rows, std::size_t cols,
                       std::size_t stride, const std::size_t* win, std::size_t t,
                       std::size_t low_bits, std::uint64_t* q, std::uint64_t* r,
                       std::int32_t* mult, std::size_t cap, std::int32_t* total_weight) {
    return guarded([&] {
        const auto m = make_matrix(words, rows, cols, stride);
        const auto w = m.row_window(to_rows(win, t));
        const auto prep = bmmpy::build_compact_split_window(w, low_bits);
        *total_weight = prep.total_weight;
        const std::size_t n = prep.multiplicity.size();
        for (std::size_t i = 0; i < n && i < cap; ++i) {
            q[i] = prep.q[i];
            r[i] = prep.r[i];
            mult[i] = prep.multiplicity[i];
        }
        return static_cast<long>(n);
    });
}

// Per-target best combination (weight of row_target XOR rows in S, all S over
// `others`, S = 0 included, ties by smallest S) computed through the
// reference's own bmmpy::fwht_inplace on the signed column histogram.  Used to
// make golden vectors for the per-target workloads; the histogram fill is
// harness code, the transform is the reference's.
long refh_target_best_fwht(const std::uint64_t* words, std::size_t rows, std::size_t cols,
                           std::size_t stride, std::size_t target, const std::size_t* others,
                           std::size_t k, std::uint64_t* out_mask, std::uint32_t* out_weight) {
    return guarded([&] {
        if (k >= 31)
            throw std::invalid_argument("refh_target_best_fwht: k too large");
        const auto m = make_matrix(words, rows, cols, stride);
        const std::size_t n = std::size_t{1} << k;
        std::vector<std::int32_t> h(n, 0);
        for (std::size_t c = 0; c < cols; ++c) {
            std::size_t p = 0;
            for (std::size_t j = 0; j < k; ++j)
                if (m.get(others[j], c))
                    p |= std::size_t{1} << j;
            h[p] += m.get(target, c) ? -1 : 1;
        }
        bmmpy::fwht_inplace(h.data(), n);
        std::size_t best = 0;
        for (std::size_t s = 1; s < n; ++s)
            if (h[s] > h[best])
                best = s;
        *out_mask = best;
        *out_weight = static_cast<std::uint32_t>((static_cast<std::int64_t>(cols) - h[best]) / 2);
        return 1L;
    });
}

// Single-island bmmpy::ga::GeneticAlgorithm run; best_score after
// initialize() and after each generation is written to scores[0..gens].
// GeneticAlgorithmConfig fields, laid out like orc_ga_config (bmm_oracle.h);
// flags: 1 max_generations, 2 max_stale_generations, 4 target_total_weight.
struct refh_ga_config {
    std::size_t population_size, elite_count, num_parents, num_offspring, tournament_size;
    int enable_catastrophe;
    std::size_t catastrophe_threshold;
    double catastrophe_survival_rate, mutation_rate;
    unsigned flags;
    std::uint64_t max_generations, max_stale_generations, target_total_weight;
};

// The reference bmmpy::ga::GeneticAlgorithm: initialize(), then step() until
// done() or max_steps.  scores[g] = best_score() after g steps; best_masks
// (n * ceil(n/64) words) / best_weights receive best_individual().  Returns
// the number of steps; seconds receives the wall time.
long refh_ga_run(const std::uint64_t* words, std::size_t rows, std::size_t cols,
                 std::size_t stride, const std::size_t* win, std::size_t t,
                 const refh_ga_config* c, std::uint64_t seed, std::size_t max_steps,
                 std::uint64_t* scores, std::uint64_t* best_masks, std::uint32_t* best_weights,
                 double* seconds) {
    return guarded([&] {
        const auto m = make_matrix(words, rows, cols, stride);
        const auto w = m.row_window(to_rows(win, t));
        bmmpy::ga::GeneticAlgorithmConfig cfg;
        cfg.population_size = c->population_size;
        cfg.elite_count = c->elite_count;
        cfg.num_parents = c->num_parents;
        cfg.num_offspring = c->num_offspring;
        cfg.tournament_size = c->tournament_size;
        cfg.enable_catastrophe = c->enable_catastrophe != 0;
        cfg.catastrophe_threshold = c->catastrophe_threshold;
        cfg.catastrophe_survival_rate = c->catastrophe_survival_rate;
        cfg.mutation_rate = c->mutation_rate;
        cfg.seed = seed;
        if (c->flags & 1u)
            cfg.stop.max_generations = c->max_generations;
        if (c->flags & 2u)
            cfg.stop.max_stale_generations = c->max_stale_generations;
        if (c->flags & 4u)
            cfg.stop.target_total_weight = c->target_total_weight;
        bmmpy::ga::GeneticAlgorithm ga(cfg);
        const auto t0 = std::chrono::steady_clock::now();
        ga.initialize(w);
        scores[0] = ga.best_score();
        std::size_t g = 0;
        while (!ga.done() && g < max_steps) {
            ga.step();
            ++g;
            scores[g] = ga.best_score();
        }
        *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        const auto best = ga.best_individual();
        const std::size_t mw = (t + 63) / 64;
        for (std::size_t i = 0; i < best.size() && i < t; ++i) {
            for (std::size_t q = 0; q < mw; ++q)
                best_masks[i * mw + q] = q < best[i].mask.size() ? best[i].mask[q] : 0;
            best_weights[i] = best[i].weight;
        }
        return static_cast<long>(g);
    });
}

// The reference bmmpy::ga::IslandModel (one std::thread per island, shared
// BoundedChannel pool) run to completion with a wall-clock cap enforced by
// request_stop().  Returns the best score; seconds receives the wall time.
long refh_island_run(const std::uint64_t* words, std::size_t rows, std::size_t cols,
                     std::size_t stride, const std::size_t* win, std::size_t t,
                     std::size_t islands, std::size_t population, std::size_t interval,
                     std::uint64_t seed, std::size_t max_gens, std::uint64_t target_weight,
                     double cap_seconds, std::uint64_t* best_score, double* seconds) {
    return guarded([&] {
        const auto m = make_matrix(words, rows, cols, stride);
        const auto w = m.row_window(to_rows(win, t));
        bmmpy::ga::IslandModelConfig mc;
        for (std::size_t i = 0; i < islands; ++i) {
            bmmpy::ga::IslandSpec spec;
            spec.island_id = i;
            spec.migration.interval_generations = interval;
            spec.migration.export_count = 1;
            spec.migration.import_count = 1;
            mc.islands.push_back(spec);
        }
        auto factory = [&](const bmmpy::ga::IslandSpec& spec) {
            bmmpy::ga::GeneticAlgorithmConfig cfg;
            cfg.population_size = population;
            cfg.seed = seed + spec.island_id;
            cfg.stop.max_generations = max_gens;
            if (target_weight != 0)
                cfg.stop.target_total_weight = target_weight;
            return std::unique_ptr<bmmpy::ga::Algorithm>(new bmmpy::ga::GeneticAlgorithm(cfg));
        };
        bmmpy::ga::IslandModel model(
            mc, factory, std::make_unique<bmmpy::ga::migration::BoundedChannel>(128));
        const auto t0 = std::chrono::steady_clock::now();
        model.initialize(w);
        model.start();
        while (model.running()) {
            const auto snap = model.snapshot();
            bool all_done = true;
            for (const auto& is : snap.islands)
                all_done = all_done && is.finished;
            if (all_done)
                break;
            if (target_weight != 0 && snap.best_score <= target_weight)
                break;
            const double el =
                std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            if (el > cap_seconds)
                break;
            std::this_thread::sleep_for(std::chrono::milliseconds(20));
        }
        model.request_stop();
        model.wait();
        *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        *best_score = model.snapshot().best_score;
        return 0L;
    });
}

// GreedyApplier (stochastic, seed) / GlobalGreedyApplier (require_improvement)
// applied to the window of the matrix; the matrix words after the apply go to
// out_words (rows x stride); applied / improvement receive the ApplyResult.
// Candidate masks: n_cand x mw words.
long refh_apply(const std::uint64_t* words, std::size_t rows, std::size_t cols,
                std::size_t stride, const std::size_t* win, std::size_t t,
                const std::uint64_t* cand_masks, std::size_t mw, const std::uint32_t* cand_w,
                std::size_t n_cand, int global, std::uint64_t min_gain, int stochastic,
                std::uint64_t seed, int require_improvement, std::uint64_t* out_words,
                std::uint64_t* applied, std::uint64_t* improvement) {
    return guarded([&] {
        auto m = make_matrix(words, rows, cols, stride);
        auto w = m.row_window(to_rows(win, t));
        std::vector<bmmpy::Candidate> cands;
        for (std::size_t c = 0; c < n_cand; ++c) {
            std::vector<std::uint64_t> mask(cand_masks + c * mw, cand_masks + (c + 1) * mw);
            cands.emplace_back(std::move(mask), cand_w[c]);
        }
        bmmpy::ApplyResult r;
        if (global) {
            bmmpy::GlobalGreedyApplier a(require_improvement != 0);
            r = a.apply(w, cands);
        } else {
            bmmpy::GreedyApplier a(min_gain, stochastic != 0, seed);
            r = a.apply(w, cands);
        }
        const std::size_t wpr = m.words_per_row();
        for (std::size_t i = 0; i < rows; ++i)
            for (std::size_t q = 0; q < stride; ++q)
                out_words[i * stride + q] = q < wpr ? m.row_words(i)[q] : 0;
        *applied = r.applied_count;
        *improvement = r.weight_improvement;
        return 0L;
    });
}

// ExactBasisSolver({max_rows, max_states, max_storage_bytes}).solve(window).
// scalars[0..4] = input_rows, cols, rank, enumerated_states, total_weight;
// masks / weights get basis_masks / basis_weights (room for t); transform
// receives rank words (row k of transform_matrix, t <= 64 columns) and
// basis_words rank x stride words of basis_matrix.  Returns the rank.
long refh_exact_basis(const std::uint64_t* words, std::size_t rows, std::size_t cols,
                      std::size_t stride, const std::size_t* win, std::size_t t,
                      std::size_t max_rows, std::uint64_t max_states, std::size_t max_storage,
                      std::uint64_t* scalars, std::uint32_t* masks, std::uint32_t* weights,
                      std::uint64_t* transform, std::uint64_t* basis_words) {
    return guarded([&] {
        auto m = make_matrix(words, rows, cols, stride);
        auto w = m.row_window(to_rows(win, t));
        bmmpy::ExactBasisSolverConfig cfg;
        cfg.max_rows = max_rows;
        cfg.max_states = max_states;
        cfg.max_storage_bytes = max_storage;
        const bmmpy::ExactBasisResult r = bmmpy::ExactBasisSolver(cfg).solve(w);
        scalars[0] = r.input_rows;
        scalars[1] = r.cols;
        scalars[2] = r.rank;
        scalars[3] = r.enumerated_states;
        scalars[4] = r.total_weight;
        for (std::size_t k = 0; k < r.basis_masks.size(); ++k) {
            masks[k] = r.basis_masks[k];
            weights[k] = r.basis_weights[k];
        }
        for (std::size_t k = 0; k < r.transform_matrix.rows(); ++k)
            transform[k] = r.transform_matrix.cols() ? r.transform_matrix.row_words(k)[0] : 0;
        const std::size_t wpr = r.basis_matrix.words_per_row();
        for (std::size_t k = 0; k < r.basis_matrix.rows(); ++k)
            for (std::size_t q = 0; q < stride; ++q)
                basis_words[k * stride + q] = q < wpr ? r.basis_matrix.row_words(k)[q] : 0;
        return static_cast<long>(r.rank);
    });
}

// SASelector(config).select(matrix, window_size).  scalars[0..5] = score,
// accepted_moves, iterations_run, best_iteration, restart_index, seed;
// out_rows gets the rows (room for window_size).  Returns the row count.
long refh_sa_select(const std::uint64_t* words, std::size_t rows, std::size_t cols,
                    std::size_t stride, std::size_t window_size, std::size_t iterations,
                    std::size_t restarts, std::uint64_t seed, int score_policy,
                    std::size_t probe_samples, double p0, double cooling, double min_temp,
                    std::int64_t* scalars, std::size_t* out_rows) {
    return guarded([&] {
        auto m = make_matrix(words, rows, cols, stride);
        bmmpy::SASelectorConfig c;
        c.iterations = iterations;
        c.restarts = restarts;
        c.seed = seed;
        c.score_policy = score_policy == 0 ? bmmpy::WindowScorePolicyKind::PairwiseSynergy
                                           : bmmpy::WindowScorePolicyKind::HigherOrderSynergy;
        c.temperature_probe_samples = probe_samples;
        c.initial_acceptance_probability = p0;
        c.cooling_rate = cooling;
        c.min_temperature = min_temp;
        const bmmpy::SASelectionResult r = bmmpy::SASelector(c).select(m, window_size);
        scalars[0] = r.score;
        scalars[1] = static_cast<std::int64_t>(r.accepted_moves);
        scalars[2] = static_cast<std::int64_t>(r.iterations_run);
        scalars[3] = static_cast<std::int64_t>(r.best_iteration);
        scalars[4] = static_cast<std::int64_t>(r.restart_index);
        scalars[5] = static_cast<std::int64_t>(r.seed);
        for (std::size_t i = 0; i < r.rows.size(); ++i)
            out_rows[i] = r.rows[i];
        return static_cast<long>(r.rows.size());
    });
}

// Message of the last exception a shim caught on this thread.
const char* refh_last_error() { return g_last_error.c_str(); }

// BitMatrix::load_text over a string.  dims[0..1] = rows, cols; the words go
// to out (rows x stride) when cap_words allows.  Returns 0.
long refh_matrix_from_text(const char* text, std::size_t len, std::uint64_t* dims,
                           std::uint64_t* out, std::size_t stride, std::size_t cap_words) {
    return guarded([&] {
        std::istringstream in(std::string(text, len));
        const bmmpy::BitMatrix m = bmmpy::BitMatrix::load_text(in);
        dims[0] = m.rows();
        dims[1] = m.cols();
        if (m.rows() * stride <= cap_words)
            copy_words(m, out, stride);
        return 0L;
    });
}

// BitMatrix::save_text; returns the length (the text goes to out when it fits).
long refh_matrix_to_text(const std::uint64_t* words, std::size_t rows, std::size_t cols,
                         std::size_t stride, char* out, std::size_t cap) {
    return guarded([&] {
        auto m = make_matrix(words, rows, cols, stride);
        std::ostringstream o;
        m.save_text(o);
        const std::string t = o.str();
        if (t.size() <= cap)
            std::memcpy(out, t.data(), t.size());
        return static_cast<long>(t.size());
    });
}

// BitMatrix::hash into hex (65 bytes).
long refh_matrix_hash(const std::uint64_t* words, std::size_t rows, std::size_t cols,
                      std::size_t stride, char* hex) {
    return guarded([&] {
        const std::string h = make_matrix(words, rows, cols, stride).hash();
        std::memcpy(hex, h.c_str(), h.size() + 1);
        return 0L;
    });
}

long refh_matrix_save_binary(const char* path, const std::uint64_t* words, std::size_t rows,
                             std::size_t cols, std::size_t stride) {
    return guarded([&] {
        make_matrix(words, rows, cols, stride).save_binary(std::filesystem::path(path));
        return 0L;
    });
}

// BitMatrix::load_binary: dims and words as refh_matrix_from_text.
long refh_matrix_load_binary(const char* path, std::uint64_t* dims, std::uint64_t* out,
                             std::size_t stride, std::size_t cap_words) {
    return guarded([&] {
        const bmmpy::BitMatrix m = bmmpy::BitMatrix::load_binary(std::filesystem::path(path));
        dims[0] = m.rows();
        dims[1] = m.cols();
        if (m.rows() * stride <= cap_words)
            copy_words(m, out, stride);
        return 0L;
    });
}

} // extern "C"
