/* CPU oracle: a plain-C restatement of the reference's weight-minimisation
 * hot path (MortimerDe/bmmpy v0.5.3).  TEST INFRASTRUCTURE ONLY: the tests,
 * __graft_entry__.smoke() and bench.py's CPU baseline leg use it as the
 * checker; the product never links or calls it.
 *
 * Parity is pinned two ways (see tests/test_oracle.py): against the reference
 * library itself compiled from its own sources (oracle/_ref/libbmmref.so) and
 * against the reference's known-answer tests, committed as golden vectors
 * under tests/golden/.
 *
 * Matrix layout everywhere: row-major uint64 words, bit c of a row in word
 * c>>6 at bit c&63, `stride` words between rows, bits past `cols` zero
 * (include/bmmpy/core/bit_matrix.hpp:27-127, src/core/bit_matrix.cpp:67-72).
 *
 * Error returns mirror the reference exceptions: ORC_EINVAL for
 * std::invalid_argument, ORC_EOVERFLOW for std::overflow_error.
 */
#ifndef BMM_ORACLE_H
#define BMM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_EINVAL (-1)
#define ORC_EOVERFLOW (-2)

/* xorshift64 (13, 7, 17); seed 0 maps to 0x9E3779B97F4A7C15
 * (include/bmmpy/core/detail/xorshift64.hpp:10-40). */
uint64_t orc_xs_next(uint64_t* state);
uint64_t orc_xs_seed(uint64_t seed);

/* Seeded synthetic instance: Bernoulli(p) fill (row-major, column inner,
 * bit = unit_double < p), then `scrambles` row XORs r_i ^= r_j with
 * i = next_index(rows), j redrawn until j != i.  Returns the planted weight
 * (weight before scrambling). */
uint64_t orc_gen_instance(uint64_t* words, size_t rows, size_t cols, size_t stride, double p,
                          uint64_t seed, size_t scrambles);

/* Unnormalised in-place Walsh-Hadamard transform with wrapping add/sub
 * (src/math/fwht.cpp:28-57, src/math/fwht_scalar.cpp:19-39). */
int orc_fwht_i32(int32_t* data, size_t n);
int orc_fwht_i16(int16_t* data, size_t n);

/* FwhtSearch::search (src/search/fwht_search.cpp:34-132): top-k (weight asc,
 * mask asc) over every nonzero mask of the window rows `win[0..t)`.  Writes
 * min(count, cap) results; returns count or a negative error. */
long orc_fwht_search(const uint64_t* words, size_t stride, size_t cols, const size_t* win,
                     size_t t, size_t max_rows, size_t k, uint64_t* out_mask,
                     uint32_t* out_weight, size_t cap);

/* build_compact_split_window (src/search/split_window_prep.cpp:42-137):
 * unique column patterns sorted ascending, split into q = p >> low and
 * r = p & lowmask, with multiplicities.  Returns the unique count. */
long orc_split_window(const uint64_t* words, size_t stride, size_t cols, const size_t* win,
                      size_t t, size_t low_bits, uint64_t* q, uint64_t* r, int32_t* mult,
                      size_t cap, int32_t* total_weight);

/* MitmFwhtSearch::search (src/search/mitm_fwht_search.cpp:56-60,91-186,233-322). */
long orc_mitm_search(const uint64_t* words, size_t stride, size_t cols, const size_t* win,
                     size_t t, size_t k, uint64_t* out_mask, uint32_t* out_weight, size_t cap);

/* BruteforceSearch::search (src/search/bruteforce_search.cpp:113-170,300-329). */
long orc_bruteforce_search(const uint64_t* words, size_t stride, size_t cols, const size_t* win,
                           size_t t, size_t k, size_t chunk_bits, uint64_t* out_mask,
                           uint32_t* out_weight, size_t cap);

/* Per-target best XOR combination: minimise popcount(row[target] ^ XOR of
 * rows others[j] for j in S) over all S (S = 0 included).  Reflected-Gray
 * enumeration as in the reference's sweep (src/search/bruteforce_search.cpp:
 * 157-169).  tiebreak 0: smallest S (the reference's (weight, mask) order,
 * since its window mask is (S<<1)|1); tiebreak 1: smallest Gray index. */
int orc_target_best_gray(const uint64_t* words, size_t stride, size_t cols, size_t target,
                         const size_t* others, size_t k, int tiebreak, uint64_t* best_mask,
                         uint32_t* best_weight);

/* The same answer (tiebreak 0) through the signed column histogram and one
 * 2^k-point transform: weight(S) = (cols - WHT[S]) / 2. */
int orc_target_best_fwht(const uint64_t* words, size_t stride, size_t cols, size_t target,
                         const size_t* others, size_t k, uint64_t* best_mask,
                         uint32_t* best_weight);

/* Genetic-algorithm kernels (src/ga/genetic_algorithm_internal.hpp:41-103,
 * src/ga/genetic_algorithm_operators.cpp:100-192).  An individual is n
 * candidate masks of mw = ceil(n/64) words each over the n window rows. */
uint32_t orc_eval_cand_weight(const uint64_t* words, size_t stride, size_t cols,
                              const size_t* win, size_t n, const uint64_t* mask, size_t mw);

/* GeneticAlgorithm::mutate: count = max(1, floor(n*rate)) pair draws (i, j)
 * from the xorshift state; i != j: mask_i ^= mask_j and re-score i. */
void orc_mutate(const uint64_t* words, size_t stride, size_t cols, const size_t* win, size_t n,
                uint64_t* masks, uint32_t* weights, size_t mw, double rate, uint64_t* rng_state);

/* GeneticAlgorithm::local_improvement: materialise, then up to 10 greedy
 * pairwise passes. */
void orc_local_improvement(const uint64_t* words, size_t stride, size_t cols, const size_t* win,
                           size_t n, uint64_t* masks, uint32_t* weights, size_t mw);

/* GeneticAlgorithm::crossover: parents individuals of n candidates laid out
 * one after another; the child's masks/weights (unit padding weighs 1). */
void orc_crossover(size_t n, size_t parents, const uint64_t* parent_masks,
                   const uint32_t* parent_weights, uint64_t* child_masks,
                   uint32_t* child_weights);

/* GeneticAlgorithmConfig (include/bmmpy/ga/genetic_algorithm.hpp:17-29);
 * flags: 1 max_generations, 2 max_stale_generations, 4 target_total_weight. */
typedef struct orc_ga_config {
    size_t population_size, elite_count, num_parents, num_offspring, tournament_size;
    int enable_catastrophe;
    size_t catastrophe_threshold;
    double catastrophe_survival_rate, mutation_rate;
    unsigned flags;
    uint64_t max_generations, max_stale_generations, target_total_weight;
} orc_ga_config;

/* initialize() then step() until done() or max_steps steps.  scores[g] is
 * best_score() after g steps (scores[0] after initialize); best_masks /
 * best_weights receive best_individual().  Returns the number of steps. */
long orc_ga_run(const uint64_t* words, size_t stride, size_t cols, const size_t* win, size_t n,
                const orc_ga_config* cfg, uint64_t seed, uint64_t max_steps, uint64_t* scores,
                uint64_t* best_masks, uint32_t* best_weights);

/* ExactBasisSolver::solve (src/solver/exact_basis_solver.cpp:58-157) without
 * its configurable caps: every nonzero combination of the t <= 32 window rows
 * in reflected-Gray order, bucketed by weight, offered in that order to a
 * greedy GF(2) basis until the window's rank is reached.  masks / weights get
 * the accepted combinations (room for t); *total their total weight.
 * Returns the rank, -1 when t > 32, -2 when memory runs out. */
long orc_exact_basis(const uint64_t* words, size_t stride, size_t cols, const size_t* win,
                     size_t t, uint32_t* masks, uint32_t* weights, uint64_t* total);

/* Weight histogram of the 2^t - 1 nonzero combinations (counts[0..cols]). */
int orc_basis_weight_counts(const uint64_t* words, size_t stride, size_t cols, const size_t* win,
                            size_t t, uint64_t* counts);

/* SASelector::select (src/search/sa_selector.cpp:10-75; restarts
 * src/search/sa_selector_pairwise.cpp:118-170 and
 * src/search/sa_selector_higher_order.cpp:171-225).  score_policy 0 pairwise,
 * 1 higher order.  scalars[0..5] = score, accepted_moves, iterations_run,
 * best_iteration, restart_index, seed; out_rows gets the sorted rows.
 * Returns the row count, -1 for an invalid argument. */
long orc_sa_select(const uint64_t* words, size_t stride, size_t rows, size_t cols,
                   size_t window_size, uint64_t iterations, uint64_t restarts, uint64_t seed,
                   int score_policy, uint64_t probe_samples, double p0, double cooling,
                   double min_temp, int64_t* scalars, size_t* out_rows);

#ifdef __cplusplus
}
#endif

#endif
