/* bmm_b200.h -- C ABI of the B200 (sm_100a) weight-minimisation kernels.
 *
 * This is the drop-in boundary for bmmpy's search / FWHT / GA hot path.  It
 * replaces the reference's launch seams and the bodies of its searcher
 * classes (MortimerDe/bmmpy v0.5.3; citations are paths in that project):
 *
 *   bmm_fwht_search      FwhtSearch::search          src/search/fwht_search.cpp:34-132
 *   bmm_mitm_search      MitmFwhtSearch::search      src/search/mitm_fwht_search.cpp:267-322
 *                        CudaMitmFwhtSearch::search  src/search/cuda_mitm_fwht_search.cpp:123-180
 *                        run_cuda_mitm_fwht_search   include/bmmpy/search/cuda_mitm_fwht_launch.hpp:15-16
 *   bmm_gray_search      BruteforceSearch::search    src/search/bruteforce_search.cpp:300-329
 *                        CudaBruteforceSearch::search src/search/cuda_bruteforce_search.cpp:38-103
 *                        run_cuda_bruteforce_search  include/bmmpy/search/cuda_bruteforce_launch.hpp:22-23
 *   bmm_fwht_i32/_i16    fwht_inplace                include/bmmpy/math/fwht.hpp:8-9
 *   bmm_runtime_features get_runtime_features        include/bmmpy/stub.hpp:19-21
 *   bmm_gray_targets / bmm_fwht_targets / bmm_batch_fwht_targets
 *                        per-target form of the searches above: for target
 *                        row i and k other rows, the reference window search
 *                        over [i, o_1..o_k] restricted to masks with bit 0 set
 *                        (best = (S << 1) | 1 in the reference's mask order).
 *   bmm_ga_*             GeneticAlgorithm / IslandModel (whole generations on the
 *                        device) and their operators
 *                        src/ga/genetic_algorithm_lifecycle.cpp:16-200,
 *                        src/ga/genetic_algorithm_operators.cpp:15-192,
 *                        src/ga/genetic_algorithm_internal.hpp:41-103,
 *                        src/ga/island.cpp:149-228.
 *   bmm_sa_select        SASelector::select  src/search/sa_selector.cpp:10-75,
 *                        src/search/sa_selector_pairwise.cpp:21-172,
 *                        src/search/sa_selector_higher_order.cpp:11-227.
 *   bmm_matrix_*         BitMatrix text / binary IO and hash
 *                        src/core/bit_matrix_io.cpp:34-175,
 *                        src/core/bit_matrix_hash.cpp:30-58.
 *   bmm_exact_basis      ExactBasisSolver::solve
 *                        src/solver/exact_basis_solver.cpp:58-157,
 *                        include/bmmpy/solver/exact_basis_solver.hpp:12-43.
 *
 * Conventions
 *  - Every function returns an int status (BMM_OK == 0, negative on error)
 *    and never throws; bmm_last_error() gives the calling thread's message.
 *    The status classes map to the reference's exception types:
 *    BMM_EINVAL -> std::invalid_argument, BMM_EOVERFLOW -> std::overflow_error,
 *    BMM_ECUDA / BMM_ENODEV / BMM_ETIMEOUT / BMM_ERUNTIME -> std::runtime_error,
 *    BMM_EMATRIX -> bmmpy::MatrixError (a std::runtime_error).
 *  - A matrix is row-major packed uint64 words: bit c of a row sits in word
 *    c >> 6 at bit c & 63; `stride` words separate rows; bits at and past
 *    `cols` must be zero (the reference BitMatrix layout).  A window is a list
 *    of `t` row indices `win[0..t)`; mask bit j selects win[j].
 *  - Functions without a suffix take HOST pointers, copy to the device,
 *    run and copy back synchronously (the reference's calling convention).
 *    Functions ending in _dev take DEVICE pointers and a cudaStream_t passed
 *    as void*, are asynchronous, and never synchronise the device.
 *  - Results are ordered by (weight ascending, mask ascending) -- the
 *    reference's candidate_less -- and mask 0 is never reported by the
 *    window searches.
 *  - Calls from different host threads are safe; each thread owns its own
 *    device workspace and stream per device.
 */
#ifndef BMM_B200_H
#define BMM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define BMM_API __attribute__((visibility("default")))
#else
#define BMM_API
#endif

#define BMM_OK 0
#define BMM_EINVAL (-1)
#define BMM_EOVERFLOW (-2)
#define BMM_ECUDA (-3)
#define BMM_ENODEV (-4)
#define BMM_ETIMEOUT (-5)
#define BMM_ENOMEM (-6)
#define BMM_ERUNTIME (-7)
#define BMM_EMATRIX (-8)

/* DeviceTopKEntry of include/bmmpy/search/cuda_launch_topk.cuh:11-14 (16 B). */
typedef struct bmm_candidate {
    uint64_t mask;
    uint32_t weight;
    uint32_t reserved;
} bmm_candidate;

/* RuntimeFeatures (include/bmmpy/stub.hpp:7-17), CUDA part. */
typedef struct bmm_features {
    int cuda_compiled;
    int cuda_available;
    int device_count;
    int sm_count;      /* of the current device, 0 if none */
    int cc_major;
    int cc_minor;
    char device_name[64];
} bmm_features;

/* Seeded synthetic instance (host memory, no device work): xorshift64
 * (13, 7, 17; seed 0 -> 0x9E3779B97F4A7C15, include/bmmpy/core/detail/
 * xorshift64.hpp:10-40) Bernoulli(p) fill, row-major with the column inner,
 * bit = (next >> 11) * 2^-53 < p; then `scrambles` row XORs r_i ^= r_j with
 * i = next % rows and j redrawn until j != i.  Returns the weight before
 * scrambling (the planted weight). */
BMM_API uint64_t bmm_gen_instance(uint64_t* words, size_t rows, size_t cols, size_t stride,
                                  double p, uint64_t seed, size_t scrambles);

/* Autotuner hook for the per-target Gray-code kernel (no reference
 * counterpart): hs_blocks = carry-save blocks of 8 words per 64-word lane
 * (0, 2-6, 8; -1 = built-in policy), chunk_bits = Gray-swept low bits per
 * prefix (-1 = built-in policy).  Process-wide; results never change, only
 * speed. */
BMM_API int bmm_gray_tune(int hs_blocks, int chunk_bits);
/* Lanes per prefix of the per-target Gray kernel for rows of 33-64 words:
 * 1 (a lane holds the whole row) or 2 (a lane pair, 32 words each, more
 * warps per SM); -1 = built-in policy.  Results never change, only speed. */
BMM_API int bmm_gray_tune_lanes(int lanes);
/* Per-shape autotuner entries (no reference counterpart): for per-target
 * Gray searches of rows of words_per_row words against k others, use
 * hs_blocks / chunk_bits / lanes (each -1 = built-in policy; same ranges as
 * above, at most 4 blocks with lanes = 2).  The process-wide settings of
 * bmm_gray_tune / bmm_gray_tune_lanes, where set, take precedence.
 * bmm_spectrum_tune_shape records the spectrum split (low_bits, see
 * bmm_spectrum_topk_slices_dev) for t-row windows, 15 <= t <= 40; a
 * bmm_spectrum_tune setting takes precedence.  bmm_tune_reset drops every
 * entry and setting.  Results never change, only speed. */
BMM_API int bmm_gray_tune_shape(size_t words_per_row, size_t k, int hs_blocks, int chunk_bits,
                                int lanes);
BMM_API int bmm_spectrum_tune_shape(size_t t, int low_bits);
BMM_API int bmm_tune_reset(void);

/* ---- batched per-target searches (thousands of uneven instances) ----
 * Instance i is a rows x cols matrix stored at words + word_offset with
 * `stride` words per row; every row r is a target searched against the k
 * others (r + 1 + j) mod rows, j < k (1 <= k <= min(16, rows - 1)); its
 * result goes to best_mask/best_weight[out_offset + r] (S over the others,
 * ties to the smallest S, as bmm_gray_targets).  One persistent launch with
 * a global work queue; the plan orders items longest first and picks per
 * shape the transform (cols <= 32767) or the Gray enumeration (cols <= 512)
 * by the policy below. */
typedef struct bmm_instance {
    uint64_t word_offset;
    uint32_t rows;
    uint32_t cols;
    uint32_t stride;
    uint32_t k;
    uint64_t out_offset;
} bmm_instance;

typedef struct bmm_batch bmm_batch;

/* Plan a batch from host descriptors (allocates the plan's device copy). */
BMM_API int bmm_batch_create(const bmm_instance* inst, size_t n_inst, bmm_batch** out);
/* items, output length, items per method {transform k=16, transform k<16,
 * Gray} of a plan. */
BMM_API int bmm_batch_info(const bmm_batch* b, long long* n_items, size_t* n_out, int* methods3);
/* Run on device buffers (asynchronous on `stream`).  The work-queue reset and
 * the kernel are a CUDA graph captured on the first run and replayed; new
 * buffer pointers trigger one re-capture. */
BMM_API int bmm_batch_run(bmm_batch* b, const uint64_t* d_words, uint64_t* d_best_mask,
                          uint32_t* d_best_weight, void* stream);
BMM_API int bmm_batch_destroy(bmm_batch* b);
/* Host-buffer convenience: plan, upload, run, download (synchronous). */
BMM_API int bmm_batch_targets(const uint64_t* words, size_t n_words, const bmm_instance* inst,
                              size_t n_inst, uint64_t* best_mask, uint32_t* best_weight);
/* Autotuner hook (no reference counterpart): k = 16 items whose rows have at
 * most gray_max_words words (0..8) use the Gray enumeration instead of the
 * transform (default 0: the transform everywhere); force_method (-1 none,
 * 0/1 transform, 2 Gray) overrides where legal.  Applies to plans created
 * afterwards; results never change. */
BMM_API int bmm_batch_policy(int gray_max_words, int force_method);

/* Roofline probe for the Gray-code kernels: runs a register-only kernel with
 * the per-word work of one Gray step (64-bit XOR, 64-bit POPC, add) over the
 * whole device and returns its rate in 64-bit words per second.  No
 * reference counterpart (measurement aid). */
BMM_API int bmm_probe_xor_popc(double* words_per_second);

BMM_API const char* bmm_last_error(void);
BMM_API const char* bmm_version(void);
BMM_API int bmm_runtime_features(bmm_features* out);

/* ---- FWHT (fwht_inplace, include/bmmpy/math/fwht.hpp:8-9) ----
 * Unnormalised Walsh-Hadamard transform in natural order with wrapping
 * two's-complement add/sub; n must be a power of two (BMM_EINVAL otherwise);
 * n <= 1 is a no-op. */
BMM_API int bmm_fwht_i32(int32_t* data, size_t n);
BMM_API int bmm_fwht_i16(int16_t* data, size_t n);
BMM_API int bmm_fwht_i32_dev(int32_t* d_data, size_t n, void* stream);

/* ---- window searches ----
 * `out` holds room for `k` candidates; *out_count receives the number written
 * (min(k, 2^t - 1)).  An empty result (t == 0, k == 0, cols == 0, or
 * t > max_rows for bmm_fwht_search) is BMM_OK with *out_count == 0, as in the
 * reference. */

/* FwhtSearch: t <= min(max_rows, 33) (the 2^t int32 spectrum is built in
 * device memory: 32 GB at t = 33).  BMM_EOVERFLOW when cols exceeds INT32_MAX
 * (the reference's total-weight limit, fwht_search.cpp:77-87). */
BMM_API int bmm_fwht_search(const uint64_t* words, size_t stride, size_t cols, const uint32_t* win,
                    size_t t, size_t max_rows, size_t k, bmm_candidate* out, size_t* out_count);

/* Gray-code exhaustive search (BruteforceSearch / CudaBruteforceSearch).
 * 1 <= t <= 64 (the enumeration must finish: t <= 44 in practice),
 * k <= 1024, chunk_bits 0 (auto) or in [1, t] (as BruteforceSearch). */
BMM_API int bmm_gray_search(const uint64_t* words, size_t stride, size_t cols, const uint32_t* win,
                    size_t t, size_t k, size_t chunk_bits, bmm_candidate* out,
                    size_t* out_count);

/* Meet-in-the-middle search (MitmFwhtSearch / CudaMitmFwhtSearch): the same
 * exact top-k as bmm_fwht_search for 1 <= t <= 40, k <= 1024.  The low
 * min(t, 33) bits form a spectrum in device memory; bits above 33 are
 * enumerated.  low_bits is accepted for interface compatibility (0 or in
 * [1, t - 1]) and does not change the result.  Exact in int32 for any
 * column count below 2^31 (no int16 limit). */
BMM_API int bmm_mitm_search(const uint64_t* words, size_t stride, size_t cols, const uint32_t* win,
                            size_t t, size_t k, size_t low_bits, bmm_candidate* out,
                            size_t* out_count);

/* ---- per-target searches ----
 * For each of n_targets targets: minimise popcount(row[targets[i]] ^ XOR of
 * rows others[i*k + j] for j in S) over all S in [0, 2^k) (S = 0 included).
 * best_mask[i] = S, best_weight[i] = that weight.  Ties: tiebreak 0 = the
 * smallest S (the reference's mask order), 1 = the smallest reflected-Gray
 * index of S.  Gray: k <= 40; FWHT: k <= 16 and cols <= 16383. */
BMM_API int bmm_gray_targets(const uint64_t* words, size_t rows, size_t stride, size_t cols,
                     const uint32_t* targets, const uint32_t* others, size_t n_targets, size_t k,
                     int tiebreak, uint64_t* best_mask, uint32_t* best_weight);
BMM_API int bmm_gray_targets_dev(const uint64_t* d_words, size_t rows, size_t stride, size_t cols,
                         const uint32_t* d_targets, const uint32_t* d_others, size_t n_targets,
                         size_t k, int tiebreak, uint64_t* d_best_mask, uint32_t* d_best_weight,
                         void* stream);
/* Allocation-free bmm_gray_targets_dev.  No counterpart in the reference.
 * For callers that may not allocate device memory (a host framework's pool
 * or arena that must account for every byte, plug-ins whose host forbids
 * cudaMalloc/cudaFree, latency-critical loops): all pointers are device
 * memory the caller owns, `stream` is a cudaStream_t, and the call runs
 * asynchronously without cudaMalloc, cudaFree or any allocating routine.
 * Its only scratch is a fixed per-device array of BMM_NOALLOC_MAX_TARGETS
 * 64-bit keys (128 KiB) that exists on every device that loads this library
 * until the process exits; n_targets above that limit is BMM_EINVAL.
 * The first call on each device looks up that array's device address, so
 * make the first call on a device before any stream capture.  All calls
 * share the array: calls whose executions overlap on the GPU (different
 * streams, or different host threads) race; serialise them.  The looked-up
 * address is cached for the life of the process: a cudaDeviceReset between
 * calls is not supported.  chunk_bits set by bmm_gray_tune applies here as it
 * does to bmm_gray_targets_dev. */
#define BMM_NOALLOC_MAX_TARGETS 16384
BMM_API int bmm_gray_targets_noalloc(const uint64_t* d_words, size_t rows, size_t stride,
                                     size_t cols, const uint32_t* d_targets,
                                     const uint32_t* d_others, size_t n_targets, size_t k,
                                     int tiebreak, uint64_t* d_best_mask,
                                     uint32_t* d_best_weight, void* stream);
BMM_API int bmm_fwht_targets(const uint64_t* words, size_t rows, size_t stride, size_t cols,
                     const uint32_t* targets, const uint32_t* others, size_t n_targets, size_t k,
                     uint64_t* best_mask, uint32_t* best_weight);
BMM_API int bmm_fwht_targets_dev(const uint64_t* d_words, size_t rows, size_t stride, size_t cols,
                         const uint32_t* d_targets, const uint32_t* d_others, size_t n_targets,
                         size_t k, uint64_t* d_best_mask, uint32_t* d_best_weight, void* stream);

/* ---- Genetic algorithm (island model) ------------------------------------
 * Replaces bmmpy::ga::GeneticAlgorithm (include/bmmpy/ga/genetic_algorithm.hpp:17-88)
 * and bmmpy::ga::IslandModel (include/bmmpy/ga/island_model.hpp:16-53) for
 * windows of at most 256 rows, populations of at most 1024.  An individual
 * is n candidate masks of ceil(n/64) words each (Candidate::mask) plus a
 * weight per candidate; its fitness is the sum of the weights.  Every island
 * draws from its own xorshift64 stream exactly as GeneticAlgorithm does, so
 * a single island reproduces GeneticAlgorithm::step() trajectories for the
 * same seed.  Islands exchange their best individual along a ring: island i
 * imports island i-1's best whenever island i-1's migration interval divides
 * its generation count; import_migrants rules apply (lifecycle.cpp:83-110). */
#define BMM_GA_STOP_MAX_GENERATIONS 1u /* StopCriteria::max_generations is set */
#define BMM_GA_STOP_MAX_STALE 2u       /* StopCriteria::max_stale_generations is set */
#define BMM_GA_STOP_TARGET 4u          /* StopCriteria::target_total_weight is set */
typedef struct bmm_ga_config { /* GeneticAlgorithmConfig (genetic_algorithm.hpp:17-29) */
    uint32_t population_size;  /* these eight must agree across islands */
    uint32_t elite_count;
    uint32_t num_parents;      /* 1..4 */
    uint32_t num_offspring;    /* >= 1 */
    uint32_t tournament_size;
    uint32_t enable_catastrophe;
    uint32_t catastrophe_threshold;
    uint32_t flags;            /* BMM_GA_STOP_* (per island) */
    double catastrophe_survival_rate;
    double mutation_rate;      /* per island */
    uint64_t max_generations;  /* per island */
    uint64_t max_stale_generations;
    uint64_t target_total_weight;
    uint64_t seed;             /* per island */
} bmm_ga_config;
typedef struct bmm_ga_migration { /* MigrationPolicy (ga/types.hpp:28-33) subset */
    uint32_t interval_generations; /* 0: never export */
    uint32_t import_count;         /* 0: never import */
} bmm_ga_migration;
typedef struct bmm_ga_island_stats { /* RunStats (ga/types.hpp:20-25) + IslandSnapshot */
    uint64_t generations;
    uint64_t evaluations;
    uint64_t stale_generations;
    uint64_t seed;
    uint64_t best_score;
    uint32_t done;
    uint32_t no_improvement;
    double mutation_rate;
} bmm_ga_island_stats;
typedef struct bmm_ga bmm_ga;
/* initialize(window) of `islands` islands, cfgs[i] configuring island i;
 * migration: one policy per island, or NULL (islands never exchange).
 * win: n row indices into words. */
BMM_API int bmm_ga_create(const uint64_t* words, size_t stride, size_t cols, const size_t* win,
                          size_t n, const bmm_ga_config* cfgs, size_t islands,
                          const bmm_ga_migration* migration, bmm_ga** out);
/* Up to `generations` step()s of every island not done; the host checks the
 * stop flags every check_every generations (0 = 1).  *ran: generations run. */
BMM_API int bmm_ga_run(bmm_ga* g, uint64_t generations, uint32_t check_every, uint64_t* ran,
                       int* all_done);
BMM_API int bmm_ga_stats(bmm_ga* g, size_t island, bmm_ga_island_stats* out);
/* best_individual(): island (SIZE_MAX: the model's best, first strict
 * minimum over islands); masks n*ceil(n/64) words, weights n. */
BMM_API int bmm_ga_best(bmm_ga* g, size_t island, uint64_t* masks, uint32_t* weights,
                        uint64_t* score);
/* The island's current population in order: masks P*n*ceil(n/64) words,
 * weights P*n, fitness P (each may be NULL). */
BMM_API int bmm_ga_population(bmm_ga* g, size_t island, uint64_t* masks, uint32_t* weights,
                              uint64_t* fitness);
BMM_API int bmm_ga_destroy(bmm_ga* g);
/* Learned proposal step (no reference counterpart), run after each
 * generation's population is built: for queries_per_elite target rows of
 * every elite individual (the islands' best, carried into the next
 * population), a window of 16 other rows is searched exhaustively (all 2^16
 * XOR subsets, packed FWHT) and an improving subset is applied, re-scored
 * exactly.  mode 1 draws the windows from the proposal network's scores
 * (Gumbel-top-16) with probability learned_fraction -- adapted each
 * generation towards whichever of learned and uniform windows improves more
 * often -- and uniformly otherwise, and trains the network (train_steps Adam
 * steps per generation) on the improving subsets; mode 2 uses uniform windows
 * only; mode 0 (default) is the reference GA.  Needs 17..256 window rows and
 * at most 32767 columns.  Set once, before running. */
typedef struct bmm_ga_proposal {
    uint32_t mode;
    uint32_t queries_per_elite; /* 1..64 */
    uint32_t train_steps;
    uint32_t reserved;
    float learning_rate;
    float learned_fraction;
    uint64_t seed;
} bmm_ga_proposal;
typedef struct bmm_ga_proposal_stats {
    uint64_t tried_learned;
    uint64_t improved_learned;
    uint64_t tried_uniform;
    uint64_t improved_uniform;
    uint64_t examples;      /* training examples used */
    float last_loss;        /* cross-entropy of the last training step */
    float learned_fraction; /* current share of learned windows */
    /* Improvement rates of learned and uniform windows averaged over the
     * generations that drew both (each generation weighs the same): a fair
     * comparison, whereas the totals above mix early generations, where
     * every window improves often, with late ones in different shares. */
    uint64_t paired_generations;
    double paired_rate_learned;
    double paired_rate_uniform;
} bmm_ga_proposal_stats;
BMM_API int bmm_ga_set_proposal(bmm_ga* g, const bmm_ga_proposal* p);
BMM_API int bmm_ga_get_proposal_stats(bmm_ga* g, bmm_ga_proposal_stats* out);
/* Operators on one individual, through the same device code as the
 * generation kernels.  eval: internal::eval_cand_weight
 * (genetic_algorithm_internal.hpp:41-103) of `count` masks.  mutate:
 * GeneticAlgorithm::mutate (operators.cpp:100-129) with the generator state
 * in/out (0 = the default seed).  local_improve: local_improvement
 * (operators.cpp:131-192).  crossover: crossover (operators.cpp:58-98) of
 * `parents` individuals laid out one after another. */
BMM_API int bmm_ga_eval(const uint64_t* words, size_t stride, size_t cols, const size_t* win,
                        size_t n, const uint64_t* masks, size_t count, uint32_t* weights);
BMM_API int bmm_ga_mutate(const uint64_t* words, size_t stride, size_t cols, const size_t* win,
                          size_t n, uint64_t* masks, uint32_t* weights, double mutation_rate,
                          uint64_t* rng_state);
BMM_API int bmm_ga_local_improve(const uint64_t* words, size_t stride, size_t cols,
                                 const size_t* win, size_t n, uint64_t* masks, uint32_t* weights);
BMM_API int bmm_ga_crossover(size_t n, size_t parents, const uint64_t* parent_masks,
                             const uint32_t* parent_weights, uint64_t* child_masks,
                             uint32_t* child_weights);

/* ---- Proposal network (no reference counterpart) ---------------------------
 * A 512 -> 256 -> 256 -> 256 ReLU MLP whose GEMMs run on the tcgen05 tensor
 * cores (BF16 operands, FP32 accumulation in TMEM); softmax cross-entropy
 * against target distributions; Adam (lr given, betas 0.9 / 0.999, eps 1e-8)
 * on FP32 master parameters.  Parameters are laid out W1[256][512], b1[256],
 * W2[256][256], b2, W3[256][256], b3 (bmm_mlp_param_count() floats).  The
 * host-buffer entry points below are synchronous. */
typedef struct bmm_mlp bmm_mlp;
BMM_API int bmm_mlp_create(uint64_t seed, float learning_rate, bmm_mlp** out);
BMM_API int bmm_mlp_destroy(bmm_mlp* h);
BMM_API size_t bmm_mlp_param_count(void);
BMM_API int bmm_mlp_get_params(bmm_mlp* h, float* params);
/* also resets the Adam moments and step count */
BMM_API int bmm_mlp_set_params(bmm_mlp* h, const float* params);
/* x: rows x 512 inputs; logits: rows x 256 */
BMM_API int bmm_mlp_forward(bmm_mlp* h, const float* x, size_t rows, float* logits);
/* gradient of the mean cross-entropy against target rows (rows x 256) */
BMM_API int bmm_mlp_grads(bmm_mlp* h, const float* x, const float* target, size_t rows,
                          float* grads, float* loss);
/* `steps` Adam steps on one batch; *loss: the last step's loss */
BMM_API int bmm_mlp_train(bmm_mlp* h, const float* x, const float* target, size_t rows,
                          int steps, float* loss);
/* C[M][N] = bf16(A[M][K]) . bf16(B[N][K])^T in FP32 on the tensor cores */
BMM_API int bmm_mlp_gemm(const float* A, const float* B, int M, int N, int K, float* C);
/* A network whose work runs on the caller's (created, non-null) stream; the
 * stream is not destroyed with the network. */
BMM_API int bmm_mlp_create_on_stream(uint64_t seed, float learning_rate, void* stream,
                                     bmm_mlp** out);
/* Device-pointer forms of forward / train: x [rows][512], target and logits
 * [rows][256] in device memory; enqueued on the network's stream without
 * synchronisation (errors of the kernels surface at the next host call). */
BMM_API int bmm_mlp_forward_dev(bmm_mlp* h, const float* x, size_t rows, float* logits);
BMM_API int bmm_mlp_train_dev(bmm_mlp* h, const float* x, const float* target, size_t rows,
                              int steps);
/* forward_dev with BF16 inputs x [rows][512] (the GA's proposal features). */
BMM_API int bmm_mlp_forward_bf16_dev(bmm_mlp* h, const void* x, size_t rows, float* logits);
/* GEMM operand staging: 1 (default) = TMA (cp.async.bulk.tensor, 4-stage
 * ring) for BF16 operands with K-contiguous rows, 0 = thread staging for
 * every GEMM.  Results are the same; only speed differs. */
BMM_API int bmm_mlp_tune(int use_tma);

/* ---- exact minimum-weight basis of a window ------------------------------
 * ExactBasisSolverConfig / ExactBasisResult of
 * include/bmmpy/solver/exact_basis_solver.hpp:12-29 (the two matrices are
 * left to the caller: transform row k = basis_masks[k] over the t window rows,
 * basis row k = that combination of the rows). */
typedef struct bmm_exact_basis_config {
    size_t max_rows;          /* reference default 24 */
    uint64_t max_states;      /* reference default 2^24 - 1 */
    size_t max_storage_bytes; /* reference default 128 MiB */
} bmm_exact_basis_config;

typedef struct bmm_exact_basis_result {
    size_t input_rows;
    size_t cols;
    size_t rank;
    uint64_t enumerated_states;
    uint64_t total_weight;
} bmm_exact_basis_result;

/* ExactBasisSolver::solve (src/solver/exact_basis_solver.cpp:58-157): among
 * all bases of the window's row space, the one the reference's greedy picks
 * over the 2^t - 1 combinations ordered by (weight, Gray enumeration index).
 * basis_masks / basis_weights receive `rank` entries (room for min(t, cols)),
 * in acceptance order.  Errors: the reference's messages, BMM_EINVAL for its
 * std::invalid_argument checks, BMM_ERUNTIME for its std::runtime_error. */
BMM_API int bmm_exact_basis(const uint64_t* words, size_t stride, size_t cols,
                            const uint32_t* win, size_t t, const bmm_exact_basis_config* cfg,
                            bmm_exact_basis_result* res, uint32_t* basis_masks,
                            uint32_t* basis_weights);

/* Weight histogram of the 2^t - 1 nonzero combinations of a window (t <= 32):
 * counts[w] for w in [0, cols] (the counting pass of
 * src/solver/exact_basis_solver.cpp:107-118). */
BMM_API int bmm_basis_weight_counts(const uint64_t* words, size_t stride, size_t cols,
                                    const uint32_t* win, size_t t, uint64_t* counts);

/* Device form: `rows` holds the t window rows (1 <= t <= 32) row-major,
 * (cols + 63) / 64 words each with the bits at and past `cols` clear; counts
 * (cols + 1 entries) is overwritten on `stream`.  Asynchronous. */
BMM_API int bmm_basis_weight_counts_dev(const uint64_t* rows, size_t t, size_t cols,
                                        uint64_t* counts, void* stream);

/* ---- simulated-annealing window selection ---------------------------------
 * SASelectorConfig / SASelectionResult of include/bmmpy/search/sa_selector.hpp:14-45.
 * score_policy: 0 PairwiseSynergy, 1 HigherOrderSynergy; cooling_policy:
 * 0 AdaptiveGeometric. */
typedef struct bmm_sa_config {
    uint64_t iterations;                 /* reference default 10000 */
    uint64_t restarts;                   /* 8 */
    uint64_t seed;                       /* 0 -> 0x9E3779B97F4A7C15 */
    uint32_t score_policy;
    uint32_t cooling_policy;
    uint64_t temperature_probe_samples;  /* 64 */
    double initial_acceptance_probability; /* 0.8 */
    double cooling_rate;                 /* 0.99 */
    double min_temperature;              /* 1e-6 */
} bmm_sa_config;

typedef struct bmm_sa_result {
    int64_t score;
    uint64_t accepted_moves;
    uint64_t iterations_run;
    uint64_t best_iteration;
    uint64_t restart_index;
    uint64_t seed;
    size_t n_rows;  /* rows written to out_rows (window_size, or 0) */
} bmm_sa_result;

/* SASelector::select (src/search/sa_selector.cpp:10-75) over a whole matrix of
 * `rows` rows: the best window of window_size rows found by the reference's
 * annealing chain (same generator stream, same result).  out_rows receives the
 * sorted row indices.  The pairwise synergy table is built on the device; the
 * chain runs on the calling thread.  Errors: the reference's messages. */
BMM_API int bmm_sa_select(const uint64_t* words, size_t stride, size_t rows, size_t cols,
                          size_t window_size, const bmm_sa_config* cfg, bmm_sa_result* res,
                          size_t* out_rows);

/* The pairwise synergy table of build_pairwise_synergy_table
 * (src/search/sa_selector_pairwise.cpp:21-52): table[i * rows + j] =
 * 2 * popc(row_i & row_j) for i != j, 0 on the diagonal.  Host form (rows^2
 * uint32 out) and device form (asynchronous on `stream`). */
BMM_API int bmm_sa_pairwise_table(const uint64_t* words, size_t stride, size_t rows, size_t cols,
                                  uint32_t* table);
BMM_API int bmm_sa_pairwise_table_dev(const uint64_t* words, size_t stride, size_t rows,
                                      size_t cols, uint32_t* table, void* stream);

/* ---- matrix IO (src/core/bit_matrix_io.cpp, bit_matrix_hash.cpp) ----------
 * Text: "rows cols\n", then rows x cols '0'/'1' characters; on input any ASCII
 * whitespace may separate them (BitMatrix::load_text / save_text).  Binary:
 * "BMMPYB1\0", u64 rows, u64 cols (little endian), then (cols + 63) / 64
 * words per row, unpadded (load_binary / save_binary).  Errors carry the
 * reference's messages: BMM_ERUNTIME for its std::runtime_error, BMM_EMATRIX
 * for MatrixError (SizeTooLarge). */

/* The dimensions of a text matrix (in >> rows >> cols). */
BMM_API int bmm_matrix_text_header(const char* text, size_t len, uint64_t* rows, uint64_t* cols);
/* Parse a whole text matrix (header included) into rows x stride words; the
 * payload is parsed on the device. */
BMM_API int bmm_matrix_from_text(const char* text, size_t len, uint64_t* words, size_t stride,
                                 size_t rows, size_t cols);
/* Device form: `payload` is the text after the two header numbers (rows and
 * cols from bmm_matrix_text_header), already on the device; words (rows x
 * stride, device) are overwritten on `stream`, which is synchronised to
 * report the parse result. */
BMM_API int bmm_matrix_from_text_dev(const char* payload, size_t len, uint64_t* words,
                                     size_t stride, size_t rows, size_t cols, void* stream);
/* Bytes of save_text's output for a rows x cols matrix. */
BMM_API int bmm_matrix_text_size(size_t rows, size_t cols, size_t* len);
/* save_text into out (cap bytes, not NUL-terminated); formatted on the device. */
BMM_API int bmm_matrix_to_text(const uint64_t* words, size_t stride, size_t rows, size_t cols,
                               char* out, size_t cap, size_t* len);
BMM_API int bmm_matrix_save_binary(const char* path, const uint64_t* words, size_t stride,
                                   size_t rows, size_t cols);
BMM_API int bmm_matrix_binary_header(const char* path, uint64_t* rows, uint64_t* cols);
/* Load into host words (rows x stride, padding words cleared) ... */
BMM_API int bmm_matrix_load_binary(const char* path, uint64_t* words, size_t stride, size_t rows,
                                   size_t cols);
/* ... or straight into device words through pinned staging (synchronous). */
BMM_API int bmm_matrix_load_binary_dev(const char* path, uint64_t* words, size_t stride,
                                       size_t rows, size_t cols, void* stream);
/* BitMatrix::hash: SHA-256 hex (64 characters + NUL) of rows, cols and the
 * tail-masked row words as little-endian u64 values. */
BMM_API int bmm_matrix_hash(const uint64_t* words, size_t stride, size_t rows, size_t cols,
                            char* hex);

/* ---- device-resident search -> apply ---------------------------------------
 * search_apply (bmmpy/workflows.py:45-90) over n_windows windows of t rows of
 * a DEVICE matrix, in order, all on `stream`: per window the exact top-k
 * spectrum search (MitmFwhtSearch / FwhtSearch candidates) and the applier
 * (0: GreedyApplier(min_gain, stochastic, seed) -- one generator carried from
 * window to window as one applier object would; 1: GlobalGreedyApplier(
 * require_improvement)) update the matrix rows in place.  windows: host array
 * of n_windows x t row indices, each < rows (checked on the host before any
 * launch: BMM_EINVAL, where the reference raises IndexError).  results: one
 * ApplyResult per window; when a window fails (BMM_ERUNTIME) the later
 * windows of the call are left untouched, as the reference loop stops there.
 * cfg->seed is the greedy generator's state on entry (0 -> 0xDEADB, as the
 * constructor); final_state (optional) receives it on exit.  Synchronises
 * `stream` once, at the end. */
typedef struct bmm_sweep_config {
    uint64_t max_candidates;
    uint32_t applier;
    uint32_t stochastic;
    uint64_t min_gain;
    uint64_t seed;
    uint32_t require_improvement;
    uint32_t reserved;
} bmm_sweep_config;

typedef struct bmm_apply_result {
    uint64_t applied_count;
    uint64_t weight_improvement;
} bmm_apply_result;

BMM_API int bmm_search_apply_dev(uint64_t* words, size_t rows, size_t stride, size_t cols,
                                 const uint32_t* windows, size_t t, size_t n_windows,
                                 const bmm_sweep_config* cfg, bmm_apply_result* results,
                                 uint64_t* final_state, void* stream);

/* ---- spectrum slices: one window's masks split across devices ----------
 * No reference counterpart (the reference searches a window on one device).
 * The t-bit masks of a window split into low_bits low bits, materialised as
 * one 2^low_bits spectrum per slice, and t - low_bits high bits, the slice
 * index x.  bmm_spectrum_topk_slices_dev writes to d_out (device, k entries,
 * empty ones with weight 0xffffffff) the k smallest (weight, mask) over the
 * nonzero masks whose slice lies in [slice_begin, slice_end), of the t rows
 * d_rows (device, t x W words, W >= ceil(cols / 64), bits past cols zero);
 * asynchronous on `stream`.  Ranks that take disjoint slice ranges covering
 * [0, 2^(t - low_bits)) and merge their lists by (weight, mask) get exactly
 * the window's MitmFwhtSearch / FwhtSearch result.  low_bits = -1 uses
 * bmm_spectrum_low_bits(t); otherwise 14 <= low_bits <= min(t, 33).
 * bmm_spectrum_tune sets the default split (-1: min(t, 33)); results never
 * change, only speed and memory (2^low_bits int32 per call). */
BMM_API int bmm_spectrum_tune(int low_bits);
/* The spectrum's last transform pass (fused with the top-k scan): 1 = one
 * double-buffered CTA per SM (default), 0 = two single-buffered CTAs per SM.
 * Results never change, only speed. */
BMM_API int bmm_spectrum_tune_last_pass(int double_buffered);
/* Transform passes of 6..9 bits with k <= 128: register-resident (HBM
 * straight into registers, one shared-memory exchange per tile) with
 * 2 = two CTAs per SM (default) or 1 = one CTA per SM that prefetches the
 * next tile into registers; 0 = the cp.async tile passes (then
 * bmm_spectrum_tune_last_pass applies).  Results never change. */
BMM_API int bmm_spectrum_tune_passes(int register_resident);
BMM_API int bmm_spectrum_low_bits(size_t t);
BMM_API int bmm_spectrum_topk_slices_dev(const uint64_t* d_rows, size_t t, size_t W, size_t cols,
                                         size_t k, int low_bits, int64_t slice_begin,
                                         int64_t slice_end, bmm_candidate* d_out, void* stream);

/* ---- split-window preparation on the device ----------------------------
 * build_compact_split_window (include/bmmpy/search/split_window_prep.hpp:21-26,
 * src/search/split_window_prep.cpp:42-137) over the t rows d_rows (device,
 * t x W words, W >= ceil(cols / 64); bits past cols are ignored): the
 * distinct nonzero t-bit column patterns (bit i = row i) in ascending order,
 * written as d_q[i] = pattern >> low_bits, d_r[i] = pattern & (2^low_bits - 1)
 * and d_mult[i] = its column count, for i < *n_unique; *total_weight = the
 * number of active columns.  cap = the room in d_q / d_r / d_mult (cols
 * always suffices); more distinct patterns than cap is BMM_EINVAL.  The
 * reference's checks and messages: low_bits > t, t > 64.  Synchronises
 * `stream` (the counts are returned on the host). */
BMM_API int bmm_split_window_dev(const uint64_t* d_rows, size_t t, size_t W, size_t cols,
                                 size_t low_bits, uint64_t* d_q, uint64_t* d_r, int32_t* d_mult,
                                 size_t cap, size_t* n_unique, int32_t* total_weight,
                                 void* stream);

/* Autotuner hook for the enumeration kernel (no reference counterpart):
 * carry-save blocks of 8 words per 64-word lane (0, 2, 5 or 8; -1 = built-in
 * policy).  Process-wide; results never change, only speed. */
BMM_API int bmm_basis_tune(int hs_blocks);

#ifdef __cplusplus
}
#endif

#endif
