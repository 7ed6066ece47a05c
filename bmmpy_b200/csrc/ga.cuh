// Device state of the island-model genetic algorithm (ga.cu).
#pragma once

#include "common.cuh"

#include <cuda_bf16.h>
#include <vector>

struct bmm_mlp;

namespace bmm {
namespace ga {

constexpr int kMaxN = 256;  // candidates per individual (masks of 4 words)
constexpr int kMW = 4;      // mask words held per candidate on the device

// Per-island bookkeeping: GeneticAlgorithm's _best_score, _no_improvement,
// _catastrophe, _stats and _rng (genetic_algorithm.hpp:67-87).
struct IslandStat {
    unsigned long long best;         // _best_score
    unsigned long long generations;  // RunStats::generations
    unsigned long long evaluations;  // RunStats::evaluations
    unsigned long long stale;        // RunStats::stale_generations
    unsigned long long rng;          // XorShift64 state after the last draw
    double rate;                     // GeneticAlgorithmConfig::mutation_rate (adapted)
    uint32_t no_improvement;
    uint32_t catastrophe;
    uint32_t cur;       // population buffer (0/1) holding the current population
    uint32_t done;      // should_stop() was true
    uint32_t stepped;   // the island runs the generation being built
    uint32_t count;     // mutation draws per child this generation
    uint32_t cat_now;   // a catastrophe rebuilt the population this generation
    uint32_t migrated;  // a migrant was imported this generation
};

// One population: I*P individuals of N candidates.
struct Pop {
    uint64_t* masks;          // [I*P][N][4]
    uint64_t* rows;           // [I*P][N][W]  materialised candidate rows
    uint32_t* wts;            // [I*P][N]
    unsigned long long* fit;  // [I*P]
};

// How slot s of an island's next population is built.
enum SlotKind : uint32_t {
    kCopy = 0,       // copy current individual par[0] (elites, catastrophe survivors)
    kChild = 1,      // crossover of par[0..np) then mutation
    kRandom = 2,     // make_random
    kIdentity = 3,   // make_identity
    kHeuristic = 4,  // make_heuristic
};

struct Sched {
    unsigned long long rng;  // generator state at the slot's first draw
    uint32_t kind;
    uint32_t np;
    uint16_t par[4];
};

// Settings every island shares (they fix the device layout and schedule).
struct Config {
    int N, W, P, E, T, parents, offspring;
    int cat_enable, cat_threshold, cat_survivors;
};

// Per-island settings: StopCriteria (ga/types.hpp:13-18) and MigrationPolicy.
struct IslandCfg {
    unsigned long long max_gen, max_stale, target;
    uint32_t flags;         // 1 max_gen, 2 max_stale, 4 target are set
    uint32_t interval;      // export the best every `interval` generations (0: never)
    uint32_t import_count;  // 0: never import
    uint32_t pad;
};

struct State {
    Config c;
    int I;
    const IslandCfg* icfg;      // [I]
    const uint64_t* base;       // [N][W] window rows
    Pop pop[2];
    uint32_t* order;            // [I*P] ranked positions of the current population
    IslandStat* stat;           // [I]
    Sched* sched;               // [I*P]
    const uint64_t* jump_mut;   // [N + 1][64]: xorshift^(2c) as 64 GF(2) columns, c <= N
    const uint64_t* jump_rand;  // [64]: xorshift^(6N) (one make_random)
    uint64_t* best_masks;       // [I][N][4]
    uint64_t* best_rows;        // [I][N][W]
    uint32_t* best_wts;         // [I][N]
    uint32_t* Gs;               // per-CTA N x N overlap scratch for local improvement
};

// Learned proposal step (ga_propose.cu): per elite individual, qpc target
// rows; for each, a window of 16 other rows -- chosen by the proposal network
// or uniformly -- is searched exhaustively (packed FWHT over all 2^16
// subsets) and an improving subset is XORed into the target row.
struct PropBuf {
    int mode;         // 1 learned windows (with uniform exploration), 2 uniform windows,
                      // 3 the 16 rows of smallest pairwise weight change
    int qpc;          // queries per elite individual
    uint64_t seed;
    float learned_frac;
    const uint32_t* cols;  // [256] sampled columns of the row sketch
    uint16_t* target;      // [Q] target row of each query
    uint16_t* perm;        // [Q][256] row at each rank position
    __nv_bfloat16* X;      // [Q][512] network inputs
    float* logits;         // [Q][256]
    float* T;              // [Q][256] training targets of improving queries
    uint8_t* valid;        // [Q] the query found an improving subset
    unsigned long long* counters;  // tried / improved, learned then uniform
    __nv_bfloat16* Xb;     // replay buffer of improving examples [cap][512]
    float* Tb;             // [cap][256]
    int* batch_rows;       // new examples this generation, then their query indices
};

constexpr int kPropBatchCap = 4096;  // replay buffer of improving examples
constexpr int kPropMinibatch = 512;

}  // namespace ga
}  // namespace bmm

// The GA handle (bmm_ga_* in include/bmm_b200.h).
struct bmm_ga {
    int device = -1;
    cudaStream_t stream = nullptr;
    bmm::ga::State st{};
    int I = 0;
    std::vector<uint32_t> intervals;  // per island export interval
    unsigned long long gen = 0;       // generations run by the islands still active
    int build_grid = 0, local_grid = 0;
    size_t build_smem = 0;
    int rank_threads = 0;
    std::vector<void*> allocs;
    bmm::ga::IslandStat* h_stat = nullptr;  // pinned
    std::vector<uint64_t> seeds;
    uint32_t cols = 0;
    int search_grid = 0;
    // proposal step
    bmm::ga::PropBuf prop{};
    unsigned long long tot[4] = {0, 0, 0, 0};  // tried / improved: learned, uniform
    bmm_mlp* net = nullptr;
    int train_steps = 0;
    unsigned long long* h_counters = nullptr;  // pinned, 4
    unsigned long long examples = 0;
    float last_loss = 0.f;
    double ema_tried[2] = {0, 0}, ema_improved[2] = {0, 0};  // learned, uniform (decayed)
    double paired_rate[2] = {0, 0};  // per-generation rates summed over paired generations
    unsigned long long paired_gens = 0;
    int replay_head = 0, replay_fill = 0;
};

namespace bmm {
namespace ga {
// Runs the proposal step on the next population of the generation being
// built (after build_kernel, before local improvement); synchronises.
int propose_generation(bmm_ga* g);
int propose_setup(bmm_ga* g, int mode, int qpc, int train_steps, float lr, float learned_frac,
                  uint64_t seed);
void propose_free(bmm_ga* g);
}  // namespace ga
}  // namespace bmm
