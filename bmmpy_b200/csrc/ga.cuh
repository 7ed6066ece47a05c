// Device state of the island-model genetic algorithm (ga.cu).
#pragma once

#include "common.cuh"

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

}  // namespace ga
}  // namespace bmm
