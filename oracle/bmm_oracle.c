/* CPU oracle: plain-C restatement of the reference hot path.  TEST
 * INFRASTRUCTURE ONLY -- see bmm_oracle.h for the contract and the pinning.
 * Each function names the reference file:line range it restates. */
#include "bmm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define WORD_BITS 64u

static unsigned popc64(uint64_t x) { return (unsigned)__builtin_popcountll(x); }
static unsigned ctz64(uint64_t x) { return (unsigned)__builtin_ctzll(x); }

static uint64_t tail_mask_for_cols(size_t cols) {
    /* src/search/fwht_search.cpp:24-30 */
    const size_t tail = cols % WORD_BITS;
    return tail == 0 ? ~(uint64_t)0 : (((uint64_t)1 << tail) - 1);
}

/* ---- xorshift64 (include/bmmpy/core/detail/xorshift64.hpp:10-40) ---- */
uint64_t orc_xs_seed(uint64_t seed) { return seed == 0 ? 0x9E3779B97F4A7C15ull : seed; }

uint64_t orc_xs_next(uint64_t* state) {
    uint64_t x = *state;
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    *state = x;
    return x;
}

static size_t xs_index(uint64_t* state, size_t n) {
    return n == 0 ? 0 : (size_t)(orc_xs_next(state) % n);
}

static double xs_unit(uint64_t* state) {
    return (double)(orc_xs_next(state) >> 11) * (1.0 / 9007199254740992.0);
}

uint64_t orc_gen_instance(uint64_t* words, size_t rows, size_t cols, size_t stride, double p,
                          uint64_t seed, size_t scrambles) {
    uint64_t st = orc_xs_seed(seed);
    uint64_t planted = 0;
    memset(words, 0, rows * stride * sizeof(uint64_t));
    for (size_t r = 0; r < rows; ++r)
        for (size_t c = 0; c < cols; ++c)
            if (xs_unit(&st) < p) {
                words[r * stride + c / 64] |= (uint64_t)1 << (c % 64);
                ++planted;
            }
    if (rows < 2)
        return planted;
    for (size_t s = 0; s < scrambles; ++s) {
        const size_t i = xs_index(&st, rows);
        size_t j = xs_index(&st, rows);
        while (j == i)
            j = xs_index(&st, rows);
        for (size_t w = 0; w < stride; ++w)
            words[i * stride + w] ^= words[j * stride + w];
    }
    return planted;
}

/* ---- FWHT (src/math/fwht.cpp:28-57, src/math/fwht_scalar.cpp:19-39) ---- */
static int is_pow2(size_t n) { return n != 0 && (n & (n - 1)) == 0; }

int orc_fwht_i32(int32_t* d, size_t n) {
    if (n <= 1)
        return 0;
    if (!is_pow2(n))
        return ORC_EINVAL;
    for (size_t len = 1; len < n; len <<= 1)
        for (size_t base = 0; base < n; base += 2 * len)
            for (size_t i = 0; i < len; ++i) {
                const uint32_t u = (uint32_t)d[base + i], v = (uint32_t)d[base + len + i];
                d[base + i] = (int32_t)(u + v); /* two's-complement wrap */
                d[base + len + i] = (int32_t)(u - v);
            }
    return 0;
}

int orc_fwht_i16(int16_t* d, size_t n) {
    if (n <= 1)
        return 0;
    if (!is_pow2(n))
        return ORC_EINVAL;
    for (size_t len = 1; len < n; len <<= 1)
        for (size_t base = 0; base < n; base += 2 * len)
            for (size_t i = 0; i < len; ++i) {
                const uint16_t u = (uint16_t)d[base + i], v = (uint16_t)d[base + len + i];
                d[base + i] = (int16_t)(uint16_t)(u + v);
                d[base + len + i] = (int16_t)(uint16_t)(u - v);
            }
    return 0;
}

/* ---- exact top-k by (weight asc, mask asc) ----
 * Same order as candidate_less (src/search/fwht_search.cpp:15-22) and
 * topk_less / insert_topk (src/search/bruteforce_search.cpp:29-54).  A bounded
 * sorted insertion keeps exactly the k smallest pairs seen; mask 0 is never
 * inserted. */
typedef struct {
    uint64_t* mask;
    uint32_t* weight;
    size_t size, k;
} topk_t;

static int pair_less(uint32_t wa, uint64_t ma, uint32_t wb, uint64_t mb) {
    return wa < wb || (wa == wb && ma < mb);
}

static void topk_init(topk_t* t, size_t k) {
    t->k = k;
    t->size = 0;
    t->mask = (uint64_t*)malloc((k ? k : 1) * sizeof(uint64_t));
    t->weight = (uint32_t*)malloc((k ? k : 1) * sizeof(uint32_t));
}

static void topk_free(topk_t* t) {
    free(t->mask);
    free(t->weight);
}

static void topk_insert(topk_t* t, uint64_t mask, uint32_t w) {
    if (mask == 0 || t->k == 0)
        return;
    if (t->size == t->k && !pair_less(w, mask, t->weight[t->size - 1], t->mask[t->size - 1]))
        return;
    /* lower_bound */
    size_t lo = 0, hi = t->size;
    while (lo < hi) {
        const size_t mid = (lo + hi) / 2;
        if (pair_less(t->weight[mid], t->mask[mid], w, mask))
            lo = mid + 1;
        else
            hi = mid;
    }
    size_t last = t->size < t->k ? t->size : t->k - 1;
    for (size_t i = last; i > lo; --i) {
        t->mask[i] = t->mask[i - 1];
        t->weight[i] = t->weight[i - 1];
    }
    t->mask[lo] = mask;
    t->weight[lo] = w;
    if (t->size < t->k)
        ++t->size;
}

static long topk_emit(topk_t* t, uint64_t* out_mask, uint32_t* out_w, size_t cap) {
    const size_t n = t->size < cap ? t->size : cap;
    for (size_t i = 0; i < n; ++i) {
        out_mask[i] = t->mask[i];
        out_w[i] = t->weight[i];
    }
    const long count = (long)t->size;
    topk_free(t);
    return count;
}

/* Column pattern of window rows at word w, bit b. */
static uint64_t col_pattern(const uint64_t* words, size_t stride, const size_t* win, size_t t,
                            size_t w, unsigned b) {
    uint64_t p = 0;
    for (size_t r = 0; r < t; ++r)
        if ((words[win[r] * stride + w] >> b) & 1u)
            p |= (uint64_t)1 << r;
    return p;
}

/* ---- FwhtSearch::search (src/search/fwht_search.cpp:34-132) ---- */
long orc_fwht_search(const uint64_t* words, size_t stride, size_t cols, const size_t* win,
                     size_t t, size_t max_rows, size_t k, uint64_t* out_mask,
                     uint32_t* out_weight, size_t cap) {
    if (t == 0 || t > max_rows || k == 0) /* :36-37 */
        return 0;
    if (t > 64 || t >= 8 * sizeof(size_t)) /* :39-46 */
        return ORC_EINVAL;
    const size_t wpr = (cols + 63) / 64;
    if (wpr == 0) /* :50-51 */
        return 0;
    const size_t n = (size_t)1 << t;
    int32_t* h = (int32_t*)calloc(n, sizeof(int32_t));
    if (!h)
        return ORC_EINVAL;
    uint64_t total = 0;
    const uint64_t tail = tail_mask_for_cols(cols);
    for (size_t w = 0; w < wpr; ++w) { /* :59-91 histogram of active columns */
        uint64_t active = 0;
        for (size_t r = 0; r < t; ++r)
            active |= words[win[r] * stride + w];
        if (w + 1 == wpr)
            active &= tail;
        while (active) {
            const unsigned b = ctz64(active);
            const uint64_t p = col_pattern(words, stride, win, t, w, b);
            if (h[p] == INT32_MAX) {
                free(h);
                return ORC_EOVERFLOW;
            }
            ++h[p];
            if (++total > (uint64_t)INT32_MAX) {
                free(h);
                return ORC_EOVERFLOW;
            }
            active &= active - 1;
        }
    }
    orc_fwht_i32(h, n); /* :93 */
    topk_t best;
    topk_init(&best, k);
    for (size_t mask = 1; mask < n; ++mask) { /* :105-126 */
        const int64_t w2 = (int64_t)total - (int64_t)h[mask];
        if (w2 < 0 || (w2 & 1))
            continue;
        topk_insert(&best, mask, (uint32_t)(w2 / 2));
    }
    free(h);
    return topk_emit(&best, out_mask, out_weight, cap);
}

/* ---- build_compact_split_window (src/search/split_window_prep.cpp:42-137) ---- */
static int cmp_u64(const void* a, const void* b) {
    const uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return x < y ? -1 : (x > y);
}

long orc_split_window(const uint64_t* words, size_t stride, size_t cols, const size_t* win,
                      size_t t, size_t low_bits, uint64_t* q, uint64_t* r, int32_t* mult,
                      size_t cap, int32_t* total_weight) {
    if (low_bits > t || t > 64) /* :442-449 */
        return ORC_EINVAL;
    *total_weight = 0;
    const size_t wpr = (cols + 63) / 64;
    if (t == 0 || wpr == 0)
        return 0;
    uint64_t* pats = (uint64_t*)malloc((cols ? cols : 1) * sizeof(uint64_t));
    size_t np = 0;
    const uint64_t tail = tail_mask_for_cols(cols);
    for (size_t w = 0; w < wpr; ++w) {
        uint64_t active = 0;
        for (size_t i = 0; i < t; ++i)
            active |= words[win[i] * stride + w];
        if (w + 1 == wpr)
            active &= tail;
        while (active) {
            pats[np++] = col_pattern(words, stride, win, t, w, ctz64(active));
            active &= active - 1;
        }
    }
    if (np > (size_t)INT32_MAX) {
        free(pats);
        return ORC_EOVERFLOW;
    }
    *total_weight = (int32_t)np;
    qsort(pats, np, sizeof(uint64_t), cmp_u64); /* sorted by pattern, :509-511 */
    const uint64_t low_mask =
        low_bits == 0 ? 0 : (low_bits >= 64 ? ~(uint64_t)0 : (((uint64_t)1 << low_bits) - 1));
    size_t u = 0;
    for (size_t i = 0; i < np;) {
        size_t j = i;
        while (j < np && pats[j] == pats[i])
            ++j;
        if (u < cap) {
            q[u] = low_bits == 64 ? 0 : (pats[i] >> low_bits);
            r[u] = pats[i] & low_mask;
            mult[u] = (int32_t)(j - i);
        }
        ++u;
        i = j;
    }
    free(pats);
    return (long)u;
}

/* ---- MitmFwhtSearch::search (src/search/mitm_fwht_search.cpp) ---- */
long orc_mitm_search(const uint64_t* words, size_t stride, size_t cols, const size_t* win,
                     size_t t, size_t k, uint64_t* out_mask, uint32_t* out_weight, size_t cap) {
    if (k == 0 || t == 0) /* :270-275 */
        return 0;
    if (t > 64)
        return ORC_EINVAL;
    /* get_split_info :56-60 */
    const size_t high = t <= 26 ? t / 2 : (t / 2 < 13 ? t / 2 : 13);
    const size_t low = t - high;
    if (low > 30 || low >= 31 || high >= 31) /* :283-289 */
        return ORC_EINVAL;
    const size_t wpr = (cols + 63) / 64;
    size_t ucap = cols ? cols : 1;
    uint64_t* q = (uint64_t*)malloc(ucap * sizeof(uint64_t));
    uint64_t* r = (uint64_t*)malloc(ucap * sizeof(uint64_t));
    int32_t* mult = (int32_t*)malloc(ucap * sizeof(int32_t));
    int32_t total = 0;
    long u = wpr ? orc_split_window(words, stride, cols, win, t, low, q, r, mult, ucap, &total) : 0;
    if (u <= 0) {
        free(q);
        free(r);
        free(mult);
        return u < 0 ? u : 0;
    }
    /* build_adjacency :91-143: per low bit, the unique patterns whose r has it */
    size_t* off = (size_t*)calloc(low + 1, sizeof(size_t));
    for (long i = 0; i < u; ++i)
        for (uint64_t m = r[i]; m; m &= m - 1)
            ++off[ctz64(m) + 1];
    for (size_t b = 0; b < low; ++b)
        off[b + 1] += off[b];
    size_t* cur = (size_t*)malloc((low + 1) * sizeof(size_t));
    memcpy(cur, off, (low + 1) * sizeof(size_t));
    int32_t* adj = (int32_t*)malloc((off[low] ? off[low] : 1) * sizeof(int32_t));
    for (long i = 0; i < u; ++i)
        for (uint64_t m = r[i]; m; m &= m - 1)
            adj[cur[ctz64(m)]++] = (int32_t)i;
    /* initialize_buckets :145-162 */
    const size_t n_high = (size_t)1 << high;
    int32_t* buckets = (int32_t*)calloc(n_high, sizeof(int32_t));
    int32_t* tmp = (int32_t*)malloc(n_high * sizeof(int32_t));
    int32_t* sgn = (int32_t*)malloc(u * sizeof(int32_t));
    for (long i = 0; i < u; ++i) {
        buckets[q[i]] += mult[i];
        sgn[i] = mult[i];
    }
    topk_t best;
    topk_init(&best, k);
    const size_t n_loop = (size_t)1 << low;
    uint64_t x_low = 0;
    for (size_t i = 0; i < n_loop; ++i) {
        if (i != 0) { /* apply_bit_flip :164-186 */
            const size_t bit = ctz64(i);
            for (size_t j = off[bit]; j < off[bit + 1]; ++j) {
                const int32_t c = adj[j];
                buckets[q[c]] -= 2 * sgn[c];
                sgn[c] = -sgn[c];
            }
            x_low ^= (uint64_t)1 << bit;
        }
        /* process_candidate :233-265 */
        memcpy(tmp, buckets, n_high * sizeof(int32_t));
        orc_fwht_i32(tmp, n_high);
        for (size_t xh = 0; xh < n_high; ++xh) {
            const int64_t w2 = (int64_t)total - (int64_t)tmp[xh];
            if (w2 < 0 || (w2 & 1))
                continue;
            const uint64_t mask = ((uint64_t)xh << low) | x_low;
            if (mask)
                topk_insert(&best, mask, (uint32_t)(w2 / 2));
        }
    }
    free(q);
    free(r);
    free(mult);
    free(off);
    free(cur);
    free(adj);
    free(buckets);
    free(tmp);
    free(sgn);
    return topk_emit(&best, out_mask, out_weight, cap);
}

/* ---- BruteforceSearch::search (src/search/bruteforce_search.cpp) ---- */
long orc_bruteforce_search(const uint64_t* words, size_t stride, size_t cols, const size_t* win,
                           size_t t, size_t k, size_t chunk_bits, uint64_t* out_mask,
                           uint32_t* out_weight, size_t cap) {
    if (k == 0 || t == 0) /* :301-306 */
        return 0;
    if (t > 64)
        return ORC_EINVAL;
    const size_t wpr = (cols + 63) / 64;
    if (wpr == 0)
        return 0;
    if (cols > (size_t)UINT32_MAX)
        return ORC_EOVERFLOW;
    /* resolve_chunk_bits :113-123 */
    size_t chunk = chunk_bits;
    if (chunk == 0)
        chunk = t < 12 ? t : 12;
    else if (chunk > t || chunk >= 64)
        return ORC_EINVAL;
    const size_t high_bits = t - chunk;
    if (high_bits >= 63)
        return ORC_EINVAL; /* the reference cannot enumerate this either */
    const uint64_t prefixes = (uint64_t)1 << high_bits;
    uint64_t* cur = (uint64_t*)malloc(wpr * sizeof(uint64_t));
    topk_t best;
    topk_init(&best, k);
    for (uint64_t prefix = 0; prefix < prefixes; ++prefix) { /* sweep_prefix :126-170 */
        memset(cur, 0, wpr * sizeof(uint64_t));
        for (size_t hb = 0; hb < high_bits; ++hb)
            if ((prefix >> hb) & 1u)
                for (size_t w = 0; w < wpr; ++w)
                    cur[w] ^= words[win[chunk + hb] * stride + w];
        uint64_t mask = prefix << chunk;
        uint32_t wt = 0;
        for (size_t w = 0; w < wpr; ++w)
            wt += popc64(cur[w]);
        topk_insert(&best, mask, wt);
        const uint64_t states = (uint64_t)1 << chunk;
        for (uint64_t s = 1; s < states; ++s) {
            const unsigned b = ctz64(s);
            const uint64_t* row = words + win[b] * stride;
            wt = 0;
            for (size_t w = 0; w < wpr; ++w) {
                cur[w] ^= row[w];
                wt += popc64(cur[w]);
            }
            mask ^= (uint64_t)1 << b;
            topk_insert(&best, mask, wt);
        }
    }
    free(cur);
    return topk_emit(&best, out_mask, out_weight, cap);
}

/* ---- per-target best ---- */
static uint64_t inverse_gray(uint64_t s) {
    for (unsigned sh = 1; sh < 64; sh <<= 1)
        s ^= s >> sh;
    return s;
}

int orc_target_best_gray(const uint64_t* words, size_t stride, size_t cols, size_t target,
                         const size_t* others, size_t k, int tiebreak, uint64_t* best_mask,
                         uint32_t* best_weight) {
    if (k >= 63)
        return ORC_EINVAL;
    const size_t wpr = (cols + 63) / 64;
    uint64_t* cur = (uint64_t*)malloc((wpr ? wpr : 1) * sizeof(uint64_t));
    memcpy(cur, words + target * stride, wpr * sizeof(uint64_t));
    uint32_t bw = 0;
    for (size_t w = 0; w < wpr; ++w)
        bw += popc64(cur[w]);
    uint64_t bm = 0, bkey = 0, mask = 0;
    const uint64_t states = (uint64_t)1 << k;
    for (uint64_t s = 1; s < states; ++s) {
        const unsigned b = ctz64(s);
        const uint64_t* row = words + others[b] * stride;
        uint32_t wt = 0;
        for (size_t w = 0; w < wpr; ++w) {
            cur[w] ^= row[w];
            wt += popc64(cur[w]);
        }
        mask ^= (uint64_t)1 << b;
        const uint64_t key = tiebreak ? s : mask; /* s == inverse_gray(mask) */
        if (wt < bw || (wt == bw && key < bkey)) {
            bw = wt;
            bm = mask;
            bkey = key;
        }
    }
    (void)inverse_gray;
    free(cur);
    *best_mask = bm;
    *best_weight = bw;
    return 0;
}

int orc_target_best_fwht(const uint64_t* words, size_t stride, size_t cols, size_t target,
                         const size_t* others, size_t k, uint64_t* best_mask,
                         uint32_t* best_weight) {
    if (k >= 31)
        return ORC_EINVAL;
    const size_t n = (size_t)1 << k;
    int32_t* h = (int32_t*)calloc(n, sizeof(int32_t));
    for (size_t c = 0; c < cols; ++c) {
        uint64_t p = 0;
        for (size_t j = 0; j < k; ++j)
            if ((words[others[j] * stride + c / 64] >> (c % 64)) & 1u)
                p |= (uint64_t)1 << j;
        h[p] += ((words[target * stride + c / 64] >> (c % 64)) & 1u) ? -1 : 1;
    }
    orc_fwht_i32(h, n);
    size_t best = 0;
    for (size_t s = 1; s < n; ++s)
        if (h[s] > h[best])
            best = s;
    *best_mask = best;
    *best_weight = (uint32_t)(((int64_t)cols - h[best]) / 2);
    free(h);
    return 0;
}

/* ---- GA (src/ga/genetic_algorithm_internal.hpp:41-103) ---- */
uint32_t orc_eval_cand_weight(const uint64_t* words, size_t stride, size_t cols,
                              const size_t* win, size_t n, const uint64_t* mask, size_t mw) {
    const size_t wpr = (cols + 63) / 64;
    uint32_t total = 0;
    const uint64_t tail = tail_mask_for_cols(cols);
    for (size_t w = 0; w < wpr; ++w) {
        uint64_t acc = 0;
        for (size_t mi = 0; mi < mw; ++mi)
            for (uint64_t m = mask[mi]; m; m &= m - 1) {
                const size_t row = mi * 64 + ctz64(m);
                if (row < n)
                    acc ^= words[win[row] * stride + w];
            }
        if (w + 1 == wpr)
            acc &= tail;
        total += popc64(acc);
    }
    return total;
}

/* GeneticAlgorithm::mutate (src/ga/genetic_algorithm_operators.cpp:100-129) */
void orc_mutate(const uint64_t* words, size_t stride, size_t cols, const size_t* win, size_t n,
                uint64_t* masks, uint32_t* weights, size_t mw, double rate, uint64_t* rng_state) {
    if (n < 2)
        return;
    size_t count = (size_t)((double)n * rate);
    if (count < 1)
        count = 1;
    for (size_t c = 0; c < count; ++c) {
        const size_t i = xs_index(rng_state, n);
        const size_t j = xs_index(rng_state, n);
        if (i == j)
            continue;
        for (size_t w = 0; w < mw; ++w)
            masks[i * mw + w] ^= masks[j * mw + w];
        weights[i] = orc_eval_cand_weight(words, stride, cols, win, n, masks + i * mw, mw);
    }
}

/* GeneticAlgorithm::local_improvement (src/ga/genetic_algorithm_operators.cpp:131-192) */
void orc_local_improvement(const uint64_t* words, size_t stride, size_t cols, const size_t* win,
                           size_t n, uint64_t* masks, uint32_t* weights, size_t mw) {
    if (n < 2 || cols == 0)
        return;
    const size_t wpr = (cols + 63) / 64;
    const uint64_t tail = tail_mask_for_cols(cols);
    uint64_t* mat = (uint64_t*)calloc(n * wpr, sizeof(uint64_t));
    for (size_t i = 0; i < n; ++i) {
        for (size_t w = 0; w < wpr; ++w) {
            uint64_t acc = 0;
            for (size_t mi = 0; mi < mw; ++mi)
                for (uint64_t m = masks[i * mw + mi]; m; m &= m - 1) {
                    const size_t row = mi * 64 + ctz64(m);
                    if (row < n)
                        acc ^= words[win[row] * stride + w];
                }
            if (w + 1 == wpr)
                acc &= tail;
            mat[i * wpr + w] = acc;
        }
        uint32_t wt = 0;
        for (size_t w = 0; w < wpr; ++w)
            wt += popc64(mat[i * wpr + w]);
        weights[i] = wt;
    }
    for (int iter = 0; iter < 10; ++iter) {
        int improved = 0;
        for (size_t i = 0; i < n; ++i) {
            const uint64_t wi = weights[i];
            if (wi == 0)
                continue;
            size_t best_j = n;
            uint64_t best_w = wi;
            for (size_t j = 0; j < n; ++j) {
                if (i == j)
                    continue;
                const uint64_t wj = weights[j];
                if (wj >= 2 * wi)
                    continue;
                uint64_t ov = 0;
                for (size_t w = 0; w < wpr; ++w)
                    ov += popc64(mat[i * wpr + w] & mat[j * wpr + w]);
                const uint64_t cw = wi + wj - 2 * ov;
                if (cw < best_w) {
                    best_w = cw;
                    best_j = j;
                }
            }
            if (best_j == n)
                continue;
            for (size_t w = 0; w < mw; ++w)
                masks[i * mw + w] ^= masks[best_j * mw + w];
            for (size_t w = 0; w < wpr; ++w)
                mat[i * wpr + w] ^= mat[best_j * wpr + w];
            weights[i] = (uint32_t)best_w;
            improved = 1;
        }
        if (!improved)
            break;
    }
    free(mat);
}

/* ---- GA crossover (src/ga/genetic_algorithm_operators.cpp:58-98) and the
 * PivotBasis it fills (include/bmmpy/core/detail/xor_basis.hpp:117-155). ---- */
static int highest_bit_words(const uint64_t* v, size_t mw) {
    for (size_t w = mw; w-- > 0;)
        if (v[w])
            return (int)(w * 64 + 63 - __builtin_clzll(v[w]));
    return -1;
}

/* Greedy insertion with the pivot at the highest set bit; returns 1 when
 * the vector was independent (stored at its pivot), 0 otherwise. */
static int pivot_try_insert(uint64_t* basis, unsigned char* used, const uint64_t* cand, size_t mw,
                            uint64_t* tmp) {
    memcpy(tmp, cand, mw * sizeof(uint64_t));
    for (;;) {
        const int hb = highest_bit_words(tmp, mw);
        if (hb < 0)
            return 0;
        if (!used[hb]) {
            used[hb] = 1;
            memcpy(basis + (size_t)hb * mw, tmp, mw * sizeof(uint64_t));
            return 1;
        }
        for (size_t w = 0; w < mw; ++w)
            tmp[w] ^= basis[(size_t)hb * mw + w];
    }
}

typedef struct {
    uint32_t weight;
    uint32_t pc;
    size_t idx;
} orc_pool_entry;

static int pool_cmp(const void* a, const void* b) {
    const orc_pool_entry* x = (const orc_pool_entry*)a;
    const orc_pool_entry* y = (const orc_pool_entry*)b;
    if (x->weight != y->weight)
        return x->weight < y->weight ? -1 : 1;
    if (x->pc != y->pc)
        return x->pc < y->pc ? -1 : 1;
    return x->idx < y->idx ? -1 : (x->idx > y->idx); /* stable */
}

void orc_crossover(size_t n, size_t parents, const uint64_t* parent_masks,
                   const uint32_t* parent_weights, uint64_t* child_masks, uint32_t* child_weights) {
    const size_t mw = (n + 63) / 64, pool = parents * n;
    orc_pool_entry* e = (orc_pool_entry*)malloc(pool * sizeof(orc_pool_entry));
    for (size_t q = 0; q < pool; ++q) {
        uint32_t pc = 0;
        for (size_t w = 0; w < mw; ++w)
            pc += popc64(parent_masks[q * mw + w]);
        e[q].weight = parent_weights[q];
        e[q].pc = pc;
        e[q].idx = q;
    }
    qsort(e, pool, sizeof(orc_pool_entry), pool_cmp);
    uint64_t* basis = (uint64_t*)calloc(n * mw, sizeof(uint64_t));
    unsigned char* used = (unsigned char*)calloc(n, 1);
    uint64_t* tmp = (uint64_t*)malloc(mw * sizeof(uint64_t));
    uint64_t* unit = (uint64_t*)malloc(mw * sizeof(uint64_t));
    size_t nchild = 0;
    for (size_t q = 0; q < pool && nchild < n; ++q)
        if (pivot_try_insert(basis, used, parent_masks + e[q].idx * mw, mw, tmp)) {
            memcpy(child_masks + nchild * mw, parent_masks + e[q].idx * mw, mw * sizeof(uint64_t));
            child_weights[nchild++] = parent_weights[e[q].idx];
        }
    for (size_t i = 0; i < n && nchild < n; ++i) {
        memset(unit, 0, mw * sizeof(uint64_t));
        unit[i / 64] = (uint64_t)1 << (i % 64);
        if (pivot_try_insert(basis, used, unit, mw, tmp)) {
            memcpy(child_masks + nchild * mw, unit, mw * sizeof(uint64_t));
            child_weights[nchild++] = 1; /* Candidate(unit_mask, 1) */
        }
    }
    free(unit);
    free(tmp);
    free(used);
    free(basis);
    free(e);
}

/* ---- One GeneticAlgorithm run (src/ga/genetic_algorithm_lifecycle.cpp:16-200,
 * genetic_algorithm_population.cpp:10-83, genetic_algorithm_operators.cpp:15-192,
 * genetic_algorithm_core.cpp:10-41). ---- */
typedef struct {
    const uint64_t* words;
    size_t stride, cols, n, mw, P;
    const size_t* win;
    const orc_ga_config* cfg;
    uint64_t rng;
    double rate;
} orc_ga_ctx;

static uint64_t ind_fitness(const uint32_t* w, size_t n) {
    uint64_t s = 0;
    for (size_t i = 0; i < n; ++i)
        s += w[i];
    return s;
}

static uint32_t row_popcount(const orc_ga_ctx* g, size_t r) {
    const size_t wpr = (g->cols + 63) / 64;
    const uint64_t tail = tail_mask_for_cols(g->cols);
    uint32_t s = 0;
    for (size_t w = 0; w < wpr; ++w) {
        uint64_t v = g->words[g->win[r] * g->stride + w];
        if (w + 1 == wpr)
            v &= tail;
        s += popc64(v);
    }
    return s;
}

static void make_identity(const orc_ga_ctx* g, uint64_t* m, uint32_t* w) {
    memset(m, 0, g->n * g->mw * sizeof(uint64_t));
    for (size_t i = 0; i < g->n; ++i) {
        m[i * g->mw + i / 64] = (uint64_t)1 << (i % 64);
        w[i] = row_popcount(g, i);
    }
}

static void make_random(orc_ga_ctx* g, uint64_t* m, uint32_t* w) {
    make_identity(g, m, w);
    for (size_t k = 0; k < g->n * 3; ++k) {
        const size_t i = xs_index(&g->rng, g->n);
        const size_t j = xs_index(&g->rng, g->n);
        if (i == j)
            continue;
        for (size_t q = 0; q < g->mw; ++q)
            m[i * g->mw + q] ^= m[j * g->mw + q];
    }
    for (size_t i = 0; i < g->n; ++i)
        w[i] = orc_eval_cand_weight(g->words, g->stride, g->cols, g->win, g->n, m + i * g->mw,
                                    g->mw);
}

static void make_heuristic(const orc_ga_ctx* g, uint64_t* m, uint32_t* w) {
    make_identity(g, m, w);
    const size_t n = g->n, mw = g->mw;
    if (n < 2)
        return;
    size_t* order = (size_t*)malloc(n * sizeof(size_t));
    for (size_t i = 0; i < n; ++i)
        order[i] = i;
    for (size_t a = 1; a < n; ++a) { /* stable insertion sort, descending weight */
        const size_t v = order[a];
        size_t b = a;
        while (b > 0 && w[order[b - 1]] < w[v]) {
            order[b] = order[b - 1];
            --b;
        }
        order[b] = v;
    }
    const size_t probes = n < 5 ? n : 5;
    for (size_t pos = 0; pos < probes; ++pos) {
        const size_t i = order[pos];
        uint32_t cur = w[i];
        for (size_t j = 0; j < n; ++j) {
            if (i == j)
                continue;
            for (size_t q = 0; q < mw; ++q)
                m[i * mw + q] ^= m[j * mw + q];
            const uint32_t cw =
                orc_eval_cand_weight(g->words, g->stride, g->cols, g->win, n, m + i * mw, mw);
            if (cw < cur) {
                w[i] = cw;
                cur = cw;
                break;
            }
            for (size_t q = 0; q < mw; ++q)
                m[i * mw + q] ^= m[j * mw + q];
        }
    }
    free(order);
}

typedef struct {
    uint64_t fit;
    size_t idx;
} orc_rank;

static int rank_cmp(const void* a, const void* b) {
    const orc_rank* x = (const orc_rank*)a;
    const orc_rank* y = (const orc_rank*)b;
    if (x->fit != y->fit)
        return x->fit < y->fit ? -1 : 1;
    return x->idx < y->idx ? -1 : (x->idx > y->idx);
}

static int should_stop(const orc_ga_config* c, uint64_t gens, uint64_t stale, uint64_t best) {
    if ((c->flags & 1u) && gens >= c->max_generations)
        return 1;
    if ((c->flags & 2u) && stale >= c->max_stale_generations)
        return 1;
    if ((c->flags & 4u) && best <= c->target_total_weight)
        return 1;
    return 0;
}

long orc_ga_run(const uint64_t* words, size_t stride, size_t cols, const size_t* win, size_t n,
                const orc_ga_config* cfg, uint64_t seed, uint64_t max_steps, uint64_t* scores,
                uint64_t* best_masks, uint32_t* best_weights) {
    orc_ga_ctx g;
    g.words = words;
    g.stride = stride;
    g.cols = cols;
    g.win = win;
    g.n = n;
    g.mw = (n + 63) / 64;
    g.P = cfg->population_size;
    g.cfg = cfg;
    g.rng = orc_xs_seed(seed);
    g.rate = cfg->mutation_rate;
    if (n == 0 || cols == 0 || g.P == 0)
        return ORC_EINVAL;
    const size_t P = g.P, mw = g.mw, isz = n * mw;
    uint64_t* pm = (uint64_t*)malloc(P * isz * sizeof(uint64_t));
    uint32_t* pw = (uint32_t*)malloc(P * n * sizeof(uint32_t));
    uint64_t* nm = (uint64_t*)malloc(P * isz * sizeof(uint64_t));
    uint32_t* nw = (uint32_t*)malloc(P * n * sizeof(uint32_t));
    uint64_t* fit = (uint64_t*)malloc(P * sizeof(uint64_t));
    orc_rank* rk = (orc_rank*)malloc(P * sizeof(orc_rank));
    const size_t np = cfg->num_parents ? cfg->num_parents : 1;
    uint64_t* par_m = (uint64_t*)malloc(np * isz * sizeof(uint64_t));
    uint32_t* par_w = (uint32_t*)malloc(np * n * sizeof(uint32_t));
    uint64_t* child_m = (uint64_t*)malloc(isz * sizeof(uint64_t));
    uint32_t* child_w = (uint32_t*)malloc(n * sizeof(uint32_t));

    /* initialize */
    make_identity(&g, pm, pw);
    size_t heur = P / 4 < P - 1 ? P / 4 : P - 1;
    size_t filled = 1;
    for (size_t i = 0; i < heur; ++i, ++filled)
        make_heuristic(&g, pm + filled * isz, pw + filled * n);
    for (; filled < P; ++filled)
        make_random(&g, pm + filled * isz, pw + filled * n);
    for (size_t i = 0; i < P; ++i)
        fit[i] = ind_fitness(pw + i * n, n);
    size_t bi = 0;
    for (size_t i = 1; i < P; ++i)
        if (fit[i] < fit[bi])
            bi = i;
    uint64_t best = fit[bi];
    memcpy(best_masks, pm + bi * isz, isz * sizeof(uint64_t));
    memcpy(best_weights, pw + bi * n, n * sizeof(uint32_t));
    uint64_t gens = 0, stale = 0, no_imp = 0, cat = 0;
    scores[0] = best;
    int done = should_stop(cfg, gens, stale, best);
    long steps = 0;
    while (!done && (uint64_t)steps < max_steps) {
        /* adapt_mutation_rate */
        if (no_imp > 10)
            g.rate = g.rate * 1.5 < 0.8 ? g.rate * 1.5 : 0.8;
        else if (no_imp > 5)
            g.rate = g.rate * 1.3 < 0.6 ? g.rate * 1.3 : 0.6;
        else
            g.rate = g.rate * 0.95 > 0.3 ? g.rate * 0.95 : 0.3;
        for (size_t i = 0; i < P; ++i) {
            rk[i].fit = fit[i];
            rk[i].idx = i;
        }
        qsort(rk, P, sizeof(orc_rank), rank_cmp);
        size_t out = 0;
        for (size_t e = 0; e < cfg->elite_count && e < P; ++e, ++out) {
            memcpy(nm + out * isz, pm + rk[e].idx * isz, isz * sizeof(uint64_t));
            memcpy(nw + out * n, pw + rk[e].idx * n, n * sizeof(uint32_t));
        }
        while (out < P) {
            if (no_imp > 15 && xs_unit(&g.rng) < 0.2) {
                make_random(&g, nm + out * isz, nw + out * n);
                ++out;
                continue;
            }
            for (size_t p = 0; p < np; ++p) { /* tournament_selection */
                size_t b = xs_index(&g.rng, P);
                for (size_t t = 1; t < cfg->tournament_size; ++t) {
                    const size_t c = xs_index(&g.rng, P);
                    if (fit[c] < fit[b])
                        b = c;
                }
                memcpy(par_m + p * isz, pm + b * isz, isz * sizeof(uint64_t));
                memcpy(par_w + p * n, pw + b * n, n * sizeof(uint32_t));
            }
            orc_crossover(n, np, par_m, par_w, child_m, child_w);
            for (size_t o = 0; o < cfg->num_offspring && out < P; ++o, ++out) {
                uint64_t* cm = nm + out * isz;
                uint32_t* cw = nw + out * n;
                memcpy(cm, child_m, isz * sizeof(uint64_t));
                memcpy(cw, child_w, n * sizeof(uint32_t));
                orc_mutate(words, stride, cols, win, n, cm, cw, mw, g.rate, &g.rng);
                if (gens % 3 == 0)
                    orc_local_improvement(words, stride, cols, win, n, cm, cw, mw);
            }
        }
        uint64_t* tm = pm;
        pm = nm;
        nm = tm;
        uint32_t* tw = pw;
        pw = nw;
        nw = tw;
        for (size_t i = 0; i < P; ++i)
            fit[i] = ind_fitness(pw + i * n, n);
        ++gens;
        bi = 0;
        for (size_t i = 1; i < P; ++i)
            if (fit[i] < fit[bi])
                bi = i;
        if (fit[bi] < best) {
            best = fit[bi];
            memcpy(best_masks, pm + bi * isz, isz * sizeof(uint64_t));
            memcpy(best_weights, pw + bi * n, n * sizeof(uint32_t));
            stale = 0;
            no_imp = 0;
            cat = 0;
        } else {
            ++stale;
            ++no_imp;
            ++cat;
        }
        if (cfg->enable_catastrophe && cat == cfg->catastrophe_threshold) {
            /* catastrophe(): ranked survivors, then make_random */
            const size_t sv = (size_t)((double)P * cfg->catastrophe_survival_rate);
            for (size_t i = 0; i < P; ++i) {
                rk[i].fit = fit[i];
                rk[i].idx = i;
            }
            qsort(rk, P, sizeof(orc_rank), rank_cmp);
            size_t o = 0;
            for (; o < sv && o < P; ++o) {
                memcpy(nm + o * isz, pm + rk[o].idx * isz, isz * sizeof(uint64_t));
                memcpy(nw + o * n, pw + rk[o].idx * n, n * sizeof(uint32_t));
            }
            for (; o < P; ++o)
                make_random(&g, nm + o * isz, nw + o * n);
            tm = pm;
            pm = nm;
            nm = tm;
            tw = pw;
            pw = nw;
            nw = tw;
            for (size_t i = 0; i < P; ++i)
                fit[i] = ind_fitness(pw + i * n, n);
            cat = 0;
            bi = 0;
            for (size_t i = 1; i < P; ++i)
                if (fit[i] < fit[bi])
                    bi = i;
            if (fit[bi] < best) {
                best = fit[bi];
                memcpy(best_masks, pm + bi * isz, isz * sizeof(uint64_t));
                memcpy(best_weights, pw + bi * n, n * sizeof(uint32_t));
            }
        }
        done = should_stop(cfg, gens, stale, best);
        ++steps;
        scores[steps] = best;
    }
    free(child_w);
    free(child_m);
    free(par_w);
    free(par_m);
    free(rk);
    free(fit);
    free(nw);
    free(nm);
    free(pw);
    free(pm);
    return steps;
}

/* ---- ExactBasisSolver (src/solver/exact_basis_solver.cpp:29-157) ---------- */
static void window_rows(const uint64_t* words, size_t stride, size_t cols, const size_t* win,
                        size_t t, uint64_t* rows) {
    const size_t W = (cols + 63) / 64;
    const uint64_t tail = tail_mask_for_cols(cols);
    for (size_t r = 0; r < t; ++r)
        for (size_t w = 0; w < W; ++w)
            rows[r * W + w] = words[win[r] * stride + w] & (w + 1 == W ? tail : ~0ull);
}

static uint32_t combo_weight(const uint64_t* cur, size_t W) {
    uint32_t s = 0;
    for (size_t w = 0; w < W; ++w)
        s += popc64(cur[w]);
    return s;
}

int orc_basis_weight_counts(const uint64_t* words, size_t stride, size_t cols, const size_t* win,
                            size_t t, uint64_t* counts) {
    const size_t W = (cols + 63) / 64;
    memset(counts, 0, (cols + 1) * sizeof(uint64_t));
    if (t == 0)
        return 0;
    if (t > 32)
        return -1;
    uint64_t* rows = (uint64_t*)calloc(t * W + 1, sizeof(uint64_t));
    uint64_t* cur = (uint64_t*)calloc(W + 1, sizeof(uint64_t));
    if (!rows || !cur) {
        free(rows);
        free(cur);
        return -2;
    }
    window_rows(words, stride, cols, win, t, rows);
    const uint64_t states = (1ull << t) - 1;
    uint32_t prev = 0;
    for (uint64_t index = 1; index <= states; ++index) {
        const uint32_t gray = (uint32_t)(index ^ (index >> 1));
        const size_t r = ctz64((uint64_t)(gray ^ prev));
        for (size_t w = 0; w < W; ++w)
            cur[w] ^= rows[r * W + w];
        ++counts[combo_weight(cur, W)];
        prev = gray;
    }
    free(rows);
    free(cur);
    return 0;
}

long orc_exact_basis(const uint64_t* words, size_t stride, size_t cols, const size_t* win,
                     size_t t, uint32_t* masks, uint32_t* weights, uint64_t* total) {
    *total = 0;
    if (t == 0)
        return 0;
    if (t > 32)
        return -1;
    const size_t W = (cols + 63) / 64, mw = W ? W : 1;
    const uint64_t states = (1ull << t) - 1;
    uint64_t* rows = (uint64_t*)calloc(t * mw, sizeof(uint64_t));
    uint64_t* cur = (uint64_t*)calloc(mw, sizeof(uint64_t));
    uint64_t* tmp = (uint64_t*)calloc(mw, sizeof(uint64_t));
    uint64_t* basis = (uint64_t*)calloc((cols + 1) * mw, sizeof(uint64_t));
    unsigned char* used = (unsigned char*)calloc(cols + 1, 1);
    uint64_t* offs = (uint64_t*)calloc(cols + 2, sizeof(uint64_t));
    uint32_t* packed = (uint32_t*)malloc((size_t)states * sizeof(uint32_t));
    long rc = -2;
    if (!rows || !cur || !tmp || !basis || !used || !offs || !packed)
        goto done;
    window_rows(words, stride, cols, win, t, rows);
    /* rank of the materialized window */
    size_t rank = 0;
    for (size_t r = 0; r < t; ++r)
        rank += (size_t)pivot_try_insert(basis, used, rows + r * mw, mw, tmp);
    memset(basis, 0, (cols + 1) * mw * sizeof(uint64_t));
    memset(used, 0, cols + 1);
    if (rank == 0) {
        rc = 0;
        goto done;
    }
    /* counting sort of the Gray enumeration by weight */
    for (int pass = 0; pass < 2; ++pass) {
        uint32_t prev = 0;
        memset(cur, 0, mw * sizeof(uint64_t));
        for (uint64_t index = 1; index <= states; ++index) {
            const uint32_t gray = (uint32_t)(index ^ (index >> 1));
            const size_t r = ctz64((uint64_t)(gray ^ prev));
            for (size_t w = 0; w < mw; ++w)
                cur[w] ^= rows[r * mw + w];
            const uint32_t wt = combo_weight(cur, mw);
            if (pass == 0)
                ++offs[wt + 1];
            else
                packed[offs[wt]++] = gray;
            prev = gray;
        }
        if (pass == 0)
            for (size_t w = 0; w <= cols; ++w)
                offs[w + 1] += offs[w];
        else
            for (size_t w = cols + 1; w-- > 0;)
                offs[w + 1] = offs[w]; /* restore bucket starts */
        if (pass == 1)
            offs[0] = 0;
    }
    /* greedy insertion, lightest bucket first */
    size_t got = 0;
    for (size_t wt = 0; wt <= cols && got < rank; ++wt)
        for (uint64_t i = offs[wt]; i < offs[wt + 1] && got < rank; ++i) {
            const uint32_t mask = packed[i];
            memset(cur, 0, mw * sizeof(uint64_t));
            for (size_t r = 0; r < t; ++r)
                if ((mask >> r) & 1u)
                    for (size_t w = 0; w < mw; ++w)
                        cur[w] ^= rows[r * mw + w];
            if (!pivot_try_insert(basis, used, cur, mw, tmp))
                continue;
            masks[got] = mask;
            weights[got] = (uint32_t)wt;
            *total += wt;
            ++got;
        }
    rc = (long)got;
done:
    free(rows);
    free(cur);
    free(tmp);
    free(basis);
    free(used);
    free(offs);
    free(packed);
    return rc;
}

/* ---- SASelector (src/search/sa_selector*.cpp) ------------------------------ */
typedef struct {
    const uint64_t* words;
    size_t stride, cols, W, n;
    uint64_t tail;
    int policy;
    uint32_t* table;  /* pairwise: n x n synergy 2*popc(ri & rj) */
    uint32_t* count;  /* higher order: per-column counts of the window */
} orc_sa;

static uint64_t sa_word(const orc_sa* S, size_t r, size_t w) {
    const uint64_t v = S->words[r * S->stride + w];
    return w + 1 == S->W ? (v & S->tail) : v;
}

static int64_t ho_term(uint32_t c) {
    const int64_t n = (int64_t)c;
    return n * (n - 1) * (n - 1);
}

static int64_t sa_score(orc_sa* S, const size_t* win, size_t t) {
    int64_t s = 0;
    if (S->policy == 0) {
        for (size_t i = 0; i < t; ++i)
            for (size_t j = i + 1; j < t; ++j)
                s += (int64_t)S->table[win[i] * S->n + win[j]];
        return s;
    }
    memset(S->count, 0, S->cols * sizeof(uint32_t));
    for (size_t i = 0; i < t; ++i)
        for (size_t w = 0; w < S->W; ++w)
            for (uint64_t b = sa_word(S, win[i], w); b; b &= b - 1)
                ++S->count[w * 64 + ctz64(b)];
    for (size_t c = 0; c < S->cols; ++c)
        s += ho_term(S->count[c]);
    return s;
}

static int64_t sa_delta(const orc_sa* S, const size_t* win, size_t t, size_t out_idx, size_t in) {
    const size_t out = win[out_idx];
    int64_t d = 0;
    if (S->policy == 0) {
        for (size_t i = 0; i < t; ++i) {
            if (i == out_idx)
                continue;
            d += (int64_t)S->table[in * S->n + win[i]];
            d -= (int64_t)S->table[out * S->n + win[i]];
        }
        return d;
    }
    for (size_t w = 0; w < S->W; ++w) {
        const uint64_t o = sa_word(S, out, w), a = sa_word(S, in, w);
        for (uint64_t b = o & ~a; b; b &= b - 1) {
            const uint32_t c = S->count[w * 64 + ctz64(b)];
            d += ho_term(c - 1) - ho_term(c);
        }
        for (uint64_t b = a & ~o; b; b &= b - 1) {
            const uint32_t c = S->count[w * 64 + ctz64(b)];
            d += ho_term(c + 1) - ho_term(c);
        }
    }
    return d;
}

static void sa_moved(orc_sa* S, size_t out, size_t in) {
    if (S->policy == 0)
        return;
    for (size_t w = 0; w < S->W; ++w) {
        const uint64_t o = sa_word(S, out, w), a = sa_word(S, in, w);
        for (uint64_t b = o & ~a; b; b &= b - 1)
            --S->count[w * 64 + ctz64(b)];
        for (uint64_t b = a & ~o; b; b &= b - 1)
            ++S->count[w * 64 + ctz64(b)];
    }
}

static int cmp_size(const void* a, const void* b) {
    const size_t x = *(const size_t*)a, y = *(const size_t*)b;
    return x < y ? -1 : x > y;
}

/* lexicographic comparison of two sorted row lists of length t */
static int rows_less(const size_t* a, const size_t* b, size_t t) {
    for (size_t i = 0; i < t; ++i)
        if (a[i] != b[i])
            return a[i] < b[i];
    return 0;
}

static int sa_better(int64_t ls, const size_t* lr, int64_t rs, const size_t* rr, size_t t) {
    return ls != rs ? ls > rs : rows_less(lr, rr, t);
}

typedef struct {
    int64_t score;
    uint64_t accepted, iterations_run, best_iteration;
} orc_sa_restart;

static void sa_restart(orc_sa* S, size_t t, uint64_t iterations, uint64_t probe_samples,
                       double p0, double cooling, double min_temp, uint64_t* rng,
                       size_t* win, size_t* pool, size_t* tmp, size_t* best_rows,
                       orc_sa_restart* best) {
    const size_t n = S->n, np = n - t;
    for (size_t i = 0; i < n; ++i)
        pool[i] = i;
    for (size_t i = 0; i < t; ++i) {
        const size_t j = i + xs_index(rng, n - i);
        const size_t x = pool[i];
        pool[i] = pool[j];
        pool[j] = x;
    }
    memcpy(win, pool, t * sizeof(size_t));
    memmove(pool, pool + t, np * sizeof(size_t));
    int64_t score = sa_score(S, win, t);
    memcpy(best_rows, win, t * sizeof(size_t));
    qsort(best_rows, t, sizeof(size_t), cmp_size);
    best->score = score;
    best->accepted = 0;
    best->best_iteration = 0;
    best->iterations_run = np == 0 ? 0 : iterations;
    if (np == 0 || iterations == 0)
        return;
    double temp = 1.0;
    {
        const uint64_t samples = probe_samples > 1 ? probe_samples : 1;
        double neg_sum = 0.0;
        uint64_t neg = 0;
        for (uint64_t k = 0; k < samples; ++k) {
            const size_t iw = xs_index(rng, t);
            const size_t ip = xs_index(rng, np);
            const int64_t d = sa_delta(S, win, t, iw, pool[ip]);
            if (d < 0) {
                neg_sum += (double)(-d);
                ++neg;
            }
        }
        if (neg) {
            const double avg = neg_sum / (double)neg;
            const double t0 = -avg / log(p0);
            temp = t0 < min_temp ? min_temp : t0;
        }
    }
    uint64_t accepted = 0;
    for (uint64_t it = 0; it < iterations; ++it) {
        const size_t iw = xs_index(rng, t);
        const size_t ip = xs_index(rng, np);
        const size_t in = pool[ip];
        const int64_t d = sa_delta(S, win, t, iw, in);
        int accept = d > 0;
        if (!accept && temp > min_temp)
            accept = xs_unit(rng) < exp((double)d / temp);
        if (accept) {
            sa_moved(S, win[iw], in);
            pool[ip] = win[iw];
            win[iw] = in;
            score += d;
            ++accepted;
            memcpy(tmp, win, t * sizeof(size_t));
            qsort(tmp, t, sizeof(size_t), cmp_size);
            if (sa_better(score, tmp, best->score, best_rows, t)) {
                memcpy(best_rows, tmp, t * sizeof(size_t));
                best->score = score;
                best->accepted = accepted;
                best->best_iteration = it + 1;
            }
        }
        const double next = temp * cooling;
        temp = min_temp < next ? next : min_temp;
    }
}

long orc_sa_select(const uint64_t* words, size_t stride, size_t rows, size_t cols,
                   size_t window_size, uint64_t iterations, uint64_t restarts, uint64_t seed,
                   int score_policy, uint64_t probe_samples, double p0, double cooling,
                   double min_temp, int64_t* scalars, size_t* out_rows) {
    if (restarts == 0 || !(p0 > 0.0 && p0 < 1.0) || cooling <= 0.0 || cooling > 1.0 ||
        min_temp <= 0.0 || window_size > rows)
        return -1;
    memset(scalars, 0, 6 * sizeof(int64_t));
    uint64_t rng = orc_xs_seed(seed);
    scalars[5] = (int64_t)rng;
    if (window_size == 0)
        return 0;
    orc_sa S = {words, stride, cols, (cols + 63) / 64, rows, tail_mask_for_cols(cols),
                score_policy, NULL, NULL};
    if (score_policy == 0) {
        S.table = (uint32_t*)calloc(rows * rows, sizeof(uint32_t));
        for (size_t i = 0; i < rows; ++i)
            for (size_t j = i + 1; j < rows; ++j) {
                uint64_t ov = 0;
                for (size_t w = 0; w < S.W; ++w)
                    ov += popc64(sa_word(&S, i, w) & sa_word(&S, j, w));
                S.table[i * rows + j] = S.table[j * rows + i] = (uint32_t)(2 * ov);
            }
    } else {
        S.count = (uint32_t*)calloc(cols + 1, sizeof(uint32_t));
    }
    const size_t t = window_size;
    size_t* win = (size_t*)malloc(t * sizeof(size_t));
    size_t* pool = (size_t*)malloc(rows * sizeof(size_t));
    size_t* tmp = (size_t*)malloc(t * sizeof(size_t));
    size_t* cand = (size_t*)malloc(t * sizeof(size_t));
    orc_sa_restart best, r;
    int have = 0;
    for (uint64_t k = 0; k < restarts; ++k) {
        sa_restart(&S, t, iterations, probe_samples, p0, cooling, min_temp, &rng, win, pool, tmp,
                   cand, &r);
        if (!have || sa_better(r.score, cand, best.score, out_rows, t)) {
            best = r;
            memcpy(out_rows, cand, t * sizeof(size_t));
            scalars[4] = (int64_t)k;
            have = 1;
        }
    }
    scalars[0] = best.score;
    scalars[1] = (int64_t)best.accepted;
    scalars[2] = (int64_t)best.iterations_run;
    scalars[3] = (int64_t)best.best_iteration;
    free(S.table);
    free(S.count);
    free(win);
    free(pool);
    free(tmp);
    free(cand);
    return (long)t;
}
