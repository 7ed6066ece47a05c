// Population counts on the integer pipes: the carry-save (Harley-Seal)
// reduction that moves most of a row's popcount from the quarter-rate POPC
// unit (XU pipe) to LOP3 on the ALU pipe, shared by the Gray-code kernels.
#pragma once

#include <cstdint>

namespace bmm {

// Carry-save adder: l = a ^ b ^ c (weight 1), h = majority(a, b, c) (weight 2).
__device__ __forceinline__ void csa(uint32_t& h, uint32_t& l, uint32_t a, uint32_t b, uint32_t c) {
    const uint32_t u = a ^ b;
    h = (a & b) | (u & c);
    l = u ^ c;
}

// Harley-Seal step over 16 words (Mula, Kurz, Lemire, "Faster population
// counts using AVX2 instructions", 2018): 15 carry-save adders fold the block
// into running ones/twos/fours/eights and emit one "sixteens" word, so 16
// words cost 30 LOP3 + 1 POPC instead of 16 POPC.
__device__ __forceinline__ void hs16(const uint32_t (&d)[16], uint32_t& ones, uint32_t& twos,
                                     uint32_t& fours, uint32_t& eights, uint32_t& n16) {
    uint32_t twosA, twosB, foursA, foursB, eightsA, eightsB, sixteens;
    csa(twosA, ones, ones, d[0], d[1]);
    csa(twosB, ones, ones, d[2], d[3]);
    csa(foursA, twos, twos, twosA, twosB);
    csa(twosA, ones, ones, d[4], d[5]);
    csa(twosB, ones, ones, d[6], d[7]);
    csa(foursB, twos, twos, twosA, twosB);
    csa(eightsA, fours, fours, foursA, foursB);
    csa(twosA, ones, ones, d[8], d[9]);
    csa(twosB, ones, ones, d[10], d[11]);
    csa(foursA, twos, twos, twosA, twosB);
    csa(twosA, ones, ones, d[12], d[13]);
    csa(twosB, ones, ones, d[14], d[15]);
    csa(foursB, twos, twos, twosA, twosB);
    csa(eightsB, fours, fours, foursA, foursB);
    csa(sixteens, eights, eights, eightsA, eightsB);
    n16 += __popc(sixteens);
}

// XOR a shared-memory row into cur and return popcount(cur).  The first
// NHB blocks of 8 words go through the carry-save tree (ALU pipe), the rest
// through POPC (XU pipe); NHB balances the two pipes.
// `step` is the distance, in 16-byte chunks, between consecutive chunks of
// the row (1 for a contiguous row).
template <int WPL, int NHB>
__device__ __forceinline__ uint32_t xor_row_popc_hs(uint64_t (&cur)[WPL], const uint64_t* srow,
                                                    int step = 1) {
    static_assert(NHB * 8 <= WPL, "carry-save blocks exceed the row");
    const ulonglong2* p = reinterpret_cast<const ulonglong2*>(srow);
    uint32_t ones = 0, twos = 0, fours = 0, eights = 0, n16 = 0;
#pragma unroll
    for (int blk = 0; blk < NHB; ++blk) {
        uint32_t d[16];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const ulonglong2 v = p[(blk * 4 + j) * step];
            uint64_t& a = cur[blk * 8 + 2 * j];
            uint64_t& b = cur[blk * 8 + 2 * j + 1];
            a ^= v.x;
            b ^= v.y;
            d[4 * j + 0] = (uint32_t)a;
            d[4 * j + 1] = (uint32_t)(a >> 32);
            d[4 * j + 2] = (uint32_t)b;
            d[4 * j + 3] = (uint32_t)(b >> 32);
        }
        hs16(d, ones, twos, fours, eights, n16);
    }
    uint32_t s = 0;
#pragma unroll
    for (int i = NHB * 4; i < WPL / 2; ++i) {
        const ulonglong2 v = p[i * step];
        cur[2 * i] ^= v.x;
        cur[2 * i + 1] ^= v.y;
        s += __popcll(cur[2 * i]) + __popcll(cur[2 * i + 1]);
    }
    if (NHB > 0)
        s += 16 * n16 + 8 * __popc(eights) + 4 * __popc(fours) + 2 * __popc(twos) + __popc(ones);
    return s;
}

// a * m + c as an integer multiply-add.  With m a value the compiler cannot
// see (a kernel argument holding 1, or a power of two derived from one), the
// add is an IMAD on the FMA pipe, which the XOR/popcount work leaves idle,
// instead of an IADD on the ALU pipe, which bounds the Gray-code kernels.
__device__ __forceinline__ uint32_t mad_u32(uint32_t a, uint32_t m, uint32_t c) {
    uint32_t d;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(m), "r"(c));
    return d;
}

// xor_row_popc_hs with every popcount accumulated through mad_u32(., one, .)
// (`one` == 1 at run time): same result, fewer ALU-pipe instructions.
template <int WPL, int NHB>
__device__ __forceinline__ uint32_t xor_row_popc_hs_fma(uint64_t (&cur)[WPL],
                                                        const uint64_t* srow, uint32_t one) {
    static_assert(NHB * 8 <= WPL, "carry-save blocks exceed the row");
    const ulonglong2* p = reinterpret_cast<const ulonglong2*>(srow);
    uint32_t ones = 0, twos = 0, fours = 0, eights = 0, n16 = 0;
#pragma unroll
    for (int blk = 0; blk < NHB; ++blk) {
        uint32_t d[16];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const ulonglong2 v = p[blk * 4 + j];
            uint64_t& a = cur[blk * 8 + 2 * j];
            uint64_t& b = cur[blk * 8 + 2 * j + 1];
            a ^= v.x;
            b ^= v.y;
            d[4 * j + 0] = (uint32_t)a;
            d[4 * j + 1] = (uint32_t)(a >> 32);
            d[4 * j + 2] = (uint32_t)b;
            d[4 * j + 3] = (uint32_t)(b >> 32);
        }
        uint32_t sixteens_count = 0;
        hs16(d, ones, twos, fours, eights, sixteens_count);
        n16 = mad_u32(sixteens_count, one, n16);
    }
    uint32_t s = 0;
#pragma unroll
    for (int i = NHB * 4; i < WPL / 2; ++i) {
        const ulonglong2 v = p[i];
        cur[2 * i] ^= v.x;
        cur[2 * i + 1] ^= v.y;
        s = mad_u32(__popcll(cur[2 * i]), one, s);
        s = mad_u32(__popcll(cur[2 * i + 1]), one, s);
    }
    if (NHB > 0) {
        const uint32_t two = one + one, four = two + two, eight = four + four;
        s = mad_u32(n16, eight + eight, s);
        s = mad_u32(__popc(eights), eight, s);
        s = mad_u32(__popc(fours), four, s);
        s = mad_u32(__popc(twos), two, s);
        s = mad_u32(__popc(ones), one, s);
    }
    return s;
}

// Blocks of 8 words per row that go through the carry-save tree, by words
// per lane: balances the ALU and XU pipes (measured on the Gray kernels).
constexpr int default_nhb(int wpl) { return wpl >= 64 ? 5 : wpl >= 32 ? 2 : wpl >= 16 ? 1 : 0; }

}  // namespace bmm
