// Matrix text and binary formats and the matrix hash
// (src/core/bit_matrix_io.cpp:34-175, src/core/bit_matrix_hash.cpp:30-58).
//
// Text ("rows cols\n" then rows x cols '0'/'1' characters, any ASCII
// whitespace between them) is parsed and written on the device: the payload is
// one pass of byte classification, a prefix sum of the bit characters, and a
// scatter of bit i to (row i / cols, column i % cols); the reference's three
// failure modes follow from positions -- the first character that is neither a
// bit nor whitespace, and the position of the last payload bit.  Writing gives
// every output byte its own thread.  Binary ("BMMPYB1\0", u64 rows, u64 cols,
// then (cols + 63) / 64 unpadded words per row) streams through pinned host
// memory into the padded device layout with strided copies.  The hash is
// SHA-256 (FIPS 180-4) over the little-endian u64 sequence rows, cols, then
// the row words with the bits past cols cleared -- one sequential chain, so
// it runs on the host.
#include "common.cuh"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace bmm {
namespace io {

constexpr int kChunk = 8192;      // text bytes per CTA
constexpr int kPerThread = 32;    // text bytes per thread (256 threads)

__device__ __forceinline__ bool is_ws(unsigned char c) {
    return c == ' ' || c == '\n' || c == '\r' || c == '\t' || c == '\f' || c == '\v';
}

// The 32 text bytes of thread j of CTA b, [b * kChunk + 32 j, + 32), as
// eight little-endian words: two 16-byte loads when the run is whole and
// aligned, else byte by byte (past the end: spaces).
__device__ __forceinline__ void load32(const unsigned char* __restrict__ text,
                                       unsigned long long len, unsigned long long p,
                                       uint32_t (&w)[8]) {
    if (p + kPerThread <= len && ((reinterpret_cast<uintptr_t>(text + p) & 15) == 0)) {
        const uint4 x = *reinterpret_cast<const uint4*>(text + p);
        const uint4 y = *reinterpret_cast<const uint4*>(text + p + 16);
        w[0] = x.x, w[1] = x.y, w[2] = x.z, w[3] = x.w;
        w[4] = y.x, w[5] = y.y, w[6] = y.z, w[7] = y.w;
    } else {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            uint32_t v = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const unsigned long long q = p + 4 * i + k;
                v |= (uint32_t)(q < len ? text[q] : (unsigned char)' ') << (8 * k);
            }
            w[i] = v;
        }
    }
}

// Classes of a thread's 32 bytes as bit masks (byte k at bit k): bit
// characters '0'/'1', the '1's, and bytes that are neither bits nor ASCII
// whitespace (' ', '\t' .. '\r').  Four bits at a time when all four bytes
// are bit characters (the common case), byte by byte otherwise.
struct Classes {
    uint32_t bit, one, other;
};

__device__ __forceinline__ Classes classify(const uint32_t (&w)[8]) {
    Classes c{0, 0, 0};
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const uint32_t t = w[i] ^ 0x30303030u;  // '0' -> 0, '1' -> 1
        if ((t & 0xfefefefeu) == 0) {
            c.bit |= 0xfu << (4 * i);
            c.one |= ((t * 0x10204080u) >> 28) << (4 * i);
        } else {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const uint32_t ch = (w[i] >> (8 * k)) & 0xffu;
                const uint32_t at = 1u << (4 * i + k);
                if (ch == '0' || ch == '1') {
                    c.bit |= at;
                    if (ch == '1')
                        c.one |= at;
                } else if (!is_ws((unsigned char)ch)) {
                    c.other |= at;
                }
            }
        }
    }
    return c;
}

// Per-CTA count of bit characters; the first other non-whitespace byte.
__global__ void __launch_bounds__(256)
    text_count_kernel(const unsigned char* __restrict__ text, unsigned long long len,
                      unsigned long long* __restrict__ counts,
                      unsigned long long* __restrict__ first_other) {
    const unsigned long long p0 =
        (unsigned long long)blockIdx.x * kChunk + (unsigned long long)threadIdx.x * kPerThread;
    uint32_t b[8];
    load32(text, len, p0, b);
    const Classes cl = classify(b);
    unsigned n = __popc(cl.bit);
    unsigned long long other = cl.other ? p0 + (__ffs(cl.other) - 1) : ~0ull;
    for (int o = 16; o > 0; o >>= 1) {
        n += __shfl_xor_sync(kFull, n, o);
        other = min(other, __shfl_xor_sync(kFull, other, o));
    }
    __shared__ unsigned s_n[8];
    __shared__ unsigned long long s_o[8];
    if ((threadIdx.x & 31) == 0) {
        s_n[threadIdx.x >> 5] = n;
        s_o[threadIdx.x >> 5] = other;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned t = 0;
        unsigned long long mo = ~0ull;
        for (int w = 0; w < 8; ++w) {
            t += s_n[w];
            mo = min(mo, s_o[w]);
        }
        counts[blockIdx.x] = t;
        if (mo != ~0ull)
            atomicMin(first_other, mo);
    }
}

// Exclusive scan of the per-CTA counts (one CTA of 1024 threads).
__global__ void __launch_bounds__(1024)
    scan_kernel(const unsigned long long* __restrict__ counts, long long n,
                unsigned long long* __restrict__ offsets, unsigned long long* __restrict__ total) {
    __shared__ unsigned long long wsum[32];
    __shared__ unsigned long long run;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0)
        run = 0;
    __syncthreads();
    for (long long c0 = 0; c0 < n; c0 += 1024) {
        const long long i = c0 + threadIdx.x;
        const unsigned long long v = i < n ? counts[i] : 0ull;
        unsigned long long incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long t = __shfl_up_sync(kFull, incl, o);
            if (lane >= o)
                incl += t;
        }
        if (lane == 31)
            wsum[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            unsigned long long ws = wsum[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long t = __shfl_up_sync(kFull, ws, o);
                if (lane >= o)
                    ws += t;
            }
            wsum[lane] = ws;
        }
        __syncthreads();
        const unsigned long long before = run + (warp ? wsum[warp - 1] : 0ull);
        if (i < n)
            offsets[i] = before + incl - v;
        __syncthreads();
        if (threadIdx.x == 0)
            run += wsum[31];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        *total = run;
}

// Bit character number i (in text order) is matrix bit i when i < nbits;
// bits are OR-ed into the zeroed padded rows.  Records the text position of
// bit character nbits - 1 (the end of the payload).
__global__ void __launch_bounds__(256)
    text_scatter_kernel(const unsigned char* __restrict__ text, unsigned long long len,
                        const unsigned long long* __restrict__ offsets, unsigned long long nbits,
                        unsigned long long cols, unsigned long long stride,
                        unsigned long long* __restrict__ words,
                        unsigned long long* __restrict__ last_pos) {
    __shared__ unsigned s_warp[8];
    const unsigned long long base = (unsigned long long)blockIdx.x * kChunk;
    const unsigned long long p0 = base + (unsigned long long)threadIdx.x * kPerThread;
    uint32_t mine[8];
    load32(text, len, p0, mine);
    const Classes cl = classify(mine);
    const unsigned n = __popc(cl.bit);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned incl = n;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned t = __shfl_up_sync(kFull, incl, o);
        if (lane >= o)
            incl += t;
    }
    if (lane == 31)
        s_warp[warp] = incl;
    __syncthreads();
    unsigned before = 0;
    for (int w = 0; w < warp; ++w)
        before += s_warp[w];
    const unsigned long long idx = offsets[blockIdx.x] + before + incl - n;
    if (n == 0 || idx >= nbits)
        return;
    // the '1' flags of the bit characters, compacted to n consecutive bits
    uint32_t packed = cl.one;
    if (cl.bit != 0xffffffffu) {
        packed = 0;
        int j = 0;
        for (uint32_t m = cl.bit; m; m &= m - 1, ++j)
            packed |= ((cl.one >> (__ffs(m) - 1)) & 1u) << j;
    }
    unsigned take = n;  // bit characters past the payload are not matrix bits
    if (nbits - idx < take) {
        take = (unsigned)(nbits - idx);
        // bit character take - 1 of this run ends the payload
        uint32_t m = cl.bit;
        for (unsigned j = 0; j + 1 < take; ++j)
            m &= m - 1;
        *last_pos = p0 + (__ffs(m) - 1);
    } else if (nbits - idx == take) {
        *last_pos = p0 + (31 - __clz(cl.bit));
    }
    // deposit bits idx .. idx + take - 1, splitting at row ends
    unsigned long long r = idx / cols, col = idx % cols;
    unsigned long long bits = packed;
    if (take < 32)
        bits &= (1ull << take) - 1;
    while (take) {
        const unsigned m = (unsigned)min((unsigned long long)take, cols - col);
        const unsigned long long part = m == 64 ? bits : bits & ((1ull << m) - 1);
        if (part) {
            unsigned long long* w = words + r * stride + (col >> 6);
            const unsigned sh = (unsigned)(col & 63);
            atomicOr(w, part << sh);
            if (sh + m > 64)
                atomicOr(w + 1, part >> (64 - sh));
        }
        bits >>= m;
        take -= m;
        col += m;
        if (col == cols) {
            col = 0;
            ++r;
        }
    }
}

// Output line r of the payload: cols '0'/'1' characters and '\n' at
// r * (cols + 1); CTAs stride over rows (y) and column chunks (x).
__global__ void text_format_kernel(const unsigned long long* __restrict__ words,
                                   unsigned long long stride, unsigned long long rows,
                                   unsigned long long cols, char* __restrict__ out) {
    for (unsigned long long r = blockIdx.y; r < rows; r += gridDim.y) {
        const unsigned long long* row = words + r * stride;
        char* line = out + r * (cols + 1);
        for (unsigned long long c = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
             c <= cols; c += (unsigned long long)gridDim.x * blockDim.x)
            line[c] = c == cols ? '\n' : (((row[c >> 6] >> (c & 63)) & 1ull) ? '1' : '0');
    }
}

// ---- host ------------------------------------------------------------------

bool host_ws(unsigned char c) {
    return c == ' ' || c == '\n' || c == '\r' || c == '\t' || c == '\f' || c == '\v';
}

// `in >> rows >> cols` for size_t: leading whitespace, an optional sign, at
// least one digit, no overflow.  *pos is left after the second number.
int parse_header(const char* text, size_t len, uint64_t* rows, uint64_t* cols, size_t* pos) {
    size_t p = 0;
    uint64_t v[2];
    for (int f = 0; f < 2; ++f) {
        while (p < len && host_ws((unsigned char)text[p]))
            ++p;
        bool neg = false;
        if (p < len && (text[p] == '+' || text[p] == '-'))
            neg = text[p++] == '-';
        if (p >= len || text[p] < '0' || text[p] > '9')
            return fail(BMM_ERUNTIME, "failed to read matrix text header");
        uint64_t x = 0;
        while (p < len && text[p] >= '0' && text[p] <= '9') {
            const uint64_t d = (uint64_t)(text[p++] - '0');
            if (x > (~0ull - d) / 10)
                return fail(BMM_ERUNTIME, "failed to read matrix text header");
            x = x * 10 + d;
        }
        v[f] = neg ? (~x + 1) : x;  // unsigned extraction wraps a negative value
    }
    *rows = v[0];
    *cols = v[1];
    *pos = p;
    return BMM_OK;
}

// The reference BitMatrix(rows, cols) size checks (src/core/bit_matrix.cpp:27-65).
int check_dims(uint64_t rows, uint64_t cols) {
    const uint64_t blocks = cols / 64 / 4 + ((cols / 64) % 4 != 0 || cols % 64 != 0 ? 1 : 0);
    if (blocks > ~0ull / 4)
        return fail(BMM_EMATRIX, "Matrix dimensions too large");
    const uint64_t stride = blocks * 4;
    if (stride && rows > ~0ull / stride)
        return fail(BMM_EMATRIX, "Matrix dimensions too large");
    if (rows * stride > ~0ull / 8)
        return fail(BMM_EMATRIX, "Matrix dimensions too large");
    return BMM_OK;
}

// SHA-256 (FIPS 180-4, section 6.2).
struct Sha256 {
    uint32_t h[8] = {0x6a09e667u, 0xbb67ae85u, 0x3c6ef372u, 0xa54ff53au,
                     0x510e527fu, 0x9b05688cu, 0x1f83d9abu, 0x5be0cd19u};
    unsigned char buf[64];
    size_t fill = 0;
    uint64_t bytes = 0;

    static uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

    void block(const unsigned char* p) {
        static const uint32_t K[64] = {
            0x428a2f98u, 0x71374491u, 0xb5c0fbcfu, 0xe9b5dba5u, 0x3956c25bu, 0x59f111f1u,
            0x923f82a4u, 0xab1c5ed5u, 0xd807aa98u, 0x12835b01u, 0x243185beu, 0x550c7dc3u,
            0x72be5d74u, 0x80deb1feu, 0x9bdc06a7u, 0xc19bf174u, 0xe49b69c1u, 0xefbe4786u,
            0x0fc19dc6u, 0x240ca1ccu, 0x2de92c6fu, 0x4a7484aau, 0x5cb0a9dcu, 0x76f988dau,
            0x983e5152u, 0xa831c66du, 0xb00327c8u, 0xbf597fc7u, 0xc6e00bf3u, 0xd5a79147u,
            0x06ca6351u, 0x14292967u, 0x27b70a85u, 0x2e1b2138u, 0x4d2c6dfcu, 0x53380d13u,
            0x650a7354u, 0x766a0abbu, 0x81c2c92eu, 0x92722c85u, 0xa2bfe8a1u, 0xa81a664bu,
            0xc24b8b70u, 0xc76c51a3u, 0xd192e819u, 0xd6990624u, 0xf40e3585u, 0x106aa070u,
            0x19a4c116u, 0x1e376c08u, 0x2748774cu, 0x34b0bcb5u, 0x391c0cb3u, 0x4ed8aa4au,
            0x5b9cca4fu, 0x682e6ff3u, 0x748f82eeu, 0x78a5636fu, 0x84c87814u, 0x8cc70208u,
            0x90befffau, 0xa4506cebu, 0xbef9a3f7u, 0xc67178f2u};
        uint32_t w[64];
        for (int i = 0; i < 16; ++i)
            w[i] = (uint32_t)p[4 * i] << 24 | (uint32_t)p[4 * i + 1] << 16 |
                   (uint32_t)p[4 * i + 2] << 8 | (uint32_t)p[4 * i + 3];
        for (int i = 16; i < 64; ++i) {
            const uint32_t s0 = rotr(w[i - 15], 7) ^ rotr(w[i - 15], 18) ^ (w[i - 15] >> 3);
            const uint32_t s1 = rotr(w[i - 2], 17) ^ rotr(w[i - 2], 19) ^ (w[i - 2] >> 10);
            w[i] = w[i - 16] + s0 + w[i - 7] + s1;
        }
        uint32_t a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], k = h[7];
        for (int i = 0; i < 64; ++i) {
            const uint32_t t1 = k + (rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25)) + ((e & f) ^ (~e & g)) +
                                K[i] + w[i];
            const uint32_t t2 = (rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22)) + ((a & b) ^ (a & c) ^ (b & c));
            k = g;
            g = f;
            f = e;
            e = d + t1;
            d = c;
            c = b;
            b = a;
            a = t1 + t2;
        }
        h[0] += a, h[1] += b, h[2] += c, h[3] += d, h[4] += e, h[5] += f, h[6] += g, h[7] += k;
    }
    void update(const unsigned char* p, size_t n) {
        bytes += n;
        while (n) {
            const size_t take = std::min(n, (size_t)64 - fill);
            std::memcpy(buf + fill, p, take);
            fill += take, p += take, n -= take;
            if (fill == 64) {
                block(buf);
                fill = 0;
            }
        }
    }
    void u64le(uint64_t v) {
        unsigned char b[8];
        for (int i = 0; i < 8; ++i)
            b[i] = (unsigned char)(v >> (8 * i));
        update(b, 8);
    }
    void hex(char* out) {
        const uint64_t bits = bytes * 8;
        const unsigned char one = 0x80, zero = 0;
        update(&one, 1);
        while (fill != 56)
            update(&zero, 1);
        unsigned char len[8];
        for (int i = 0; i < 8; ++i)
            len[i] = (unsigned char)(bits >> (56 - 8 * i));
        update(len, 8);
        static const char* digits = "0123456789abcdef";
        for (int i = 0; i < 8; ++i)
            for (int j = 0; j < 4; ++j) {
                const unsigned v = (h[i] >> (24 - 8 * j)) & 0xff;
                out[8 * i + 2 * j] = digits[v >> 4];
                out[8 * i + 2 * j + 1] = digits[v & 15];
            }
        out[64] = '\0';
    }
};

// The text payload (everything after the two header numbers) on the device
// into zeroed padded rows, then the reference's error checks.  Synchronises
// `s` to read the three positions back.
int parse_payload(Workspace* ws, cudaStream_t s, const unsigned char* d_text, size_t plen,
                  size_t rows, size_t cols, size_t stride, uint64_t* d_words) {
    const unsigned long long nbits = (unsigned long long)rows * cols;
    if (rows)
        BMM_CUDA_TRY(cudaMemsetAsync(d_words, 0, rows * stride * 8, s));
    if (plen == 0) {
        if (nbits)
            return fail(BMM_ERUNTIME, "failed to read matrix text payload");
        return BMM_OK;
    }
    const size_t nblk = (plen + kChunk - 1) / kChunk;
    void *d_counts = nullptr, *d_offsets = nullptr, *d_scal = nullptr;
    BMM_TRY(ws_buffer(ws, kSlotAux, nblk * 8, &d_counts));
    BMM_TRY(ws_buffer(ws, kSlotIdx, nblk * 8, &d_offsets));
    BMM_TRY(ws_buffer(ws, kSlotCounter, 3 * 8, &d_scal));
    unsigned long long* sc = (unsigned long long*)d_scal;  // first_other, last_pos, total
    BMM_CUDA_TRY(cudaMemsetAsync(sc, 0xff, 2 * 8, s));
    text_count_kernel<<<(unsigned)nblk, 256, 0, s>>>(d_text, plen, (unsigned long long*)d_counts,
                                                     sc);
    scan_kernel<<<1, 1024, 0, s>>>((const unsigned long long*)d_counts, (long long)nblk,
                                   (unsigned long long*)d_offsets, sc + 2);
    text_scatter_kernel<<<(unsigned)nblk, 256, 0, s>>>(
        d_text, plen, (const unsigned long long*)d_offsets, nbits,
        std::max<unsigned long long>(cols, 1), stride, (unsigned long long*)d_words, sc + 1);
    BMM_CUDA_TRY(cudaGetLastError());
    unsigned long long h[3];
    BMM_CUDA_TRY(cudaMemcpyAsync(h, sc, sizeof(h), cudaMemcpyDeviceToHost, s));
    BMM_CUDA_TRY(cudaStreamSynchronize(s));
    const unsigned long long first_other = h[0], last = h[1], total = h[2];
    const bool have_other = first_other != ~0ull;
    // an invalid character inside the payload comes first in the reference's
    // sequential read; then a short payload; then anything after it
    if (have_other && (total < nbits || (nbits && first_other < last)))
        return fail(BMM_ERUNTIME, "matrix text contains invalid character");
    if (total < nbits)
        return fail(BMM_ERUNTIME, "failed to read matrix text payload");
    if (total > nbits || have_other)
        return fail(BMM_ERUNTIME, "matrix text contains trailing data");
    return BMM_OK;
}

constexpr char kMagic[8] = {'B', 'M', 'M', 'P', 'Y', 'B', '1', '\0'};

struct File {
    FILE* f = nullptr;
    ~File() {
        if (f)
            std::fclose(f);
    }
};

int read_binary_header(File& fh, const char* path, uint64_t* rows, uint64_t* cols) {
    fh.f = std::fopen(path, "rb");
    if (!fh.f)
        return fail(BMM_ERUNTIME, "failed to open matrix binary file for reading");
    char magic[8];
    if (std::fread(magic, 1, 8, fh.f) != 8)
        return fail(BMM_ERUNTIME, "failed to read matrix binary header");
    if (std::memcmp(magic, kMagic, 8) != 0)
        return fail(BMM_ERUNTIME, "invalid matrix binary format");
    uint64_t v[2];
    for (int i = 0; i < 2; ++i)
        if (std::fread(&v[i], 8, 1, fh.f) != 1)
            return fail(BMM_ERUNTIME, "failed to read matrix binary data");
    BMM_TRY(check_dims(v[0], v[1]));
    *rows = v[0];
    *cols = v[1];
    return BMM_OK;
}

}  // namespace io
}  // namespace bmm

using namespace bmm;

extern "C" {

BMM_API int bmm_matrix_text_header(const char* text, size_t len, uint64_t* rows, uint64_t* cols) {
    clear_error();
    if ((!text && len) || !rows || !cols)
        return fail(BMM_EINVAL, "matrix text: null pointer");
    size_t pos = 0;
    BMM_TRY(io::parse_header(text, len, rows, cols, &pos));
    return io::check_dims(*rows, *cols);
}

BMM_API int bmm_matrix_from_text(const char* text, size_t len, uint64_t* words, size_t stride,
                                 size_t rows, size_t cols) {
    clear_error();
    uint64_t r = 0, c = 0;
    size_t pos = 0;
    if (!text && len)
        return fail(BMM_EINVAL, "matrix text: null pointer");
    BMM_TRY(io::parse_header(text, len, &r, &c, &pos));
    BMM_TRY(io::check_dims(r, c));
    if (r != rows || c != cols)
        return fail(BMM_EINVAL, "matrix text: rows/cols differ from the header");
    if (stride < (cols + 63) / 64 || (rows && !words))
        return fail(BMM_EINVAL, "matrix text: output buffer too small");
    if (rows && cols && rows > ~0ull / cols)
        return fail(BMM_EMATRIX, "Matrix dimensions too large");
    const size_t plen = len - pos;  // payload bytes after the header numbers
    if (rows)
        std::memset(words, 0, rows * stride * 8);
    if (plen == 0) {
        if (rows && cols)
            return fail(BMM_ERUNTIME, "failed to read matrix text payload");
        return BMM_OK;
    }
    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws)
        return st;
    void *d_text = nullptr, *d_words = nullptr;
    BMM_TRY(ws_buffer(ws, kSlotExtra1, plen, &d_text));
    BMM_TRY(ws_buffer(ws, kSlotRows, std::max<size_t>(rows * stride, 1) * 8, &d_words));
    BMM_CUDA_TRY(cudaMemcpyAsync(d_text, text + pos, plen, cudaMemcpyHostToDevice, ws->stream));
    BMM_TRY(io::parse_payload(ws, ws->stream, (const unsigned char*)d_text, plen, rows, cols,
                              stride, (uint64_t*)d_words));
    if (rows)
        BMM_CUDA_TRY(cudaMemcpy(words, d_words, rows * stride * 8, cudaMemcpyDeviceToHost));
    return BMM_OK;
}

BMM_API int bmm_matrix_from_text_dev(const char* payload, size_t len, uint64_t* words,
                                     size_t stride, size_t rows, size_t cols, void* stream) {
    clear_error();
    if ((!payload && len) || (rows && !words) || stride < (cols + 63) / 64)
        return fail(BMM_EINVAL, "matrix text: bad arguments");
    BMM_TRY(io::check_dims(rows, cols));
    if (rows && cols && rows > ~0ull / cols)
        return fail(BMM_EMATRIX, "Matrix dimensions too large");
    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws)
        return st;
    return io::parse_payload(ws, (cudaStream_t)stream, (const unsigned char*)payload, len, rows,
                             cols, stride, words);
}

BMM_API int bmm_matrix_text_size(size_t rows, size_t cols, size_t* len) {
    clear_error();
    if (!len)
        return fail(BMM_EINVAL, "matrix text: null pointer");
    const std::string head = std::to_string(rows) + ' ' + std::to_string(cols) + '\n';
    if (cols + 1 != 0 && rows > (~(size_t)0 - head.size()) / (cols + 1))
        return fail(BMM_EMATRIX, "Matrix dimensions too large");
    *len = head.size() + rows * (cols + 1);
    return BMM_OK;
}

BMM_API int bmm_matrix_to_text(const uint64_t* words, size_t stride, size_t rows, size_t cols,
                               char* out, size_t cap, size_t* len) {
    clear_error();
    size_t need = 0;
    BMM_TRY(bmm_matrix_text_size(rows, cols, &need));
    if (!out || cap < need || (rows && !words) || stride < (cols + 63) / 64)
        return fail(BMM_EINVAL, "matrix text: output buffer too small");
    const std::string head = std::to_string(rows) + ' ' + std::to_string(cols) + '\n';
    std::memcpy(out, head.data(), head.size());
    if (len)
        *len = need;
    const size_t body = need - head.size();
    if (body == 0)
        return BMM_OK;
    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws)
        return st;
    void *d_words = nullptr, *d_out = nullptr;
    BMM_TRY(ws_buffer(ws, kSlotRows, std::max<size_t>(rows * stride, 1) * 8, &d_words));
    BMM_TRY(ws_buffer(ws, kSlotExtra1, body, &d_out));
    BMM_CUDA_TRY(cudaMemcpyAsync(d_words, words, rows * stride * 8, cudaMemcpyHostToDevice,
                                 ws->stream));
    const unsigned bx = (unsigned)std::min<size_t>((cols + 1 + 255) / 256, 64);
    const unsigned by = (unsigned)std::min<size_t>(rows, 65535);
    io::text_format_kernel<<<dim3(bx, by), 256, 0, ws->stream>>>(
        (const unsigned long long*)d_words, stride, rows, cols, (char*)d_out);
    BMM_CUDA_TRY(cudaGetLastError());
    BMM_CUDA_TRY(cudaMemcpyAsync(out + head.size(), d_out, body, cudaMemcpyDeviceToHost,
                                 ws->stream));
    BMM_CUDA_TRY(cudaStreamSynchronize(ws->stream));
    return BMM_OK;
}

BMM_API int bmm_matrix_save_binary(const char* path, const uint64_t* words, size_t stride,
                                   size_t rows, size_t cols) {
    clear_error();
    if (!path || (rows && !words) || stride < (cols + 63) / 64)
        return fail(BMM_EINVAL, "matrix binary: bad arguments");
    io::File fh;
    fh.f = std::fopen(path, "wb");
    if (!fh.f)
        return fail(BMM_ERUNTIME, "failed to open matrix binary file for writing");
    const uint64_t dims[2] = {rows, cols};
    if (std::fwrite(io::kMagic, 1, 8, fh.f) != 8)
        return fail(BMM_ERUNTIME, "failed to write matrix binary header");
    if (std::fwrite(dims, 8, 2, fh.f) != 2)
        return fail(BMM_ERUNTIME, "failed to write matrix binary data");
    const size_t W = (cols + 63) / 64;
    for (size_t r = 0; r < rows && W; ++r)
        if (std::fwrite(words + r * stride, 8, W, fh.f) != W)
            return fail(BMM_ERUNTIME, "failed to write matrix binary payload");
    if (std::fflush(fh.f) != 0)
        return fail(BMM_ERUNTIME, "failed to write matrix binary payload");
    return BMM_OK;
}

BMM_API int bmm_matrix_binary_header(const char* path, uint64_t* rows, uint64_t* cols) {
    clear_error();
    if (!path || !rows || !cols)
        return fail(BMM_EINVAL, "matrix binary: null pointer");
    io::File fh;
    return io::read_binary_header(fh, path, rows, cols);
}

BMM_API int bmm_matrix_load_binary(const char* path, uint64_t* words, size_t stride, size_t rows,
                                   size_t cols) {
    clear_error();
    if (!path)
        return fail(BMM_EINVAL, "matrix binary: null path");
    io::File fh;
    uint64_t r = 0, c = 0;
    BMM_TRY(io::read_binary_header(fh, path, &r, &c));
    if (r != rows || c != cols || stride < (cols + 63) / 64 || (rows && !words))
        return fail(BMM_EINVAL, "matrix binary: output does not match the header");
    const size_t W = (cols + 63) / 64;
    for (size_t i = 0; i < rows; ++i) {
        if (W && std::fread(words + i * stride, 8, W, fh.f) != W)
            return fail(BMM_ERUNTIME, "failed to read matrix binary payload");
        std::memset(words + i * stride + W, 0, (stride - W) * 8);
    }
    return BMM_OK;
}

BMM_API int bmm_matrix_load_binary_dev(const char* path, uint64_t* d_words, size_t stride,
                                       size_t rows, size_t cols, void* stream) {
    clear_error();
    if (!path)
        return fail(BMM_EINVAL, "matrix binary: null path");
    io::File fh;
    uint64_t r = 0, c = 0;
    BMM_TRY(io::read_binary_header(fh, path, &r, &c));
    if (r != rows || c != cols || stride < (cols + 63) / 64 || (rows && !d_words))
        return fail(BMM_EINVAL, "matrix binary: output does not match the header");
    const size_t W = (cols + 63) / 64;
    if (rows == 0)
        return BMM_OK;
    int st = 0;
    Workspace* ws = workspace(&st);
    if (!ws)
        return st;
    cudaStream_t s = (cudaStream_t)stream;
    BMM_CUDA_TRY(cudaMemsetAsync(d_words, 0, rows * stride * 8, s));
    if (W == 0)
        return BMM_OK;
    // two pinned halves of a staging buffer: read the next rows while the
    // previous ones are copied, one strided 2-D copy per batch
    const size_t batch_rows = std::max<size_t>(1, std::min<size_t>(rows, (32u << 20) / (W * 8)));
    void* pin = nullptr;
    BMM_TRY(ws_pinned(ws, 2 * batch_rows * W * 8, &pin));
    cudaEvent_t done[2];
    BMM_CUDA_TRY(cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming));
    BMM_CUDA_TRY(cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming));
    int rc = BMM_OK;
    size_t half = 0;
    for (size_t r0 = 0; r0 < rows && rc == BMM_OK; r0 += batch_rows, half ^= 1) {
        const size_t n = std::min(batch_rows, rows - r0);
        uint64_t* stage = (uint64_t*)pin + half * batch_rows * W;
        if (r0 >= 2 * batch_rows && cudaEventSynchronize(done[half]) != cudaSuccess) {
            rc = fail(BMM_ECUDA, "matrix binary: staging copy failed");
            break;
        }
        if (std::fread(stage, 8, n * W, fh.f) != n * W) {
            rc = fail(BMM_ERUNTIME, "failed to read matrix binary payload");
            break;
        }
        if (cudaMemcpy2DAsync(d_words + r0 * stride, stride * 8, stage, W * 8, W * 8, n,
                              cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaEventRecord(done[half], s) != cudaSuccess)
            rc = fail(BMM_ECUDA, "matrix binary: staging copy failed");
    }
    // the staging buffer is reused by later calls: wait for the copies in flight
    cudaEventSynchronize(done[0]);
    cudaEventSynchronize(done[1]);
    cudaEventDestroy(done[0]);
    cudaEventDestroy(done[1]);
    return rc;
}

BMM_API int bmm_matrix_hash(const uint64_t* words, size_t stride, size_t rows, size_t cols,
                            char* hex) {
    clear_error();
    if (!hex || (rows && cols && !words) || stride < (cols + 63) / 64)
        return fail(BMM_EINVAL, "matrix hash: bad arguments");
    io::Sha256 h;
    h.u64le(rows);
    h.u64le(cols);
    const size_t W = (cols + 63) / 64;
    const uint64_t tail = (cols & 63) ? ((1ull << (cols & 63)) - 1) : ~0ull;
    if (W)
        for (size_t r = 0; r < rows; ++r)
            for (size_t w = 0; w < W; ++w)
                h.u64le(w + 1 == W ? words[r * stride + w] & tail : words[r * stride + w]);
    h.hex(hex);
    return BMM_OK;
}

}  // extern "C"
