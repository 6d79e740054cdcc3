// codec_kernels.cuh -- the lsCOMP block codec (uint16 and uint32 stacks) as
// sm_100a kernels.
//
// One launch encodes (or decodes) a whole X x Y x Z stack (z fastest) in a
// single pass over HBM:
//
//   * The stack is cut into *tiles* of consecutive 8x8 blocks (block index
//     order = the stream's order, lsCOMP/src/cuLSZ_kernel.cu:868-872).  A tile
//     is either G whole block-rows (when a block-row has at most
//     Elem<T>::kTileBlocks blocks; the tile's input is then one contiguous
//     byte range) or one chunk of a single block-row (8 row segments).
//   * Persistent CTAs claim tiles in increasing order from a ticket counter,
//     so every tile a CTA waits on in the scan belongs to a resident CTA.
//   * Encoder (one CTA per SM, warp-specialised): a producer warp fetches
//     each tile's input once with 1-D TMA bulk copies into a 3-deep ring;
//     two groups of compute warps (8, 7 or 13 warps each, the shape chosen
//     per call) take alternate tiles, derive every block's statistics,
//     pooling, bin choice and rate, publish the tile's payload size and
//     pack the bit planes into a 3-deep payload ring; a writer warp runs
//     the decoupled look-back for the tile's stream offset and copies the
//     packed payload to the stream.  Only the writer waits on other CTAs,
//     and the compute warps run up to three tiles ahead of it.  Batch
//     launches do the same over the tiles of many stacks.
//   * Decoder: a small kernel turns the header bytes into per-tile stream
//     offsets; the decode kernel then handles every tile independently
//     (plane words gathered per block, values scattered to the rows), for
//     one stack or, in batch launches, for the tiles of many.
//
// Thread layout inside a warp ("unit" = 8 consecutive blocks of a tile):
// lane = j + 8 r, j = block within the unit, r = 0..3; the lane owns rows r
// and r+4 of block j (8 values each, held as a Row: 4 words of two uint16, or
// 8 words of one uint32).  The 4 lanes of a block sit 8 lanes apart, so block
// reductions and the 4x4 byte transposes that assemble plane words are two
// xor-shuffles (8, 16).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "bitplane.h"
#include "device_prims.cuh"

// Tuning switches (compile-time; the defaults are the measured best on B200):
//   LSC_LOOKBACK      0: 32-wide look-back to the nearest inclusive prefix,
//                     1: 256-wide look-back bounded by the writer's previous tile
//   LSC_DEC_CTAS      decoder CTAs per SM the register budget is sized for
//   LSC_ENC_GROUPS    compute groups per encoder CTA (tiles in flight)
//   LSC_ENC_WPG       warps per compute group
#ifndef LSC_LOOKBACK
#define LSC_LOOKBACK 0
#endif
#ifndef LSC_DEC_CTAS
#define LSC_DEC_CTAS 6  // decoder CTAs per SM the register budget is sized for (shared memory allows 6)
#endif
#ifndef LSC_ENC_GROUPS
#define LSC_ENC_GROUPS 2  // independent compute groups per encoder CTA
#endif
#ifndef LSC_ENC_WPG
#define LSC_ENC_WPG 8     // warps per compute group
#endif

namespace lsc {

constexpr int kThreads = 256;                  // 8 warps per CTA
constexpr int kWarps = kThreads / 32;
constexpr int kMaxTileBlocks = 256;            // smem tables are sized for this
constexpr int kChunkPitch = 4096 + 32;         // bytes per row segment (chunk tiles)
constexpr int kStageBytes = 33280;             // >= one tile's input + alignment slack

// bins layouts (template parameter)
constexpr int BINS_EQUAL = 0;   // all four bins equal: bin choice is always 3
constexpr int BINS_MONO = 1;    // x <= y <= z <= w (what the CLI accepts)
constexpr int BINS_GENERAL = 2; // anything else the host API allows
constexpr int BINS_IDENT = 3;   // all four bins 1 (the lossless mode): no quantisation

// Per element type: words per 8-value row, plane byte groups, largest rate
// the 5-bit header field carries, and blocks per tile (4 KB of input per
// row segment for both types).
template <typename T> struct Elem;
template <> struct Elem<uint16_t> {
    static constexpr int kWords = 4;
    static constexpr int kGroups = 2;
    static constexpr uint32_t kMaxRate = 16;
    static constexpr int kTileBlocks = 256;
};
template <> struct Elem<uint32_t> {
    static constexpr int kWords = 8;
    static constexpr int kGroups = 4;
    static constexpr uint32_t kMaxRate = 31;
    static constexpr int kTileBlocks = 128;
};

template <typename T> struct Row { uint32_t w[Elem<T>::kWords]; };

struct Geom {
    uint32_t X, Y, Z;
    uint32_t byb, bzb;         // ceil(Y/8), ceil(Z/8)
    unsigned long long nb;     // blocks
    unsigned long long R;      // roundup4(nb): payload base
    unsigned long long N;      // elements
    unsigned long long nrows_b;// block-rows = X * byb
    unsigned long long ntiles;
    uint32_t chunked;          // 0: tiles of G whole block-rows, 1: chunks of a block-row
    uint32_t G;                // block-rows per tile (whole-row tiles)
    uint32_t nc, W;            // chunks per block-row, chunk width (chunked tiles)
    uint32_t inv_bzb;          // ceil(65536 / bzb), exact b / bzb for b < 256 (whole-row tiles)
    uint32_t vec;              // batch launches: widest row access of this stack (16, 4 or 2 bytes)
    unsigned long long byb_magic, nc_magic;  // ceil(2^64 / d) of byb and nc (0 for d = 1)
};

struct Codec {
    uint32_t bins[4];
    uint32_t magic[4];             // uint16: ceil(2^32 / bin) for bin >= 2, 0 for bin == 1
    unsigned long long magic64[4]; // uint32: ceil(2^64 / bin) for bin >= 2, 0 for bin == 1
    uint32_t binc[4];              // bins for the comparisons (uint16: clamped to 65536)
    uint32_t qsm[4];               // uint16 values below 128: lsc_small_quant_magic(bin)
    int pool_min;                  // a block pools iff zero count >= pool_min (65: never)
};

template <typename T>
struct EncArgs {
    Geom g;
    Codec c;
    const T *in;
    uint8_t *out;
    unsigned long long cap;
    LaunchCtl *ctl;
    unsigned long long *state;
    uint32_t epoch;
    unsigned long long *sizes_out;  // optional device copy of {stream_len, payload}
    // batch launches: the stacks, the stack of every tile (tiles of all
    // stacks numbered in stack order) and their total; g, in, out, cap and
    // sizes_out above are unused then
    const struct BatchStack *stacks;
    const uint32_t *tile_stack;
    unsigned long long ntiles_all;
};

// One stack of a batch launch (device memory).  Its tiles are the tiles
// tile0 .. tile0 + g.ntiles - 1 of the batch; sizes receives
// {stream_len, payload} when its last tile is written.  Stacks of one launch
// may have different bins and pooling thresholds: the launch is instantiated
// for a bins layout that covers all of them.
struct BatchStack {
    Geom g;
    Codec c;  // the stack's bins and pooling threshold
    const void *in;
    uint8_t *out;
    unsigned long long cap;
    unsigned long long tile0;
    unsigned long long *sizes;
};

constexpr unsigned long long kMarker = ~0ull;  // ring entry that ends a CTA's tiles

template <typename T>
struct DecArgs {
    Geom g;
    Codec c;
    const uint8_t *in;
    T *out;
    unsigned long long cap;  // readable stream bytes
    LaunchCtl *ctl;
    unsigned long long *state;    // look-back state of the offsets kernel (per segment)
    unsigned long long *tile_off; // per-tile payload offsets
    uint32_t epoch;
    // batch launches: the stacks (in = stream, out = decoded values, cap =
    // readable stream bytes, tile0 = first tile over the batch), their
    // count and the first segment of each (nstacks + 1 entries); stack s's
    // tile offsets are tile_off[tile0 + s ...] (ntiles + 1 of them)
    const struct BatchStack *stacks;
    uint32_t nstacks;
    const unsigned long long *seg0;
    const uint32_t *tile_stack;  // the stack of every tile over the batch
};

// ---------------------------------------------------------------- geometry
struct TileInfo {
    unsigned long long k0;   // first block index
    unsigned long long rho0; // first block-row
    uint32_t nblk;           // blocks in the tile
    uint32_t nbr;            // block-rows (whole-row tiles)
    uint32_t c0;             // first block column (chunked tiles)
};

// n / d from m = ceil(2^64 / d) (m = 0 for d = 1): the high product is
// exact while n d < 2^64 and at most one too large past that
__device__ __forceinline__ unsigned long long udiv_magic(unsigned long long n, uint32_t d, unsigned long long m)
{
    if (m == 0) return n;
    unsigned long long q = __umul64hi(n, m);
    if (q * d > n) q--;
    return q;
}

__device__ __forceinline__ TileInfo tile_info(const Geom &g, unsigned long long t)
{
    TileInfo ti;
    if (!g.chunked) {
        ti.rho0 = t * g.G;
        unsigned long long left = g.nrows_b - ti.rho0;
        ti.nbr = (uint32_t)(left < g.G ? left : g.G);
        ti.nblk = ti.nbr * g.bzb;
        ti.k0 = ti.rho0 * g.bzb;
        ti.c0 = 0;
    } else {
        ti.rho0 = udiv_magic(t, g.nc, g.nc_magic);
        uint32_t ci = (uint32_t)(t - ti.rho0 * g.nc);
        ti.c0 = ci * g.W;
        uint32_t c1 = ti.c0 + g.W;
        if (c1 > g.bzb) c1 = g.bzb;
        ti.nblk = c1 - ti.c0;
        ti.nbr = 1;
        ti.k0 = ti.rho0 * g.bzb + ti.c0;
    }
    return ti;
}

// first image row (frame-major global row index) and row count of a block-row
__device__ __forceinline__ unsigned long long brow_start(const Geom &g, unsigned long long rho, uint32_t &nrows)
{
    unsigned long long x = udiv_magic(rho, g.byb, g.byb_magic);
    uint32_t by = (uint32_t)(rho - x * g.byb);
    uint32_t r = g.Y - 8u * by;
    nrows = r < 8u ? r : 8u;
    return x * g.Y + 8ull * by;
}

// ---------------------------------------------------------------- row I/O
// Load the 8 values at p (alignment VEC bytes).
template <int VEC>
__device__ __forceinline__ void load8(const uint8_t *p, Row<uint16_t> &v)
{
    if (VEC == 16) {
        uint4 q = *reinterpret_cast<const uint4 *>(p);
        v.w[0] = q.x; v.w[1] = q.y; v.w[2] = q.z; v.w[3] = q.w;
    } else if (VEC == 4) {
        const uint32_t *q = reinterpret_cast<const uint32_t *>(p);
        v.w[0] = q[0]; v.w[1] = q[1]; v.w[2] = q[2]; v.w[3] = q[3];
    } else {
        const uint16_t *h = reinterpret_cast<const uint16_t *>(p);
#pragma unroll
        for (int i = 0; i < 4; i++) v.w[i] = (uint32_t)h[2 * i] | ((uint32_t)h[2 * i + 1] << 16);
    }
}

template <int VEC>
__device__ __forceinline__ void load8(const uint8_t *p, Row<uint32_t> &v)
{
    if (VEC == 16) {
        uint4 a = reinterpret_cast<const uint4 *>(p)[0], b = reinterpret_cast<const uint4 *>(p)[1];
        v.w[0] = a.x; v.w[1] = a.y; v.w[2] = a.z; v.w[3] = a.w;
        v.w[4] = b.x; v.w[5] = b.y; v.w[6] = b.z; v.w[7] = b.w;
    } else {
        const uint32_t *q = reinterpret_cast<const uint32_t *>(p);
#pragma unroll
        for (int i = 0; i < 8; i++) v.w[i] = q[i];
    }
}

// The first ncols (1..8) values at p (global memory), the rest 0; nothing
// past them is read.  Full rows are read VEC bytes at a time.
template <typename T, int VEC = sizeof(T)>
__device__ __forceinline__ void load_cols(const T *p, uint32_t ncols, Row<T> &v)
{
    if (ncols >= 8u) {
        load8<VEC>(reinterpret_cast<const uint8_t *>(p), v);
        return;
    }
#pragma unroll
    for (int i = 0; i < Elem<T>::kWords; i++) v.w[i] = 0;
#pragma unroll
    for (uint32_t i = 0; i < 8u; i++) {
        if (i >= ncols) break;
        if constexpr (sizeof(T) == 2) v.w[i >> 1] |= (uint32_t)p[i] << (16u * (i & 1u));
        else v.w[i] = p[i];
    }
}

// keep only the first ncols (1..8) values
__device__ __forceinline__ void mask_cols(Row<uint16_t> &v, uint32_t ncols)
{
#pragma unroll
    for (int i = 0; i < 4; i++) {
        uint32_t keep = ncols >= 2u * i + 2u ? 0xffffffffu : (ncols == 2u * i + 1u ? 0x0000ffffu : 0u);
        v.w[i] &= keep;
    }
}

__device__ __forceinline__ void mask_cols(Row<uint32_t> &v, uint32_t ncols)
{
#pragma unroll
    for (int i = 0; i < 8; i++)
        if ((uint32_t)i >= ncols) v.w[i] = 0;
}

template <int VEC>
__device__ __forceinline__ void store8(uint16_t *p, const Row<uint16_t> &v, uint32_t ncols)
{
    if (ncols >= 8u) {
        if (VEC == 16) {
            *reinterpret_cast<uint4 *>(p) = make_uint4(v.w[0], v.w[1], v.w[2], v.w[3]);
            return;
        } else if (VEC == 4) {
            uint32_t *q = reinterpret_cast<uint32_t *>(p);
            q[0] = v.w[0]; q[1] = v.w[1]; q[2] = v.w[2]; q[3] = v.w[3];
            return;
        }
    }
#pragma unroll
    for (int i = 0; i < 8; i++)
        if ((uint32_t)i < ncols) p[i] = (uint16_t)(v.w[i >> 1] >> (16 * (i & 1)));
}

template <int VEC>
__device__ __forceinline__ void store8(uint32_t *p, const Row<uint32_t> &v, uint32_t ncols)
{
    if (ncols >= 8u && VEC == 16) {
        reinterpret_cast<uint4 *>(p)[0] = make_uint4(v.w[0], v.w[1], v.w[2], v.w[3]);
        reinterpret_cast<uint4 *>(p)[1] = make_uint4(v.w[4], v.w[5], v.w[6], v.w[7]);
        return;
    }
#pragma unroll
    for (int i = 0; i < 8; i++)
        if ((uint32_t)i < ncols) p[i] = v.w[i];
}

// ---------------------------------------------------------------- arithmetic
__device__ __forceinline__ uint32_t zero_halves(uint32_t w)
{
    // count of zero 16-bit halves in w (0..2)
    uint32_t t = ((w & 0x7fff7fffu) + 0x7fff7fffu) | w;
    return 2u - __popc(t & 0x80008000u);
}

__device__ __forceinline__ uint32_t zeros(const Row<uint16_t> &v)
{
    return zero_halves(v.w[0]) + zero_halves(v.w[1]) + zero_halves(v.w[2]) + zero_halves(v.w[3]);
}

__device__ __forceinline__ uint32_t zeros(const Row<uint32_t> &v)
{
    uint32_t z = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) z += v.w[i] == 0u;
    return z;
}

// min over the row of (value - b0) mod 2^32
__device__ __forceinline__ uint32_t min_from(const Row<uint16_t> &v, uint32_t b0, uint32_t mn)
{
#pragma unroll
    for (int i = 0; i < 4; i++) {
        mn = min(mn, (v.w[i] & 0xffffu) - b0);
        mn = min(mn, (v.w[i] >> 16) - b0);
    }
    return mn;
}

__device__ __forceinline__ uint32_t min_from(const Row<uint32_t> &v, uint32_t b0, uint32_t mn)
{
#pragma unroll
    for (int i = 0; i < 8; i++) mn = min(mn, v.w[i] - b0);
    return mn;
}

__device__ __forceinline__ uint32_t value_at(const Row<uint16_t> &v, int i)
{
    return (v.w[i >> 1] >> (16 * (i & 1))) & 0xffffu;
}

__device__ __forceinline__ uint32_t value_at(const Row<uint32_t> &v, int i) { return v.w[i]; }

// four 8-bit counters of (value < binc[k])
template <typename T>
__device__ __forceinline__ uint32_t bin_counts(const Row<T> &v, const uint32_t *binc)
{
    uint32_t cnt = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        uint32_t x = value_at(v, i);
        cnt += (uint32_t)(x < binc[0]) | ((uint32_t)(x < binc[1]) << 8) | ((uint32_t)(x < binc[2]) << 16) |
               ((uint32_t)(x < binc[3]) << 24);
    }
    return cnt;
}

// quantise every value of the row by the chosen bin
__device__ __forceinline__ uint32_t quant2(uint32_t w, uint32_t m)
{
    if (m == 0u) return w;
    uint32_t lo = __umulhi(w & 0xffffu, m);
    uint32_t hi = __umulhi(w >> 16, m);
    return lo | (hi << 16);
}

__device__ __forceinline__ void quant(Row<uint16_t> &v, const Codec &c, uint32_t choice)
{
    const uint32_t m = c.magic[choice];
#pragma unroll
    for (int i = 0; i < 4; i++) v.w[i] = quant2(v.w[i], m);
}

__device__ __forceinline__ void quant(Row<uint32_t> &v, const Codec &c, uint32_t choice)
{
    const unsigned long long m = c.magic64[choice];
    if (m == 0ull) return;
#pragma unroll
    for (int i = 0; i < 8; i++) v.w[i] = (uint32_t)__umul64hi((unsigned long long)v.w[i], m);
}

// pooled values of rows a and b: floor((v[2p] + v[2p+1]) / 2) with the sum
// in 32-bit unsigned arithmetic (lsCOMP/src/cuLSZ_kernel.cu:914,1109); the 4
// of row a then the 4 of row b, as one Row
__device__ __forceinline__ Row<uint16_t> pool_rows(const Row<uint16_t> &a, const Row<uint16_t> &b)
{
    // x = the first values of two pairs, y = the second ones, in 16-bit
    // halves; floor((x + y) / 2) = (x & y) + ((x ^ y) >> 1) per half, which
    // stays below 2^16 and carries nothing into the other half
    Row<uint16_t> p;
#pragma unroll
    for (int i = 0; i < 2; i++) {
        const Row<uint16_t> &s = i ? b : a;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const uint32_t x = __byte_perm(s.w[2 * h], s.w[2 * h + 1], 0x5410u);
            const uint32_t y = __byte_perm(s.w[2 * h], s.w[2 * h + 1], 0x7632u);
            p.w[2 * i + h] = (x & y) + (((x ^ y) >> 1) & 0x7fff7fffu);
        }
    }
    return p;
}

__device__ __forceinline__ Row<uint32_t> pool_rows(const Row<uint32_t> &a, const Row<uint32_t> &b)
{
    Row<uint32_t> p;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        p.w[i] = (a.w[2 * i] + a.w[2 * i + 1]) >> 1;  // the sum wraps, as in the reference
        p.w[4 + i] = (b.w[2 * i] + b.w[2 * i + 1]) >> 1;
    }
    return p;
}

__device__ __forceinline__ uint32_t or_all(const Row<uint16_t> &v)
{
    uint32_t o = v.w[0] | v.w[1] | v.w[2] | v.w[3];
    return (o & 0xffffu) | (o >> 16);
}

__device__ __forceinline__ uint32_t or_all(const Row<uint32_t> &v)
{
    uint32_t o = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) o |= v.w[i];
    return o;
}

__device__ __forceinline__ uint32_t bitlen(uint32_t v) { return 32u - __clz(v); }

// largest value of the row (16-bit halves compared pairwise with max.u16x2)
__device__ __forceinline__ uint32_t max2u16(uint32_t a, uint32_t b)
{
    uint32_t d;
    asm("max.u16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}

__device__ __forceinline__ uint32_t max_all(const Row<uint16_t> &v)
{
    const uint32_t m = max2u16(max2u16(v.w[0], v.w[1]), max2u16(v.w[2], v.w[3]));
    return max(m & 0xffffu, m >> 16);
}

__device__ __forceinline__ uint32_t max_all(const Row<uint32_t> &v)
{
    uint32_t m = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) m = max(m, v.w[i]);
    return m;
}

__device__ __forceinline__ uint32_t min2u16(uint32_t a, uint32_t b)
{
    uint32_t d;
    asm("min.u16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}

// per 16-bit half: (w + NB) mod 2^16 (no carry between the halves); with NB
// = (2^16 - b0) mod 2^16 in both halves this is (v - b0) mod 2^16
__device__ __forceinline__ uint32_t add16x2(uint32_t w, uint32_t NB)
{
    uint32_t d;
    asm("add.u16x2 %0, %1, %2;" : "=r"(d) : "r"(w), "r"(NB));
    return d;
}

// per 16-bit half: min over the row of (v - b0) mod 2^16 (NB = -b0 mod 2^16
// in both halves)
__device__ __forceinline__ uint32_t min16_from(const Row<uint16_t> &v, uint32_t NB, uint32_t acc)
{
#pragma unroll
    for (int i = 0; i < 4; i++) acc = min2u16(acc, add16x2(v.w[i], NB));
    return acc;
}

// per 16-bit half: count of nonzero values of the row, added to acc
__device__ __forceinline__ uint32_t nonzero16(const Row<uint16_t> &v, uint32_t acc)
{
#pragma unroll
    for (int i = 0; i < 4; i++) acc += min2u16(v.w[i], 0x00010001u);
    return acc;
}

// one value quantised by the chosen bin
__device__ __forceinline__ uint32_t quant1(uint32_t v, const Codec &c, uint32_t choice, bool wide)
{
    if (wide) {
        const unsigned long long m = c.magic64[choice];
        return m ? (uint32_t)__umul64hi((unsigned long long)v, m) : v;
    }
    const uint32_t m = c.magic[choice];
    return m ? __umulhi(v, m) : v;
}

// plane bytes of byte group g (planes 8g..8g+7) of one row: on return lo holds
// planes 8g+{0,1,2,3} and hi planes 8g+{4,5,6,7}, one byte per plane
__device__ __forceinline__ void row_planes(const Row<uint16_t> &v, uint32_t g, uint32_t &lo, uint32_t &hi)
{
    lsc_row_planes(v.w[0], v.w[1], v.w[2], v.w[3], (int)g, lo, hi);
}

__device__ __forceinline__ void row_planes(const Row<uint32_t> &v, uint32_t g, uint32_t &lo, uint32_t &hi)
{
    const uint32_t s2 = g | ((g + 4u) << 4);  // byte g of the first, byte g of the second word
    lo = __byte_perm(__byte_perm(v.w[7], v.w[6], s2), __byte_perm(v.w[5], v.w[4], s2), 0x5410u);
    hi = __byte_perm(__byte_perm(v.w[3], v.w[2], s2), __byte_perm(v.w[1], v.w[0], s2), 0x5410u);
    lsc_transpose8x8(lo, hi);
}

// inverse of row_planes over all groups: P[g][0] = lo, P[g][1] = hi.
// Groups at or above wrate (the largest rate in the unit) are zero and
// need no transpose.
__device__ __forceinline__ void row_values(uint32_t P[][2], Row<uint16_t> &v, uint32_t wrate)
{
    if (wrate > 8u) {
        lsc_row_values(P[0][0], P[0][1], P[1][0], P[1][1], v.w[0], v.w[1], v.w[2], v.w[3]);
    } else {
        uint32_t lo = P[0][0], hi = P[0][1];
        lsc_transpose8x8(lo, hi);  // low value bytes: lo = q7 q6 q5 q4, hi = q3 q2 q1 q0
        // the selectors of lsc_row_values with zero high value bytes
        v.w[3] = __byte_perm(lo, 0u, 0x4051u);
        v.w[2] = __byte_perm(lo, 0u, 0x6273u);
        v.w[1] = __byte_perm(hi, 0u, 0x4051u);
        v.w[0] = __byte_perm(hi, 0u, 0x6273u);
    }
}

__device__ __forceinline__ void row_values(uint32_t P[][2], Row<uint32_t> &v, uint32_t wrate)
{
#pragma unroll
    for (int g = 0; g < 4; g++)
        if (wrate > 8u * g) lsc_transpose8x8(P[g][0], P[g][1]);  // byte g of v7..v4 / v3..v0
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const uint32_t s = (uint32_t)k | ((uint32_t)(k + 4) << 4);
        v.w[7 - k] = __byte_perm(__byte_perm(P[0][0], P[1][0], s), __byte_perm(P[2][0], P[3][0], s), 0x5410u);
        v.w[3 - k] = __byte_perm(__byte_perm(P[0][1], P[1][1], s), __byte_perm(P[2][1], P[3][1], s), 0x5410u);
    }
}

// both 16-bit halves times bin, each product kept mod 2^16 as the
// reference's uint16 store keeps it: the low half of w * bin is the first
// product, the high half of (w & 0xffff0000) * bin the second
__device__ __forceinline__ uint32_t mul16x2(uint32_t w, uint32_t bin)
{
    return __byte_perm(w * bin, (w & 0xffff0000u) * bin, 0x7610u);
}

// both halves times bin when every product is known to stay below 2^16
// (pair: the quantised values are below 2^rate and bin <= 2^16 >> rate): one
// multiply, since the low product then carries nothing into the high half
__device__ __forceinline__ uint32_t mul16x2_any(uint32_t w, uint32_t bin, bool pair)
{
    return pair ? w * bin : mul16x2(w, bin);
}

__device__ __forceinline__ void dequant(Row<uint16_t> &v, uint32_t bin, bool pair)
{
    if (bin == 1u) return;
#pragma unroll
    for (int i = 0; i < 4; i++) v.w[i] = mul16x2_any(v.w[i], bin, pair);
}

__device__ __forceinline__ void dequant(Row<uint32_t> &v, uint32_t bin, bool)
{
#pragma unroll
    for (int i = 0; i < 8; i++) v.w[i] *= bin;
}

// one output row from 4 pooled quantised values (the first half of q, or
// the second): each value de-quantised and repeated over its two columns
__device__ __forceinline__ Row<uint16_t> unpool_row(const Row<uint16_t> &q, bool second, uint32_t bin, bool pair)
{
    Row<uint16_t> v;
    const uint32_t a = mul16x2_any(q.w[second ? 2 : 0], bin, pair), b = mul16x2_any(q.w[second ? 3 : 1], bin, pair);
    v.w[0] = __byte_perm(a, 0u, 0x1010u);  // first value in both halves
    v.w[1] = __byte_perm(a, 0u, 0x3232u);  // second value in both halves
    v.w[2] = __byte_perm(b, 0u, 0x1010u);
    v.w[3] = __byte_perm(b, 0u, 0x3232u);
    return v;
}

__device__ __forceinline__ Row<uint32_t> unpool_row(const Row<uint32_t> &q, bool second, uint32_t bin, bool)
{
    Row<uint32_t> v;
#pragma unroll
    for (int i = 0; i < 4; i++) v.w[2 * i] = v.w[2 * i + 1] = q.w[(second ? 4 : 0) + i] * bin;
    return v;
}

// 4x4 byte transpose across the lanes j, j+8, j+16, j+24 (r = lane >> 3):
// lane r ends with byte c = byte r of lane c's input.  The per-lane byte
// selectors are fixed for a thread and computed once.
struct XSel {
    uint32_t a, b;
};

__device__ __forceinline__ XSel xsel(uint32_t r)
{
    XSel s;
    s.a = r < 2u ? LSC_XP_A_LOW : LSC_XP_A_HIGH;
    s.b = (r & 1u) ? LSC_XP_B_ODD : LSC_XP_B_EVEN;
    return s;
}

__device__ __forceinline__ uint32_t xpose4(uint32_t x, const XSel &s)
{
    const uint32_t z = __byte_perm(x, __shfl_xor_sync(0xffffffffu, x, 16), s.a);
    return __byte_perm(z, __shfl_xor_sync(0xffffffffu, z, 8), s.b);
}

// ---------------------------------------------------------------- shared state
// Encoder CTA: GRP x WPG compute warps in independent groups, one producer
// warp (tile claims and TMA loads) and kWriters writer warps (look-back and
// write-out), one CTA per SM.  With groups of up to 8 warps there is one
// writer per group (writer w takes group w's tiles: two look-backs and two
// copy-outs in flight per SM); groups of 13 warps keep a single writer,
// whose 896 threads already use the register file at 72 registers each.
template <int GRP, int WPG> struct EncShape {
    static constexpr int kCompute = GRP * WPG;
    static constexpr int kWriters = WPG > 8 ? 1 : GRP;
    static constexpr int kThreads = (kCompute + 1 + kWriters) * 32;
    static constexpr int kProducerWarp = kCompute;
    static constexpr int kWriterWarp0 = kCompute + 1;
};
constexpr int kInStages = 3;                  // input ring (TMA destination)
constexpr int kStStages = 3;                  // packed-payload ring (write-out source)
constexpr int kStagingBytes = 32896;          // >= one tile's worst-case payload (32768)
constexpr uint32_t kComputeBarrier = 1;       // first named barrier of the compute groups
constexpr int kMaxGroups = 2;

struct EncSmem {
    alignas(128) uint8_t in[kInStages][kStageBytes];
    alignas(128) uint8_t st[kStStages][kStagingBytes];
    uint64_t in_full[kInStages];       // producer -> compute: input of entries k = s mod 2 kInStages landed
    uint64_t in_empty[kInStages];      // compute -> producer: input slot read
    // payload packed (compute -> writer) and written out (writer -> compute)
    // for ring entry k, one barrier per k mod 2 kStStages: the two writers
    // take alternate entries and run independently, so a wait on one
    // barrier per slot could pass on the phase of the entry two uses back
    // (see st_full_bar)
    uint64_t st_full[2 * kStStages];
    uint64_t st_empty[2 * kStStages];
    unsigned long long in_tile[kInStages];
    uint32_t in_mis[kInStages][8];     // byte misalignment of each range start (mod 16)
    unsigned long long st_tile[kStStages];
    uint32_t st_agg[kStStages];
    // per input slot: whole-row tiles: element offset of block-row g from the
    // tile start and its row count (chunked tiles: rows in [0]); filled by the
    // producer warp with the load
    uint32_t br_rel[kInStages][kMaxTileBlocks];
    uint8_t br_rows[kInStages][kMaxTileBlocks];
    uint8_t hdr[kMaxGroups][kMaxTileBlocks];   // per compute group: header byte per block
    uint32_t off[kMaxGroups][kMaxTileBlocks];  // payload offset of each block inside the tile
    uint32_t agg[kMaxGroups];
    uint32_t issued;                           // input-ring entries the producer filled
    // input landed, entries k = kInStages + s mod 2 kInStages.  With one
    // barrier per entry mod 2 kInStages a group waiting for entry k cannot
    // pass on the still-pending phase of entry k - kInStages (the other
    // group's tile in the same slot, whose load may land after the group's
    // previous one): the phase before entry k's belongs to the group's own
    // entry k - 2 kInStages, which it has already consumed.
    uint64_t in_full2[kInStages];
    // batch launches: the stack of each input slot and of each payload slot
    Geom in_geom[kInStages];
    Codec in_codec[kInStages];
    Codec grp_codec[kMaxGroups];   // per compute group: its tile's codec, for pass B
    const BatchStack *in_stack[kInStages];
    uint8_t *in_out[kInStages];
    unsigned long long in_gtile[kInStages];   // tile index over the batch (look-back state)
    const BatchStack *st_stack[kStStages];
    unsigned long long st_gtile[kStStages];
};

// The landing barrier of ring entry k and the parity of its phase.
__device__ __forceinline__ uint64_t *entry_full(EncSmem &sm, uint32_t k)
{
    const uint32_t s = k % kInStages;
    return ((k / kInStages) & 1u) ? &sm.in_full2[s] : &sm.in_full[s];
}

__device__ __forceinline__ uint32_t entry_parity(uint32_t k) { return (k / (2 * kInStages)) & 1u; }

// Payload ring entry k (slot k mod kStStages): its fill barrier, its release
// barrier and the parity of their phase.  Entry k's slot is free once entry
// k - kStStages is released.  With barriers per entry mod 2 kStStages the
// phase before entry k's on either barrier is entry k - 2 kStStages's, and
// that one is always complete when entry k is waited for: the writer of k
// consumed it (same writer), and the group filling k - kStStages needed it
// released.  So a parity wait cannot pass on a stale phase.
__device__ __forceinline__ uint64_t *st_full_bar(EncSmem &sm, uint32_t k) { return &sm.st_full[k % (2 * kStStages)]; }
__device__ __forceinline__ uint64_t *st_empty_bar(EncSmem &sm, uint32_t k) { return &sm.st_empty[k % (2 * kStStages)]; }
__device__ __forceinline__ uint32_t st_parity(uint32_t k) { return (k / (2 * kStStages)) & 1u; }

// Wait until payload ring entry k's slot is free (entry k - kStStages
// written out); the first kStStages entries find their slots free.
__device__ __forceinline__ bool st_slot_free(EncSmem &sm, uint32_t k, LaunchCtl *ctl)
{
    if (k < (uint32_t)kStStages) return true;
    return mbar_wait(st_empty_bar(sm, k - kStStages), st_parity(k - kStStages), ctl);
}

// payload bytes of one tile at most (uint16: 256 blocks x 16 planes x 8
// bytes; uint32: 128 blocks x 31 planes x 8 bytes)
constexpr uint32_t kMaxTilePayload = 32768;

struct DecSmem {
    alignas(16) uint8_t pay[kMaxTilePayload + 32];  // the tile's payload (TMA destination)
    uint32_t off[kMaxTileBlocks];                    // offset of each block inside its warp's 32 blocks
    uint8_t hdr[kMaxTileBlocks];                     // header byte of each block
    uint32_t wsum[kWarps];                           // payload bytes of each warp's 32 blocks
    uint32_t br_rel[kMaxTileBlocks];
    uint8_t br_rows[kMaxTileBlocks];
    uint64_t pay_full;                               // the payload's landing
    uint32_t pay_mis;                                // byte offset of the payload's first byte in pay
};

// ---------------------------------------------------------------- scan
// Exclusive scan of per-block sizes (bytes) in smem by warp 0; returns the
// tile aggregate in every lane of warp 0.
__device__ __forceinline__ uint32_t tile_scan(const uint8_t *hdr, uint32_t *off, uint32_t nblk)
{
    const uint32_t lane = threadIdx.x & 31;
    uint32_t sz[8];
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        uint32_t b = lane * 8 + i;
        uint32_t h = b < nblk ? hdr[b] : 0u;
        sz[i] = (h & 0x1fu) * ((h & 0x80u) ? 4u : 8u);
        sum += sz[i];
    }
    uint32_t inc = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= (uint32_t)o) inc += t;
    }
    uint32_t run = inc - sum;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        uint32_t b = lane * 8 + i;
        if (b < nblk) off[b] = run;
        run += sz[i];
    }
    return __shfl_sync(0xffffffffu, inc, 31);
}

// Publish the tile aggregate, look back, publish the inclusive prefix.
// Run by warp 0; returns the tile's exclusive prefix, ok=false on timeout.
__device__ __forceinline__ unsigned long long tile_prefix(unsigned long long *state, unsigned long long tile,
                                                          uint32_t epoch, uint32_t agg, LaunchCtl *ctl, bool &ok)
{
    const uint32_t lane = threadIdx.x & 31;
    ok = true;
    if (tile == 0) {
        if (lane == 0) st_relaxed_u64(state, make_state(epoch, kFlagIncl, agg));
        return 0;
    }
    if (lane == 0) st_relaxed_u64(state + tile, make_state(epoch, kFlagAgg, agg));
    unsigned long long excl = lookback_warp(state, tile, epoch, ctl, ok);
    if (ok && lane == 0) st_relaxed_u64(state + tile, make_state(epoch, kFlagIncl, excl + agg));
    return excl;
}

// ---------------------------------------------------------------- encoder
// Producer warp, all lanes: the block-row table, range bookkeeping and TMA
// issue of tile t into input slot s; the copies complete on `full`.  The
// block-row starts of the tile are computed one per lane, so the warp's
// dependent chain is that of a single block-row.
template <typename T>
__device__ void enc_issue(const Geom &g, const T *in, EncSmem &sm, int s, unsigned long long t, uint64_t *full,
                          uint32_t lane)
{
    if (t == kMarker) {
        if (lane == 0) {
            sm.in_tile[s] = t;
            mbar_arrive(full);
        }
        return;
    }
    constexpr uint32_t ES = sizeof(T);
    const TileInfo ti = tile_info(g, t);
    // ranges: whole-row tiles -> 1 contiguous range; chunked -> one per row.
    // Lane r < nr holds range r: first element es, element count ne.
    uint32_t nr;
    unsigned long long es = 0, ne = 0;
    if (!g.chunked) {
        unsigned long long r0 = 0, rend = 0;
        for (uint32_t q0 = 0; q0 <= ti.nbr; q0 += 32) {
            const uint32_t q = q0 + lane;
            uint32_t nrows = 0;
            unsigned long long rs = 0;
            if (q <= ti.nbr) {
                const unsigned long long rho = ti.rho0 + q;
                rs = rho < g.nrows_b ? brow_start(g, rho, nrows) : (unsigned long long)g.X * g.Y;
            }
            if (q0 == 0) r0 = __shfl_sync(0xffffffffu, rs, 0);
            if (q < ti.nbr) {
                sm.br_rel[s][q] = (uint32_t)((rs - r0) * g.Z);
                sm.br_rows[s][q] = (uint8_t)nrows;
            }
            const uint32_t last = ti.nbr - q0;  // lane holding the end row in this pass
            if (last < 32u) rend = __shfl_sync(0xffffffffu, rs, last);
        }
        nr = 1;
        es = r0 * g.Z;
        ne = (rend - r0) * g.Z;
    } else {
        uint32_t rows;
        const unsigned long long r0 = brow_start(g, ti.rho0, rows);
        if (lane == 0) sm.br_rows[s][0] = (uint8_t)rows;
        const uint32_t col0 = 8u * ti.c0;
        uint32_t col1 = 8u * (ti.c0 + ti.nblk);
        if (col1 > g.Z) col1 = g.Z;
        nr = rows;
        es = (r0 + lane) * g.Z + col0;
        ne = col1 - col0;
    }
    const uintptr_t base = reinterpret_cast<uintptr_t>(in);
    const uintptr_t A0 = (base + 15) & ~(uintptr_t)15;
    const uintptr_t A1 = (base + ES * g.N) & ~(uintptr_t)15;
    uint32_t tx = 0;
    uintptr_t cs = 0, ce = 0;
    uint8_t *dst = nullptr;
    if (lane < nr) {
        uint8_t *sb = sm.in[s] + (g.chunked ? lane * kChunkPitch : 0u);
        const uintptr_t ga = base + ES * es;
        const uintptr_t ge = ga + ES * ne;
        const uintptr_t gs = ga & ~(uintptr_t)15;
        sm.in_mis[s][lane] = (uint32_t)(ga & 15);
        cs = gs > A0 ? gs : A0;
        ce = (ge + 15) & ~(uintptr_t)15;
        if (ce > A1) ce = A1;
        dst = sb + (cs - gs);
        if (ce > cs) tx = (uint32_t)(ce - cs);
        // bytes outside the 16-byte-aligned interior of the whole array
        // (only the first and last tiles): copy them element by element
        for (uintptr_t p = ga; p < ge && p < A0; p += ES)
            *reinterpret_cast<T *>(sb + (p - gs)) = *reinterpret_cast<const T *>(p);
        for (uintptr_t p = (ga > A1 ? ga : A1); p < ge; p += ES)
            *reinterpret_cast<T *>(sb + (p - gs)) = *reinterpret_cast<const T *>(p);
    }
    if (lane == 0) sm.in_tile[s] = t;
    fence_proxy_async_smem();
    tx = __reduce_add_sync(0xffffffffu, tx);
    __syncwarp();
    if (lane == 0) mbar_arrive_expect_tx(full, tx);
    __syncwarp();
    if (lane < nr && ce > cs) bulk_g2s(dst, reinterpret_cast<const void *>(cs), (uint32_t)(ce - cs), full);
}

// Where a lane's two row segments (rows r and r+4 of tile-local block b)
// live, and how many rows / columns of the block are real.
struct SegLoc {
    const uint8_t *pA, *pB;
    uint32_t nrows, ncols;
    uint32_t bz;
    unsigned long long growA;  // element offset of row r's segment from the tile's first row (decoder)
};

template <typename T, bool ENC>
__device__ __forceinline__ SegLoc seg_locate(const Geom &g, const TileInfo &ti, const uint32_t *br_rel,
                                             const uint8_t *br_rows, const uint8_t *stage, const uint32_t *mis,
                                             uint32_t b, uint32_t r)
{
    constexpr uint32_t ES = sizeof(T);
    SegLoc L;
    if (!g.chunked) {
        uint32_t gidx = (b * g.inv_bzb) >> 16;
        L.bz = b - gidx * g.bzb;
        L.nrows = br_rows[gidx];
        unsigned long long e = (unsigned long long)br_rel[gidx] + (unsigned long long)r * g.Z + 8ull * L.bz;
        if (ENC) {
            L.pA = stage + mis[0] + ES * e;
            L.pB = L.pA + 4ull * ES * g.Z;
        }
        L.growA = e;
    } else {
        L.bz = ti.c0 + b;
        L.nrows = br_rows[0];
        if (ENC) {
            L.pA = stage + r * kChunkPitch + mis[r] + 8u * ES * b;
            L.pB = stage + (r + 4) * kChunkPitch + mis[(r + 4) & 7] + 8u * ES * b;
        }
        L.growA = (unsigned long long)r * g.Z + 8ull * L.bz;
    }
    uint32_t left = g.Z - 8u * L.bz;
    L.ncols = left < 8u ? left : 8u;
    return L;
}

template <typename T, int VEC>
__device__ __forceinline__ void load_rows(const SegLoc &L, bool active, uint32_t r, Row<T> &A, Row<T> &B)
{
#pragma unroll
    for (int i = 0; i < Elem<T>::kWords; i++) A.w[i] = B.w[i] = 0;
    if (active && r < L.nrows) {
        load8<VEC>(L.pA, A);
        if (L.ncols < 8) mask_cols(A, L.ncols);
    }
    if (active && r + 4 < L.nrows) {
        load8<VEC>(L.pB, B);
        if (L.ncols < 8) mask_cols(B, L.ncols);
    }
}

// load_rows with the row access width chosen at run time (batch launches,
// whose stacks differ in width and alignment)
template <typename T>
__device__ __forceinline__ void load_rows_any(const SegLoc &L, bool active, uint32_t r, Row<T> &A, Row<T> &B,
                                              uint32_t vec)
{
    if (vec == 16) load_rows<T, 16>(L, active, r, A, B);
    else if (sizeof(T) == 4 || vec == 4) load_rows<T, 4>(L, active, r, A, B);
    else load_rows<T, 2>(L, active, r, A, B);
}

// Named barrier of one compute group (id, thread count), with the AND of a
// predicate over the group's threads.
__device__ __forceinline__ bool group_bar_and(uint32_t id, uint32_t nthreads, bool pred)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.and.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)pred), "r"(id), "r"(nthreads)
        : "memory");
    return r != 0;
}

// Pass A for one unit: statistics -> header byte (lsCOMP/src/cuLSZ_kernel.cu:898-957).
// Returns the header byte (same in the 4 lanes of a block).
template <typename T, int BINS, bool POOL, bool IDENT>
__device__ __forceinline__ uint32_t block_header(const Row<T> &A, const Row<T> &B, const Codec &c, uint32_t &range_bad)
{
    uint32_t choice = 3;
    if (BINS == BINS_MONO) {
        // the bin counts of cuLSZ_kernel.cu:906-935 are equal exactly when no
        // value lies between the two bins, so the choice is the interval
        // holding the smallest value >= bin0
        const uint32_t b0 = c.binc[0];
        uint32_t mn;
        bool any;
        if constexpr (sizeof(T) == 2) {
            // in 16-bit halves: the smallest (v - bin0) mod 2^16 over the block
            // comes from a value >= bin0 when there is one, since every wrapped
            // difference (v < bin0) is larger; bin0 > 65535 leaves none
            if (b0 <= 0xffffu) {
                const uint32_t NB = ((0x10000u - b0) & 0xffffu) * 0x10001u;
                const uint32_t m = min16_from(B, NB, min16_from(A, NB, 0xffffffffu));
                mn = min(m & 0xffffu, m >> 16);
            } else {
                mn = 0xffffu;
            }
            mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, 8));
            mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, 16));
            any = b0 <= 0xffffu && mn <= 0xffffu - b0;
        } else {
            mn = min_from(B, b0, min_from(A, b0, 0xffffffffu));
            mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, 8));
            mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, 16));
            any = mn <= ~b0;
        }
        const uint32_t v = mn + b0;  // smallest value >= bin0 (if any)
        choice = (any && v < c.binc[1])   ? 0u
                 : (any && v < c.binc[2]) ? 1u
                 : (any && v < c.binc[3]) ? 2u
                                          : 3u;
    } else if (BINS == BINS_GENERAL) {
        uint32_t cnt = bin_counts(A, c.binc) + bin_counts(B, c.binc);
        cnt += __shfl_xor_sync(0xffffffffu, cnt, 8);
        cnt += __shfl_xor_sync(0xffffffffu, cnt, 16);
        const uint32_t c0 = cnt & 0xff, c1 = (cnt >> 8) & 0xff, c2 = (cnt >> 16) & 0xff, c3 = cnt >> 24;
        choice = 0;
        if (c1 == c0) {
            choice = 1;
            if (c2 == c1) {
                choice = 2;
                if (c3 == c2) choice = 3;
            }
        }
    }
    bool pool = false;
    if (POOL) {
        uint32_t zc;
        if constexpr (sizeof(T) == 2) {
            const uint32_t nz = nonzero16(B, nonzero16(A, 0u));
            zc = 16u - ((nz & 0xffffu) + (nz >> 16));
        } else {
            zc = zeros(A) + zeros(B);
        }
        zc += __shfl_xor_sync(0xffffffffu, zc, 8);
        zc += __shfl_xor_sync(0xffffffffu, zc, 16);
        pool = (int)zc >= c.pool_min;
    }
    // rate = bit length of the largest quantised value (cuLSZ_kernel.cu:937-957);
    // quantisation is monotone, so only the block maximum is divided
    uint32_t mx;
    // (the pooled rows only when a block of the warp pools)
    if (IDENT) {
        mx = or_all(A) | or_all(B);  // same bit length as the max
        if (POOL && __any_sync(0xffffffffu, pool)) {
            const uint32_t mp = or_all(pool_rows(A, B));
            if (pool) mx = mp;
        }
        mx |= __shfl_xor_sync(0xffffffffu, mx, 8);
        mx |= __shfl_xor_sync(0xffffffffu, mx, 16);
    } else {
        mx = max(max_all(A), max_all(B));
        if (POOL && __any_sync(0xffffffffu, pool)) {
            const uint32_t mp = max_all(pool_rows(A, B));
            if (pool) mx = mp;
        }
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, 8));
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, 16));
        mx = quant1(mx, c, choice, sizeof(T) == 4);
    }
    const uint32_t rate = bitlen(mx);
    range_bad = rate > Elem<T>::kMaxRate;
    return (pool ? 0x80u : 0u) | (choice << 5) | (rate & 0x1fu);
}

// A row quantised by the block's bin; small (warp-uniform): every value of
// the unit is below 128, so one multiply quantises a pair of values.
__device__ __forceinline__ void quant_row(Row<uint16_t> &v, const Codec &c, uint32_t choice, bool small)
{
    if (small) {
        const uint32_t qsm = c.qsm[choice];
#pragma unroll
        for (int i = 0; i < 4; i++) v.w[i] = lsc_quant7x2(v.w[i], qsm);
    } else {
        quant(v, c, choice);
    }
}

__device__ __forceinline__ void quant_row(Row<uint32_t> &v, const Codec &c, uint32_t choice, bool)
{
    quant(v, c, choice);
}

// One half (rows 0-3 in y1, rows 4-7 in y2) of plane pl of this lane's
// block after the byte transpose, stored at dst.
__device__ __forceinline__ void put_plane(uint8_t *dst, uint32_t y1, uint32_t y2, uint32_t pl, uint32_t rate,
                                          bool pool, bool active)
{
    if (pool) {
        y1 = __byte_perm(y1, 0, 0x3120);  // row pairs were taken in the order 0,2,1,3
        if (active && pl < rate) *reinterpret_cast<uint32_t *>(dst + 4u * pl) = y1;
    } else if (active && pl < rate) {
        // block payloads start at multiples of 4 bytes only (a pooled block
        // has 4 bytes per plane), so the plane pairs go out as two words
        *reinterpret_cast<uint32_t *>(dst + 8u * pl) = y1;
        *reinterpret_cast<uint32_t *>(dst + 8u * pl + 4u) = y2;
    }
}

// Pass B for one unit: bit planes (lsCOMP/src/cuLSZ_kernel.cu:1100-1276) of
// the block whose header is h, stored at dst (shared memory).  IDENT: every
// bin is 1, values are their own quantisation.  NARROW (uint16; callers
// that inline this once, not once per unit): units of small values take
// shorter paths -- pair quotients below 128, planes 0-3 only below 16, one
// word for planes 0-1 of two rows below 4.
template <typename T, bool IDENT, bool NARROW>
__device__ __forceinline__ void block_pack(const Row<T> &A0, const Row<T> &B0, uint32_t h, bool active, uint32_t r,
                                           const XSel &xs, const Codec &c, uint8_t *dst)
{
    constexpr int NW = Elem<T>::kWords;
    constexpr int NG = Elem<T>::kGroups;
    const bool even = (r & 1u) == 0;
    const bool pool = (h & 0x80u) != 0;
    const uint32_t rate = h & 0x1fu;
    const uint32_t choice = (h >> 5) & 3u;
    // the unit's largest rate (the same in every lane): a unit of rate-0
    // blocks only (mostly-zero data) has no planes, so nothing is quantised
    const uint32_t wrate = __reduce_max_sync(0xffffffffu, rate);
    if (wrate == 0u) return;
    const bool small = NARROW && !IDENT && sizeof(T) == 2 &&
                       __all_sync(0xffffffffu, (or_all(A0) | or_all(B0)) < 128u);
    Row<T> A = A0, B = B0;
    if (__any_sync(0xffffffffu, active && pool)) {
        // pooled blocks: lane r=0 takes row pair (0,1), r=1 (4,5), r=2 (2,3),
        // r=3 (6,7) -- one pooled byte row each
        Row<T> P = pool_rows(A0, B0);
        if (!IDENT) quant_row(P, c, choice, small);
        Row<T> V;
#pragma unroll
        for (int i = 0; i < NW / 2; i++) {
            // even lanes send their second row, odd lanes their first
            const uint32_t t0 = __shfl_xor_sync(0xffffffffu, even ? P.w[NW / 2 + i] : P.w[i], 8);
            V.w[i] = even ? P.w[i] : t0;
            V.w[NW / 2 + i] = even ? t0 : P.w[NW / 2 + i];
        }
        if (pool) {
            A = V;
#pragma unroll
            for (int i = 0; i < NW; i++) B.w[i] = 0;
        } else if (!IDENT) {
            quant_row(A, c, choice, small);
            quant_row(B, c, choice, small);
        }
    } else if (!IDENT) {
        quant_row(A, c, choice, small);
        quant_row(B, c, choice, small);
    }
    if constexpr (NARROW && sizeof(T) == 2) {
        if (wrate <= 2u) {
            // every quantised value of the unit is below 4: planes 0 and 1 of
            // rows r and r+4 in one word (bytes: row r plane 0, plane 1, row
            // r+4 plane 0, plane 1), so one byte transpose leaves lane r with
            // plane r&1 of rows 0-3 (r < 2) or rows 4-7 (r >= 2)
            uint32_t y = xpose4(lsc_rows_planes2(A.w, B.w), xs);
            const uint32_t pl = r & 1u;
            if (pool) {
                y = __byte_perm(y, 0, 0x3120);
                if (active && r < 2u && pl < rate) *reinterpret_cast<uint32_t *>(dst + 4u * pl) = y;
            } else if (active && pl < rate) {
                *reinterpret_cast<uint32_t *>(dst + 8u * pl + 4u * (r >> 1)) = y;
            }
            return;
        }
        if (wrate <= 4u) {
            // below 16: planes 0-3 only, from one word per row
            const uint32_t y1 = xpose4(lsc_row_planes4(A.w[0], A.w[1], A.w[2], A.w[3]), xs);
            const uint32_t y2 = xpose4(lsc_row_planes4(B.w[0], B.w[1], B.w[2], B.w[3]), xs);
            put_plane(dst, y1, y2, r, rate, pool, active);
            return;
        }
    }
#pragma unroll
    for (uint32_t grp = 0; grp < (uint32_t)NG; grp++) {
        if (wrate <= 8u * grp) break;
        uint32_t aL, aH, bL, bH;
        row_planes(A, grp, aL, aH);
        row_planes(B, grp, bL, bH);
        const uint32_t pl = 8u * grp + r;  // planes pl and pl + 4
        put_plane(dst, xpose4(aL, xs), xpose4(bL, xs), pl, rate, pool, active);
        if (wrate <= 8u * grp + 4u) break;  // planes 8 grp + 4.. are empty in the whole unit
        put_plane(dst, xpose4(aH, xs), xpose4(bH, xs), pl + 4u, rate, pool, active);
    }
}

// Compute warps, in GRP independent groups of WPG warps: group g takes the
// CTA's tiles k = g, g + GRP, ..., so several tiles are in flight at once
// and the dependent steps of one tile (reductions, scan, barriers) overlap
// with another's.  Per tile: pass A from the input ring into registers and
// header bytes, tile scan and aggregate publication, pass B into the
// payload ring.  NARROW: the unrolled (register-resident) shapes also take
// block_pack's short paths for small values (the RELOAD shapes always do).
template <typename T, int VEC, int BINS, bool POOL, int GRP, int WPG, bool BATCH, bool NARROW>
__device__ __forceinline__ void enc_compute(const EncArgs<T> &a, EncSmem &sm)
{
    constexpr int UMAX = (Elem<T>::kTileBlocks / 8 + WPG - 1) / WPG;  // units per warp per tile
    // groups of more than 8 warps keep only the header bytes between the
    // passes and read the rows again from the input slot in pass B (the slot
    // is then released after pass B): fewer registers per thread, so more
    // warps fit on the SM
    constexpr bool RELOAD = WPG > 8;
    constexpr int UKEEP = RELOAD ? 1 : UMAX;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t grp = warp / WPG, wg = warp % WPG, gtid = tid - grp * WPG * 32;
    const uint32_t barid = kComputeBarrier + grp;
    const uint32_t jb = lane & 7, r = lane >> 3;
    const XSel xs = xsel(r);
    uint8_t *const hdr = sm.hdr[grp];
    uint32_t *const off = sm.off[grp];
    for (uint32_t k = grp;; k += GRP) {
        const int i = (int)(k % kInStages), j = (int)(k % kStStages);
        bool ok = mbar_wait(entry_full(sm, k), entry_parity(k), a.ctl);
        if (!group_bar_and(barid, WPG * 32, ok)) break;
        const unsigned long long t = sm.in_tile[i];  // tile index inside its stack
        if (t == kMarker) {
            // end of this CTA's tiles: hand an end marker to the writer
            if (gtid == 0 && st_slot_free(sm, k, a.ctl)) {
                sm.st_tile[j] = t;
                mbar_arrive_cnt(st_full_bar(sm, k), WPG);
            }
            break;
        }
        // the slot's batch fields are read before the slot is released (the
        // producer may refill it while this tile is packed); g is only used
        // while the slot is held
        const Geom &g = BATCH ? sm.in_geom[i] : a.g;
        uint8_t *const out = BATCH ? sm.in_out[i] : a.out;
        const BatchStack *const bstack = BATCH ? sm.in_stack[i] : nullptr;
        const unsigned long long gt = BATCH ? sm.in_gtile[i] : t;  // look-back state of the tile
        const Codec &cA = BATCH ? sm.in_codec[i] : a.c;             // pass A reads the slot's codec
        const Codec &cB = BATCH ? sm.grp_codec[grp] : a.c;          // pass B the group's copy
        if (BATCH) {
            constexpr uint32_t kCWords = sizeof(Codec) / 4;
            if (gtid < kCWords)
                reinterpret_cast<uint32_t *>(&sm.grp_codec[grp])[gtid] =
                    reinterpret_cast<const uint32_t *>(&sm.in_codec[i])[gtid];
        }
        const TileInfo ti = tile_info(g, t);
        const uint8_t *stage = sm.in[i];

        // ---- pass A: rows to registers (RELOAD: not kept), header bytes
        const uint32_t nunits = (ti.nblk + 7) >> 3;
        Row<T> A[UKEEP], B[UKEEP];
        uint32_t hq[UKEEP];
        uint32_t bad = 0;
        // rows r and r+4 of this lane's block of unit u, from the input slot
        auto load_unit = [&](uint32_t u, Row<T> &ra, Row<T> &rb_) {
            const uint32_t b = u * 8 + jb;
            const bool active = b < ti.nblk;
            SegLoc L = seg_locate<T, true>(g, ti, sm.br_rel[i], sm.br_rows[i], stage, sm.in_mis[i], active ? b : 0, r);
            if constexpr (BATCH) load_rows_any<T>(L, active, r, ra, rb_, g.vec);
            else load_rows<T, VEC>(L, active, r, ra, rb_);
        };
        auto header_unit = [&](uint32_t u, const Row<T> &ra, const Row<T> &rb_) -> uint32_t {
            const uint32_t b = u * 8 + jb;
            uint32_t rb;
            const uint32_t h =
                block_header<T, BINS == BINS_IDENT ? BINS_EQUAL : BINS, POOL, BINS == BINS_IDENT>(ra, rb_, cA, rb);
            if (b < ti.nblk && r == 0) {
                hdr[b] = (uint8_t)h;
                bad |= rb;
            }
            return h;
        };
        if constexpr (RELOAD) {
            // one copy of the unit code (the instruction cache holds the
            // whole loop); the rows are read again in pass B
#pragma unroll 1
            for (uint32_t u = wg; u < nunits; u += WPG) {
                Row<T> ra, rb_;
                load_unit(u, ra, rb_);
                header_unit(u, ra, rb_);
            }
        } else {
#pragma unroll
            for (int q = 0; q < UKEEP; q++) {
                const uint32_t u = wg + (uint32_t)q * WPG;
                hq[q] = 0;
                if (u < nunits) {
                    load_unit(u, A[q], B[q]);
                    hq[q] = header_unit(u, A[q], B[q]);
                }
            }
        }
        __syncwarp();
        if (!RELOAD && lane == 0) mbar_arrive(&sm.in_empty[i]);  // the input slot may be refilled
        if (!group_bar_and(barid, WPG * 32, bad == 0)) {
            // a uint32 quotient >= 2^31 needs 32 planes, which the 5-bit rate
            // field cannot hold
            if (gtid == 0) raise_error(a.ctl, DEV_ERR_RANGE);
            break;
        }

        // ---- tile scan; the aggregate goes out before anything waits on the writer
        if (wg == 0) {
            const uint32_t agg = tile_scan(hdr, off, ti.nblk);
            if (lane == 0) {
                sm.agg[grp] = agg;
                st_relaxed_u64(a.state + gt, make_state(a.epoch, t == 0 ? kFlagIncl : kFlagAgg, agg));
            }
        }
        for (uint32_t b = gtid; b < ti.nblk; b += WPG * 32) out[ti.k0 + b] = hdr[b];
        bool free_ok = true;
        if (gtid == 0) free_ok = st_slot_free(sm, k, a.ctl);
        if (!group_bar_and(barid, WPG * 32, free_ok)) break;

        // ---- pass B: pack (from registers, or RELOAD: from the input slot) into the payload ring
        uint8_t *const st = sm.st[j];
        if constexpr (RELOAD) {
#pragma unroll 1
            for (uint32_t u = wg; u < nunits; u += WPG) {
                const uint32_t b = u * 8 + jb;
                const bool active = b < ti.nblk;
                Row<T> ra, rb_;
                load_unit(u, ra, rb_);
                block_pack<T, BINS == BINS_IDENT, true>(ra, rb_, active ? (uint32_t)hdr[b] : 0u, active, r, xs, cB,
                                                        st + (active ? off[b] : 0u));
            }
        } else {
#pragma unroll
            for (int q = 0; q < UKEEP; q++) {
                const uint32_t u = wg + (uint32_t)q * WPG;
                if (u < nunits) {
                    const uint32_t b = u * 8 + jb;
                    const bool active = b < ti.nblk;
                    block_pack<T, BINS == BINS_IDENT, NARROW>(A[q], B[q], hq[q], active, r, xs, cB,
                                                             st + (active ? off[b] : 0u));
                }
            }
        }
        if (RELOAD) {
            __syncwarp();
            if (lane == 0) mbar_arrive(&sm.in_empty[i]);  // the input slot may be refilled
        }
        // each warp reports its part of the packed tile; the writer waits for all
        if (gtid == 0) {
            sm.st_tile[j] = t;
            sm.st_agg[j] = sm.agg[grp];
            if (BATCH) {
                sm.st_stack[j] = bstack;
                sm.st_gtile[j] = gt;
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(st_full_bar(sm, k));
    }
}

// Producer warp: claims tiles in ticket order and fills the input ring;
// after the last tile, one end marker per compute group.
// Batch launches: copy the stack of tile gt (over the batch) into input
// slot s and return the tile's index inside its stack and its input.
template <typename T>
__device__ __forceinline__ unsigned long long batch_slot(const EncArgs<T> &a, EncSmem &sm, int s,
                                                         unsigned long long gt, const T *&in, uint32_t lane)
{
    const BatchStack *st = a.stacks + a.tile_stack[gt];
    constexpr uint32_t kWords = sizeof(Geom) / 4;
    static_assert(sizeof(Geom) % 4 == 0, "geometry copied in words");
    const uint32_t *src = reinterpret_cast<const uint32_t *>(&st->g);
    uint32_t *dst = reinterpret_cast<uint32_t *>(&sm.in_geom[s]);
    for (uint32_t w = lane; w < kWords; w += 32) dst[w] = src[w];
    constexpr uint32_t kCWords = sizeof(Codec) / 4;
    static_assert(sizeof(Codec) % 4 == 0, "codec copied in words");
    const uint32_t *csrc = reinterpret_cast<const uint32_t *>(&st->c);
    uint32_t *cdst = reinterpret_cast<uint32_t *>(&sm.in_codec[s]);
    for (uint32_t w = lane; w < kCWords; w += 32) cdst[w] = csrc[w];
    if (lane == 0) {
        sm.in_stack[s] = st;
        sm.in_out[s] = st->out;
        sm.in_gtile[s] = gt;
    }
    in = static_cast<const T *>(st->in);
    const unsigned long long t = gt - st->tile0;
    __syncwarp();
    return t;
}

template <typename T, int GRP, bool BATCH>
__device__ __forceinline__ void enc_producer(const EncArgs<T> &a, EncSmem &sm)
{
    const uint32_t lane = threadIdx.x & 31;
    const unsigned long long ntiles = BATCH ? a.ntiles_all : a.g.ntiles;
    uint32_t k = 0, ends = 0;
    // lane 0 holds the next three tickets, claimed in program order (so in
    // increasing order): a claim's round trip (about a microsecond under
    // load) is spread over three tiles instead of bounding the issue rate
    // at one tile per round trip.  Tiles are still taken in claim order, so
    // every tile a look-back waits for belongs to a running CTA.
    unsigned long long q0 = 0, q1 = 0, q2 = 0;
    if (lane == 0) {
        q0 = atomicAdd(&a.ctl->ticket, 1ull);
        q1 = atomicAdd(&a.ctl->ticket, 1ull);
        q2 = atomicAdd(&a.ctl->ticket, 1ull);
    }
    for (;; k++) {
        const int i = (int)(k % kInStages);
        const uint32_t n = k / kInStages;
        bool ok = mbar_wait(&sm.in_empty[i], (n & 1u) ^ 1u, a.ctl);
        if (!__all_sync(0xffffffffu, ok)) break;
        unsigned long long t = __shfl_sync(0xffffffffu, q0, 0);
        const bool real = t < ntiles;
        if (real) {
            if (lane == 0) {
                q0 = q1;
                q1 = q2;
                q2 = atomicAdd(&a.ctl->ticket, 1ull);
            }
        } else {
            t = kMarker;
        }
        __syncwarp();
        if (BATCH && real) {
            const T *in;
            t = batch_slot<T>(a, sm, i, t, in, lane);
            enc_issue<T>(sm.in_geom[i], in, sm, i, t, entry_full(sm, k), lane);  // the whole warp
        } else {
            enc_issue<T>(a.g, a.in, sm, i, t, entry_full(sm, k), lane);  // the whole warp
        }
        if (!real && ++ends == (uint32_t)GRP) {
            k++;
            break;
        }
    }
    if (lane == 0) sm.issued = k;
}

// Writer warp w: for the CTA's tiles k = w, w + NWR, ..., the look-back
// for the tile's stream offset (bounded below by this writer's previous
// tile, whose inclusive prefix it published itself), publication of the
// inclusive prefix, and the copy of the packed payload to the stream.
template <typename T, bool BATCH, int NWR>
__device__ __forceinline__ void enc_writer(const EncArgs<T> &a, EncSmem &sm, uint32_t w)
{
    const uint32_t lane = threadIdx.x & 31;
    long long floor = -1;               // this writer's previous tile
    unsigned long long floor_incl = 0;  // and its inclusive prefix
    for (uint32_t k = w;; k += NWR) {
        const int j = (int)(k % kStStages);
        bool ok = mbar_wait(st_full_bar(sm, k), st_parity(k), a.ctl);
        if (!__all_sync(0xffffffffu, ok)) break;
        const unsigned long long t = sm.st_tile[j];  // tile index inside its stack
        if (t == kMarker) break;
        const BatchStack *bs = BATCH ? sm.st_stack[j] : nullptr;
        const Geom &g = BATCH ? bs->g : a.g;
        uint8_t *const out = BATCH ? bs->out : a.out;
        const unsigned long long cap = BATCH ? bs->cap : a.cap;
        const unsigned long long gt = BATCH ? sm.st_gtile[j] : t;  // look-back state of the tile
        const uint32_t agg = sm.st_agg[j];
        unsigned long long excl = 0;
        if (t > 0) {
            bool lok = true;
#if LSC_LOOKBACK
            excl = lookback_floor(a.state, (long long)gt, floor, floor_incl, a.epoch, a.ctl, lok);
#else
            excl = lookback_warp(a.state, gt, a.epoch, a.ctl, lok);
#endif
            if (!lok) break;
            if (lane == 0) st_relaxed_u64(a.state + gt, make_state(a.epoch, kFlagIncl, excl + agg));
        }
        floor = (long long)gt;
        floor_incl = excl + agg;
        if (g.R + excl + agg > cap) {
            if (lane == 0) raise_error(a.ctl, DEV_ERR_CAPACITY);
            break;
        }
        // copy [0, agg) of the ring slot to out + R + excl (4-byte aligned)
        const uint8_t *src = sm.st[j];
        uint8_t *dst = out + g.R + excl;
        // in consecutive words per lane: conflict-free shared loads and 128
        // contiguous bytes per warp store
        {
            const uint32_t *s32 = reinterpret_cast<const uint32_t *>(src);
            uint32_t *d32 = reinterpret_cast<uint32_t *>(dst);
            const uint32_t nw = agg / 4u;
#pragma unroll 4
            for (uint32_t w = lane; w < nw; w += 32) d32[w] = s32[w];
        }
        if (t == g.ntiles - 1) {
            if (lane == 0) {
                if (BATCH) {
                    bs->sizes[0] = g.R + excl + agg;
                    bs->sizes[1] = excl + agg;
                } else {
                    a.ctl->total = excl + agg;
                    a.ctl->stream_len = g.R + excl + agg;
                    if (a.sizes_out) {
                        a.sizes_out[0] = g.R + excl + agg;
                        a.sizes_out[1] = excl + agg;
                    }
                }
            }
            if (lane < (uint32_t)(g.R - g.nb)) out[g.nb + lane] = 0;  // header pad
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(st_empty_bar(sm, k));
    }
}

template <typename T, int VEC, int BINS, bool POOL, int GRP, int WPG, bool BATCH, bool NARROW = false>
__global__ void __launch_bounds__(EncShape<GRP, WPG>::kThreads, 1) enc_kernel(const EncArgs<T> a)
{
    using S = EncShape<GRP, WPG>;
    static_assert(GRP <= kMaxGroups, "compute groups");
    // a single writer takes every entry and stops at the first end marker
    // (no real tile follows one); several take one group's entries each
    static_assert(S::kWriters == 1 || S::kWriters == GRP, "writer w takes the tiles and the end marker of group w");
    extern __shared__ __align__(128) uint8_t smem_raw[];
    EncSmem &sm = *reinterpret_cast<EncSmem *>(smem_raw);
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    if (tid == 0) {
        for (int s = 0; s < kInStages; s++) {
            mbar_init(&sm.in_full[s], 1);
            mbar_init(&sm.in_full2[s], 1);
            mbar_init(&sm.in_empty[s], WPG);
        }
        for (int s = 0; s < 2 * kStStages; s++) {
            mbar_init(&sm.st_full[s], WPG);
            mbar_init(&sm.st_empty[s], 1);
        }
        sm.issued = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (warp < (uint32_t)S::kCompute)
        enc_compute<T, VEC, BINS, POOL, GRP, WPG, BATCH, NARROW>(a, sm);
    else if (warp == (uint32_t)S::kProducerWarp)
        enc_producer<T, GRP, BATCH>(a, sm);
    else
        enc_writer<T, BATCH, S::kWriters>(a, sm, warp - (uint32_t)S::kWriterWarp0);
    __syncthreads();
    // After an error a load may still be in flight into a slot nobody
    // consumed; the last fill of every slot must land before the CTA's
    // shared memory is released.
    if (tid == (uint32_t)S::kProducerWarp * 32) {
        const uint32_t n = sm.issued;
        for (uint32_t u = n > (uint32_t)kInStages ? n - kInStages : 0; u < n; u++)
            mbar_wait(entry_full(sm, u), entry_parity(u), a.ctl);
    }
}

// ---------------------------------------------------------------- decoder
// Decoding needs no look-back on the critical path: the header bytes hold
// every block's size, so a small first kernel turns them into per-tile
// stream offsets and the decode kernel then runs every tile independently.
constexpr int kSegTiles = 32;  // tiles per segment of the offsets kernel (one per lane of warp 0)

// Per-tile payload offsets (relative to roundup4(nb)) from the header bytes
// (sizes as in lsCOMP/src/cuLSZ_kernel.cu:1333-1339), tile_off[t].  Segments
// of kSegTiles tiles are claimed in order and chained by the look-back.
template <typename T>
__global__ void __launch_bounds__(kThreads) dec_offsets_kernel(const DecArgs<T> a)
{
    __shared__ unsigned long long seg_s;
    __shared__ uint32_t tsum[kSegTiles];
    __shared__ uint32_t ok_s;
    const Geom &g = a.g;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned long long nseg = (g.ntiles + kSegTiles - 1) / kSegTiles;
    for (;;) {
        if (tid == 0) seg_s = aborted(a.ctl) ? nseg : atomicAdd(&a.ctl->ticket, 1ull);
        __syncthreads();
        const unsigned long long sg = seg_s;
        if (sg >= nseg) break;
        const unsigned long long t0 = sg * kSegTiles;
        for (uint32_t q = warp; q < (uint32_t)kSegTiles; q += kWarps) {
            const unsigned long long t = t0 + q;
            uint32_t sum = 0;
            if (t < g.ntiles) {
                const TileInfo ti = tile_info(g, t);
                for (uint32_t b = lane; b < ti.nblk; b += 32) {
                    const uint32_t h = a.in[ti.k0 + b];
                    sum += (h & 0x1fu) * ((h & 0x80u) ? 4u : 8u);
                }
            }
            sum = __reduce_add_sync(0xffffffffu, sum);
            if (lane == 0) tsum[q] = sum;
        }
        __syncthreads();
        if (warp == 0) {
            const uint32_t v = tsum[lane];
            uint32_t inc = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t x = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= (uint32_t)o) inc += x;
            }
            const uint32_t agg = __shfl_sync(0xffffffffu, inc, 31);
            bool lok;
            const unsigned long long base = tile_prefix(a.state, sg, a.epoch, agg, a.ctl, lok);
            if (lok && t0 + lane < g.ntiles) a.tile_off[t0 + lane] = base + (inc - v);
            if (lok && t0 + lane == g.ntiles - 1) a.tile_off[g.ntiles] = base + inc;  // end of the payload
            if (lane == 0) ok_s = lok ? 1u : 0u;
        }
        __syncthreads();
        if (!ok_s) break;
    }
}

// Batch form of dec_offsets_kernel: segments numbered over all stacks (a
// segment never spans two), each stack's first segment publishes its
// inclusive prefix at once, so the look-back stays inside a stack.
template <typename T>
__global__ void __launch_bounds__(kThreads) dec_offsets_batch_kernel(const DecArgs<T> a)
{
    __shared__ unsigned long long seg_s;
    __shared__ uint32_t stk_s;
    __shared__ uint32_t tsum[kSegTiles];
    __shared__ uint32_t ok_s;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned long long nseg = a.seg0[a.nstacks];
    for (;;) {
        if (tid == 0) {
            const unsigned long long sg = aborted(a.ctl) ? nseg : atomicAdd(&a.ctl->ticket, 1ull);
            seg_s = sg;
            if (sg < nseg) {
                // the last stack whose first segment is <= sg
                uint32_t lo = 0, hi = a.nstacks - 1;
                while (lo < hi) {
                    const uint32_t mid = (lo + hi + 1) >> 1;
                    if (a.seg0[mid] <= sg) lo = mid;
                    else hi = mid - 1;
                }
                stk_s = lo;
            }
        }
        __syncthreads();
        const unsigned long long sg = seg_s;
        if (sg >= nseg) break;
        const uint32_t sk = stk_s;
        const BatchStack &st = a.stacks[sk];
        const Geom &g = st.g;
        const uint8_t *in = static_cast<const uint8_t *>(st.in);
        unsigned long long *tile_off = a.tile_off + st.tile0 + sk;
        const unsigned long long ls = sg - a.seg0[sk];  // segment inside the stack
        const unsigned long long t0 = ls * kSegTiles;
        for (uint32_t q = warp; q < (uint32_t)kSegTiles; q += kWarps) {
            const unsigned long long t = t0 + q;
            uint32_t sum = 0;
            if (t < g.ntiles) {
                const TileInfo ti = tile_info(g, t);
                for (uint32_t b = lane; b < ti.nblk; b += 32) {
                    const uint32_t h = in[ti.k0 + b];
                    sum += (h & 0x1fu) * ((h & 0x80u) ? 4u : 8u);
                }
            }
            sum = __reduce_add_sync(0xffffffffu, sum);
            if (lane == 0) tsum[q] = sum;
        }
        __syncthreads();
        if (warp == 0) {
            const uint32_t v = tsum[lane];
            uint32_t inc = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t x = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= (uint32_t)o) inc += x;
            }
            const uint32_t agg = __shfl_sync(0xffffffffu, inc, 31);
            bool lok;
            const unsigned long long base = tile_prefix(a.state + a.seg0[sk], ls, a.epoch, agg, a.ctl, lok);
            if (lok && t0 + lane < g.ntiles) tile_off[t0 + lane] = base + (inc - v);
            if (lok && t0 + lane == g.ntiles - 1) tile_off[g.ntiles] = base + inc;  // end of the payload
            if (lane == 0) ok_s = lok ? 1u : 0u;
        }
        __syncthreads();
        if (!ok_s) break;
    }
}

// Plane words of one block for this lane (planes 8 grp + r and 8 grp + r + 4;
// words 1 and 3 hold rows 4-7 of a plain block).  Loads only planes < rate.
// uint16: Z is the word a unit whose largest rate is at most 2 decodes from
// -- plane r&1 of rows 0-3 (r < 2) or rows 4-7 (r >= 2), what the encoder's
// single byte transpose of such a unit wrote.  It is loaded whatever the
// unit's rates: no load waits for the unit's largest rate, and a branch on
// it here cost more than the extra load.
template <typename T>
__device__ __forceinline__ void dec_load(const uint8_t *src, uint32_t h, uint32_t r, uint32_t Y[][4], uint32_t &Z)
{
    constexpr int NG = Elem<T>::kGroups;
    const bool pool = (h & 0x80u) != 0;
    const uint32_t rate = h & 0x1fu;
    Z = 0;
    if (sizeof(T) == 2) {
        const uint32_t pl = r & 1u;
        if (pool) {
            if (r < 2u && pl < rate) Z = *reinterpret_cast<const uint32_t *>(src + 4u * pl);
        } else if (pl < rate) {
            Z = *reinterpret_cast<const uint32_t *>(src + 8u * pl + 4u * (r >> 1));
        }
    }
#pragma unroll
    for (int grp = 0; grp < NG; grp++) {
        Y[grp][0] = Y[grp][1] = Y[grp][2] = Y[grp][3] = 0;
        const uint32_t pl = 8u * grp + r;
        if (pool) {
            if (pl < rate) Y[grp][0] = *reinterpret_cast<const uint32_t *>(src + 4u * pl);
            if (pl + 4u < rate) Y[grp][2] = *reinterpret_cast<const uint32_t *>(src + 4u * (pl + 4u));
        } else {
            if (pl < rate) {
                Y[grp][0] = *reinterpret_cast<const uint32_t *>(src + 8u * pl);
                Y[grp][1] = *reinterpret_cast<const uint32_t *>(src + 8u * pl + 4u);
            }
            if (pl + 4u < rate) {
                Y[grp][2] = *reinterpret_cast<const uint32_t *>(src + 8u * (pl + 4u));
                Y[grp][3] = *reinterpret_cast<const uint32_t *>(src + 8u * (pl + 4u) + 4u);
            }
        }
    }
}

// Values of rows r (A) and r+4 (B) of this lane's block from the unit's
// plane words: transposes back, pooled rows expanded, de-quantised by the
// header's bin.  All 32 lanes of the warp take part (one unit); wrate is
// the unit's largest rate.
template <typename T>
__device__ __forceinline__ void dec_values(uint32_t Y[][4], uint32_t Z, uint32_t h, bool active, uint32_t r,
                                           uint32_t bin, uint32_t wrate, Row<T> &A, Row<T> &B)
{
    constexpr int NW = Elem<T>::kWords;
    constexpr int NG = Elem<T>::kGroups;
    const bool even = (r & 1u) == 0;
    const bool pool = (h & 0x80u) != 0;
    if (wrate == 0u) {  // every block of the unit has rate 0: all values are 0
#pragma unroll
        for (int i = 0; i < NW; i++) A.w[i] = B.w[i] = 0;
        return;
    }
    const XSel xs = xsel(r);
    bool narrow = false;
    if constexpr (sizeof(T) == 2) {
        if (wrate <= 2u) {
            // one word: rows r and r+4, planes 0 and 1 (dec_load's Z)
            if (pool) Z = __byte_perm(Z, 0, 0x3120);  // undo the row-pair order 0,2,1,3
            lsc_rows_values2(xpose4(Z, xs), A.w, B.w);
            narrow = true;
        } else if (wrate <= 4u) {
            uint32_t y1 = Y[0][0];
            if (pool) y1 = __byte_perm(y1, 0, 0x3120);  // undo the row-pair order 0,2,1,3
            lsc_row_values4(xpose4(y1, xs), A.w[0], A.w[1], A.w[2], A.w[3]);
            lsc_row_values4(xpose4(Y[0][1], xs), B.w[0], B.w[1], B.w[2], B.w[3]);
            narrow = true;
        }
    }
    if (!narrow) {
        // plane bytes per byte group, back in row order: [grp][0/1] = lo/hi
        // half of row r (PA) and of row r+4 (PB); groups and halves above the
        // unit's largest rate stay zero without any shuffles
        uint32_t PA[NG][2], PB[NG][2];
#pragma unroll
        for (int grp = 0; grp < NG; grp++) {
            PA[grp][0] = PA[grp][1] = PB[grp][0] = PB[grp][1] = 0;
            if (wrate <= 8u * grp) continue;
            uint32_t y1 = Y[grp][0];
            if (pool) y1 = __byte_perm(y1, 0, 0x3120);  // undo the row-pair order 0,2,1,3
            PA[grp][0] = xpose4(y1, xs);
            PB[grp][0] = xpose4(Y[grp][1], xs);
            if (wrate <= 8u * grp + 4u) continue;
            uint32_t y3 = Y[grp][2];
            if (pool) y3 = __byte_perm(y3, 0, 0x3120);
            PA[grp][1] = xpose4(y3, xs);
            PB[grp][1] = xpose4(Y[grp][3], xs);
        }
        row_values(PA, A, wrate);
        row_values(PB, B, wrate);
    }
    // products below 2^16 in every block of the unit: one multiply per pair
    const bool pair = sizeof(T) == 2 && __all_sync(0xffffffffu, bin <= (0x10000u >> (h & 0x1fu)));
    if (__any_sync(0xffffffffu, active && pool)) {
        // a pooled lane holds the 8 pooled values of its row pair: 4 of the
        // first row, then 4 of the second.  Even lanes keep the first row and
        // send the second; odd lanes the reverse.
        Row<T> Q;
#pragma unroll
        for (int i = 0; i < NW / 2; i++) {
            const uint32_t t0 = __shfl_xor_sync(0xffffffffu, even ? A.w[NW / 2 + i] : A.w[i], 8);
            Q.w[i] = even ? A.w[i] : t0;                    // row r
            Q.w[NW / 2 + i] = even ? t0 : A.w[NW / 2 + i];  // row r+4
        }
        if (pool) {
            A = unpool_row(Q, false, bin, pair);
            B = unpool_row(Q, true, bin, pair);
        }
    }
    if (!pool) {
        dequant(A, bin, pair);
        dequant(B, bin, pair);
    }
}

// store8 with the row access width chosen at run time (batch launches)
template <typename T>
__device__ __forceinline__ void store8_any(T *p, const Row<T> &v, uint32_t ncols, uint32_t vec)
{
    if (vec == 16) store8<16>(p, v, ncols);
    else if (sizeof(T) == 4 || vec == 4) store8<4>(p, v, ncols);
    else store8<2>(p, v, ncols);
}

// Values of one unit from its plane words (dec_values), stored to rows r
// and r+4 of block b (BATCH: with the stack's own row access width).
template <typename T, int VEC, bool BATCH>
__device__ __forceinline__ void dec_unit(const DecArgs<T> &a, const TileInfo &ti, const DecSmem &sm, uint32_t Y[][4],
                                         uint32_t Z, uint32_t h, uint32_t wrate, uint32_t b, uint32_t r,
                                         unsigned long long ebase)
{
    const Geom &g = a.g;
    const bool active = b < ti.nblk;
    SegLoc L = seg_locate<T, false>(g, ti, sm.br_rel, sm.br_rows, nullptr, nullptr, active ? b : 0, r);
    Row<T> A, B;
    dec_values<T>(Y, Z, h, active, r, a.c.bins[(h >> 5) & 3u], wrate, A, B);
    if (active) {
        T *rowA = a.out + ebase + L.growA;
        if constexpr (BATCH) {
            if (r < L.nrows) store8_any<T>(rowA, A, L.ncols, g.vec);
            if (r + 4 < L.nrows) store8_any<T>(rowA + 4ull * g.Z, B, L.ncols, g.vec);
        } else {
            if (r < L.nrows) store8<VEC>(rowA, A, L.ncols);
            if (r + 4 < L.nrows) store8<VEC>(rowA + 4ull * g.Z, B, L.ncols);
        }
    }
}

// One CTA per tile: header bytes -> in-tile offsets -> plane words of each
// block -> values scattered to the output rows
// (lsCOMP/src/cuLSZ_kernel.cu:1440-1640).  Every element of the tile is
// written, zeros for blocks of rate 0.  The in-tile offsets take one
// barrier: thread b scans block b's size inside its warp, the warps' totals
// meet in shared memory, and each block's offset is its in-warp offset plus
// the totals of the warps before it (kept one per lane, read by shuffle).
// Thread 0's bulk copy of the payload is in flight meanwhile.
template <typename T, int VEC, bool BATCH>
__global__ void __launch_bounds__(kThreads, LSC_DEC_CTAS) dec_kernel(const DecArgs<T> a0)
{
    constexpr int NG = Elem<T>::kGroups;
    static_assert(kThreads >= kMaxTileBlocks && kWarps <= 32, "one thread per block of a tile");
    __shared__ DecSmem sm;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t jb = lane & 7, r = lane >> 3;
    // batch launches: one CTA per tile of all stacks; thread 0 looks up the
    // tile's stack and puts that stack's arguments in shared memory
    __shared__ DecArgs<T> sa;
    __shared__ unsigned long long st_s;
    if constexpr (BATCH) {
        if (tid == 0) {
            const unsigned long long tg = blockIdx.x;
            const uint32_t lo = a0.tile_stack[tg];
            const BatchStack &bs = a0.stacks[lo];
            sa = a0;
            sa.g = bs.g;
            sa.c = bs.c;
            sa.in = static_cast<const uint8_t *>(bs.in);
            sa.out = reinterpret_cast<T *>(bs.out);
            sa.cap = bs.cap;
            sa.tile_off = a0.tile_off + bs.tile0 + lo;
            st_s = tg - bs.tile0;
        }
        __syncthreads();
    }
    const DecArgs<T> &a = BATCH ? sa : a0;
    const Geom &g = a.g;
    const unsigned long long t = BATCH ? st_s : (unsigned long long)blockIdx.x;
    if (t >= g.ntiles) return;
    const unsigned long long base = a.tile_off[t], end = a.tile_off[t + 1];

    // thread 0: the tile's payload [R + base, R + end) into shared memory
    // with one bulk copy; the range is clamped to the readable stream and to
    // one tile's maximum
    if (tid == 0) {
        mbar_init(&sm.pay_full, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        uint32_t tx = 0;
        sm.pay_mis = 0;
        if (end >= base && end - base <= kMaxTilePayload && g.R + end <= a.cap) {
            const uintptr_t bp = reinterpret_cast<uintptr_t>(a.in);
            const uintptr_t A0 = (bp + 15) & ~(uintptr_t)15;
            const uintptr_t A1 = (bp + a.cap) & ~(uintptr_t)15;
            const uintptr_t ga = bp + g.R + base, ge = bp + g.R + end;
            const uintptr_t gs = ga & ~(uintptr_t)15;
            uintptr_t cs = gs > A0 ? gs : A0;
            uintptr_t ce = (ge + 15) & ~(uintptr_t)15;
            if (ce > A1) ce = A1;
            sm.pay_mis = (uint32_t)(ga - gs);
            // bytes outside the 16-byte-aligned interior of the stream buffer
            for (uintptr_t q = ga; q < ge && q < A0; q++) sm.pay[q - gs] = *reinterpret_cast<const uint8_t *>(q);
            for (uintptr_t q = (ga > A1 ? ga : A1); q < ge; q++) sm.pay[q - gs] = *reinterpret_cast<const uint8_t *>(q);
            fence_proxy_async_smem();
            if (ce > cs) tx = (uint32_t)(ce - cs);
            mbar_arrive_expect_tx(&sm.pay_full, tx);
            if (tx) bulk_g2s(sm.pay + (cs - gs), reinterpret_cast<const void *>(cs), tx, &sm.pay_full);
        } else {
            mbar_arrive(&sm.pay_full);  // nothing valid to fetch; the checks below report it
        }
    }
    const TileInfo ti = tile_info(g, t);
    uint32_t n0;
    const unsigned long long row0 = brow_start(g, ti.rho0, n0);
    if (!g.chunked) {
        if (tid < ti.nbr) {
            uint32_t nrows;
            const unsigned long long rs = brow_start(g, ti.rho0 + tid, nrows);
            sm.br_rel[tid] = (uint32_t)((rs - row0) * g.Z);
            sm.br_rows[tid] = (uint8_t)nrows;
        }
    } else if (tid == 0) {
        sm.br_rows[0] = (uint8_t)n0;
    }
    {
        // block tid: header byte, size, offset inside the warp's 32 blocks
        const uint32_t h = tid < ti.nblk ? a.in[ti.k0 + tid] : 0u;
        const uint32_t sz = (h & 0x1fu) << (3u - (h >> 7));  // rate planes of 8 bytes, or 4 when pooled
        uint32_t inc = sz;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t x = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= (uint32_t)o) inc += x;
        }
        sm.hdr[tid] = (uint8_t)h;
        sm.off[tid] = inc - sz;
        if (lane == 31) sm.wsum[warp] = inc;
    }
    __syncthreads();
    // lane w < kWarps: bytes before warp w's blocks; agg: the whole tile
    uint32_t wpre;
    {
        const uint32_t v = lane < (uint32_t)kWarps ? sm.wsum[lane] : 0u;
        uint32_t inc = v;
#pragma unroll
        for (int o = 1; o < kWarps; o <<= 1) {
            const uint32_t x = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= (uint32_t)o) inc += x;
        }
        wpre = inc - v;
    }
    const uint32_t agg = __shfl_sync(0xffffffffu, wpre, kWarps - 1) + sm.wsum[kWarps - 1];
    bool ok = true;
    if (g.R + base + agg > a.cap) {
        ok = false;
        if (tid == 0) raise_error(a.ctl, DEV_ERR_CAPACITY);
    } else if (end != base + agg) {
        ok = false;
        if (tid == 0) raise_error(a.ctl, DEV_ERR_CORRUPT);
    }
    // the payload copy must land before the CTA returns or reads it
    const bool landed = mbar_wait_landed(&sm.pay_full, 0);
    if (!ok || !__all_sync(0xffffffffu, landed)) return;

    const uint8_t *const pay = sm.pay + sm.pay_mis;
    const unsigned long long ebase = row0 * g.Z;  // element index of the tile's first row
    const uint32_t nunits = (ti.nblk + 7) >> 3;
    for (uint32_t u = warp; u < nunits; u += kWarps) {
        const uint32_t b = u * 8 + jb;
        const bool active = b < ti.nblk;
        const uint32_t h = active ? sm.hdr[b] : 0u;
        const uint32_t o = sm.off[active ? b : 0] + __shfl_sync(0xffffffffu, wpre, u >> 2);  // 4 units per warp's 32 blocks
        uint32_t Y[NG][4], Z;
        dec_load<T>(pay + (active ? o : 0u), h, r, Y, Z);
        const uint32_t wrate = __reduce_max_sync(0xffffffffu, h & 0x1fu);  // the unit's largest rate
        dec_unit<T, VEC, BATCH>(a, ti, sm, Y, Z, h, wrate, b, r, ebase);
    }
}

}  // namespace lsc
