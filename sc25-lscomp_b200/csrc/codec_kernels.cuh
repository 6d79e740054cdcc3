// codec_kernels.cuh -- the lsCOMP uint16 block codec as sm_100a kernels.
//
// One launch encodes (or decodes) a whole X x Y x Z stack (z fastest) in a
// single pass over HBM:
//
//   * The stack is cut into *tiles* of consecutive 8x8 blocks (block index
//     order = the stream's order, lsCOMP/src/cuLSZ_kernel.cu:868-872).  A tile
//     is either G whole block-rows (when a block-row has <= kTileBlocks
//     blocks; the tile's input is then one contiguous byte range) or one
//     chunk of a single block-row (8 row segments).
//   * Persistent CTAs claim tiles in increasing order from a ticket counter,
//     so every tile a CTA waits on in the scan belongs to a resident CTA.
//   * Encoder: a tile's input is fetched once with 1-D TMA bulk copies into a
//     double-buffered shared-memory stage; per-block statistics, pooling, bin
//     choice and rate come from one pass over the stage; the tile's payload
//     size is published, a warp-wide decoupled look-back yields the tile's
//     stream offset, and the bit planes are packed from shared memory
//     straight to their final place in the stream.
//   * Decoder: header bytes -> sizes -> the same look-back -> plane words
//     gathered per block -> values scattered to the output rows.
//
// Thread layout inside a warp ("unit" = 8 consecutive blocks of a tile):
// lane = j + 8 r, j = block within the unit, r = 0..3; the lane owns rows r
// and r+4 of block j (8 values each, held as 4 words of two uint16).  The 4
// lanes of a block sit 8 lanes apart, so block reductions and the 4x4 byte
// transposes that assemble plane words are two xor-shuffles (8, 16).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "bitplane.h"
#include "device_prims.cuh"

namespace lsc {

constexpr int kThreads = 256;                     // 8 warps per CTA
constexpr int kWarps = kThreads / 32;
constexpr int kTileBlocks = 256;                  // at most this many blocks per tile
constexpr int kUnitsPerTile = kTileBlocks / 8;
constexpr int kChunkPitch = kTileBlocks * 16 + 32; // bytes per row segment (chunk tiles)
constexpr int kStageBytes = 33280;                // >= one tile's input + alignment slack
constexpr int kStages = 2;

// bins layouts (template parameter)
constexpr int BINS_EQUAL = 0;   // all four bins equal: bin choice is always 3
constexpr int BINS_MONO = 1;    // x <= y <= z <= w (what the CLI accepts)
constexpr int BINS_GENERAL = 2; // anything else the host API allows

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
};

struct Codec {
    uint32_t bins[4];
    uint32_t magic[4];   // ceil(2^32 / bin) for bin >= 2, 0 for bin == 1 (identity)
    uint32_t binc[4];    // bins clamped to 65536 (same counts for 16-bit values)
    int pool_min;        // a block pools iff zero count >= pool_min (65: never)
};

struct EncArgs {
    Geom g;
    Codec c;
    const uint16_t *in;
    uint8_t *out;
    unsigned long long cap;
    LaunchCtl *ctl;
    unsigned long long *state;
    uint32_t epoch;
    unsigned long long *sizes_out;  // optional device copy of {stream_len, payload}
};

struct DecArgs {
    Geom g;
    Codec c;
    const uint8_t *in;
    uint16_t *out;
    unsigned long long cap;  // readable stream bytes
    LaunchCtl *ctl;
    unsigned long long *state;
    uint32_t epoch;
};

// ---------------------------------------------------------------- geometry
struct TileInfo {
    unsigned long long k0;   // first block index
    unsigned long long rho0; // first block-row
    uint32_t nblk;           // blocks in the tile
    uint32_t nbr;            // block-rows (whole-row tiles)
    uint32_t c0;             // first block column (chunked tiles)
};

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
        ti.rho0 = t / g.nc;
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
    unsigned long long x = rho / g.byb;
    uint32_t by = (uint32_t)(rho - x * g.byb);
    uint32_t r = g.Y - 8u * by;
    nrows = r < 8u ? r : 8u;
    return x * g.Y + 8ull * by;
}

// ---------------------------------------------------------------- row I/O
// Load 8 uint16 at p (alignment VEC bytes) as 4 packed words.
template <int VEC>
__device__ __forceinline__ void load8(const uint8_t *p, uint32_t w[4])
{
    if (VEC == 16) {
        uint4 v = *reinterpret_cast<const uint4 *>(p);
        w[0] = v.x; w[1] = v.y; w[2] = v.z; w[3] = v.w;
    } else if (VEC == 4) {
        const uint32_t *q = reinterpret_cast<const uint32_t *>(p);
        w[0] = q[0]; w[1] = q[1]; w[2] = q[2]; w[3] = q[3];
    } else {
        const uint16_t *h = reinterpret_cast<const uint16_t *>(p);
#pragma unroll
        for (int i = 0; i < 4; i++) w[i] = (uint32_t)h[2 * i] | ((uint32_t)h[2 * i + 1] << 16);
    }
}

// keep only the first ncols (1..8) values
__device__ __forceinline__ void mask_cols(uint32_t w[4], uint32_t ncols)
{
#pragma unroll
    for (int i = 0; i < 4; i++) {
        uint32_t keep = ncols >= 2u * i + 2u ? 0xffffffffu : (ncols == 2u * i + 1u ? 0x0000ffffu : 0u);
        w[i] &= keep;
    }
}

template <int VEC>
__device__ __forceinline__ void store8(uint16_t *p, const uint32_t w[4], uint32_t ncols)
{
    if (ncols >= 8u) {
        if (VEC == 16) {
            *reinterpret_cast<uint4 *>(p) = make_uint4(w[0], w[1], w[2], w[3]);
            return;
        } else if (VEC == 4) {
            uint32_t *q = reinterpret_cast<uint32_t *>(p);
            q[0] = w[0]; q[1] = w[1]; q[2] = w[2]; q[3] = w[3];
            return;
        }
    }
#pragma unroll
    for (int i = 0; i < 8; i++)
        if ((uint32_t)i < ncols) p[i] = (uint16_t)(w[i >> 1] >> (16 * (i & 1)));
}

// ---------------------------------------------------------------- arithmetic
__device__ __forceinline__ uint32_t zero_halves(uint32_t w)
{
    // count of zero 16-bit halves in w (0..2)
    uint32_t t = ((w & 0x7fff7fffu) + 0x7fff7fffu) | w;
    return 2u - __popc(t & 0x80008000u);
}

// quantise both halves of w by the bin whose magic number is m (0 = bin 1)
__device__ __forceinline__ uint32_t quant2(uint32_t w, uint32_t m)
{
    if (m == 0u) return w;
    uint32_t lo = __umulhi(w & 0xffffu, m);
    uint32_t hi = __umulhi(w >> 16, m);
    return lo | (hi << 16);
}

// pooled values of one row: floor((v[2p] + v[2p+1]) / 2), p = 0..3, packed
// as two words (p0 | p1 << 16, p2 | p3 << 16)
__device__ __forceinline__ void pool_row(const uint32_t w[4], uint32_t &a, uint32_t &b)
{
    uint32_t m0 = ((w[0] & 0xffffu) + (w[0] >> 16)) >> 1;
    uint32_t m1 = ((w[1] & 0xffffu) + (w[1] >> 16)) >> 1;
    uint32_t m2 = ((w[2] & 0xffffu) + (w[2] >> 16)) >> 1;
    uint32_t m3 = ((w[3] & 0xffffu) + (w[3] >> 16)) >> 1;
    a = m0 | (m1 << 16);
    b = m2 | (m3 << 16);
}

__device__ __forceinline__ uint32_t bitlen(uint32_t v) { return 32u - __clz(v); }

// 4x4 byte transpose across the lanes j, j+8, j+16, j+24 (r = lane >> 3):
// lane r ends with byte c = byte r of lane c's input.
__device__ __forceinline__ uint32_t xpose4(uint32_t x, uint32_t r)
{
    uint32_t t = __shfl_xor_sync(0xffffffffu, x, 16);
    uint32_t z = (r < 2u) ? __byte_perm(x, t, LSC_XP_A_LOW) : __byte_perm(t, x, LSC_XP_A_HIGH);
    t = __shfl_xor_sync(0xffffffffu, z, 8);
    return (r & 1u) ? __byte_perm(z, t, LSC_XP_B_ODD) : __byte_perm(z, t, LSC_XP_B_EVEN);
}

// ---------------------------------------------------------------- shared state
struct EncSmem {
    alignas(128) uint8_t stage[kStages][kStageBytes];
    uint64_t bar[kStages];
    unsigned long long tile[kStages];
    uint32_t mis[kStages][8];       // byte misalignment of each range start (mod 16)
    uint32_t br_rel[kTileBlocks];   // whole-row tiles: element offset of block-row g from the tile start
    uint8_t br_rows[kTileBlocks];   // rows in block-row g
    uint8_t hdr[kTileBlocks];       // header byte per block
    uint32_t off[kTileBlocks];      // payload offset of each block inside the tile
    unsigned long long base;        // stream offset of the tile payload (relative to R)
    uint32_t agg;
    uint32_t flag_ok;
};

struct DecSmem {
    unsigned long long tile;
    uint32_t br_rel[kTileBlocks];
    uint8_t br_rows[kTileBlocks];
    uint8_t hdr[kTileBlocks];
    uint32_t off[kTileBlocks];
    unsigned long long base;
    uint32_t agg;
    uint32_t flag_ok;
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
        if (lane == 0) st_release_u64(state, make_state(epoch, kFlagIncl, agg));
        return 0;
    }
    if (lane == 0) st_release_u64(state + tile, make_state(epoch, kFlagAgg, agg));
    unsigned long long excl = lookback_warp(state, tile, epoch, ctl, ok);
    if (ok && lane == 0) st_release_u64(state + tile, make_state(epoch, kFlagIncl, excl + agg));
    return excl;
}

// ---------------------------------------------------------------- encoder
// Thread 0: claim-time bookkeeping and TMA issue for one tile into stage s.
template <int VEC>
__device__ void enc_issue(const EncArgs &a, EncSmem &sm, int s, unsigned long long t)
{
    sm.tile[s] = t;
    if (t >= a.g.ntiles) {
        mbar_arrive(&sm.bar[s]);
        return;
    }
    const Geom &g = a.g;
    TileInfo ti = tile_info(g, t);
    const uintptr_t base = reinterpret_cast<uintptr_t>(a.in);
    const uintptr_t A0 = (base + 15) & ~(uintptr_t)15;
    const uintptr_t A1 = (base + 2ull * g.N) & ~(uintptr_t)15;
    uint8_t *stage = sm.stage[s];

    // ranges: whole-row tiles -> 1 contiguous range; chunked -> one per row
    uint32_t nr;
    unsigned long long es[8], ne[8];
    if (!g.chunked) {
        uint32_t rows_first, rows_last;
        unsigned long long r0 = brow_start(g, ti.rho0, rows_first);
        unsigned long long rl = brow_start(g, ti.rho0 + ti.nbr - 1, rows_last);
        es[0] = r0 * g.Z;
        ne[0] = (rl + rows_last) * g.Z - es[0];
        nr = 1;
    } else {
        uint32_t rows;
        unsigned long long r0 = brow_start(g, ti.rho0, rows);
        uint32_t col0 = 8u * ti.c0;
        uint32_t col1 = 8u * (ti.c0 + ti.nblk);
        if (col1 > g.Z) col1 = g.Z;
        nr = rows;
        for (uint32_t r = 0; r < rows; r++) {
            es[r] = (r0 + r) * g.Z + col0;
            ne[r] = col1 - col0;
        }
    }
    uint32_t tx = 0;
    uintptr_t cs_[8], ce_[8];
    uint8_t *dst_[8];
    for (uint32_t i = 0; i < nr; i++) {
        uint8_t *sb = stage + (g.chunked ? i * kChunkPitch : 0);
        uintptr_t ga = base + 2ull * es[i];
        uintptr_t ge = ga + 2ull * ne[i];
        uintptr_t gs = ga & ~(uintptr_t)15;
        sm.mis[s][i] = (uint32_t)(ga & 15);
        uintptr_t cs = gs > A0 ? gs : A0;
        uintptr_t ce = (ge + 15) & ~(uintptr_t)15;
        if (ce > A1) ce = A1;
        cs_[i] = cs; ce_[i] = ce; dst_[i] = sb + (cs - gs);
        if (ce > cs) tx += (uint32_t)(ce - cs);
        // bytes outside the 16-byte-aligned interior of the whole array
        // (only the first and last tiles): copy them as 16-bit values
        for (uintptr_t p = ga; p < ge && p < A0; p += 2)
            *reinterpret_cast<uint16_t *>(sb + (p - gs)) = *reinterpret_cast<const uint16_t *>(p);
        for (uintptr_t p = (ga > A1 ? ga : A1); p < ge; p += 2)
            *reinterpret_cast<uint16_t *>(sb + (p - gs)) = *reinterpret_cast<const uint16_t *>(p);
    }
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&sm.bar[s], tx);
    for (uint32_t i = 0; i < nr; i++)
        if (ce_[i] > cs_[i])
            bulk_g2s(dst_[i], reinterpret_cast<const void *>(cs_[i]), (uint32_t)(ce_[i] - cs_[i]), &sm.bar[s]);
}

// Where lane's two row segments (rows r and r+4 of tile-local block b) live
// in the stage, and how many rows / columns of the block are real.
struct SegLoc {
    const uint8_t *pA, *pB;
    uint32_t nrows, ncols;
    uint32_t bz;
    unsigned long long growA;  // global row index of row r (decoder)
};

template <bool ENC>
__device__ __forceinline__ SegLoc seg_locate(const Geom &g, const TileInfo &ti, const uint32_t *br_rel,
                                             const uint8_t *br_rows, const uint8_t *stage, const uint32_t *mis,
                                             uint32_t b, uint32_t r)
{
    SegLoc L;
    if (!g.chunked) {
        uint32_t gidx = (b * g.inv_bzb) >> 16;
        L.bz = b - gidx * g.bzb;
        L.nrows = br_rows[gidx];
        unsigned long long e = (unsigned long long)br_rel[gidx] + (unsigned long long)r * g.Z + 8ull * L.bz;
        if (ENC) {
            L.pA = stage + mis[0] + 2ull * e;
            L.pB = L.pA + 8ull * g.Z;
        }
        L.growA = e;  // relative element offset (decoder adds the tile start)
    } else {
        L.bz = ti.c0 + b;
        L.nrows = br_rows[0];
        if (ENC) {
            L.pA = stage + r * kChunkPitch + mis[r] + 16u * b;
            L.pB = stage + (r + 4) * kChunkPitch + mis[(r + 4) & 7] + 16u * b;
        }
        L.growA = (unsigned long long)r * g.Z + 8ull * L.bz;
    }
    uint32_t left = g.Z - 8u * L.bz;
    L.ncols = left < 8u ? left : 8u;
    return L;
}

template <int VEC, int BINS, bool POOL>
__global__ void __launch_bounds__(kThreads, 2) enc_kernel(const EncArgs a)
{
    extern __shared__ __align__(128) uint8_t smem_raw[];
    EncSmem &sm = *reinterpret_cast<EncSmem *>(smem_raw);
    const Geom &g = a.g;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t jb = lane & 7, r = lane >> 3;

    if (tid == 0) {
        for (int s = 0; s < kStages; s++) mbar_init(&sm.bar[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        for (int s = 0; s < kStages; s++) {
            unsigned long long t = atomicAdd(&a.ctl->ticket, 1ull);
            enc_issue<VEC>(a, sm, s, t);
        }
    }

    uint32_t it = 0;
    bool clean = false;
    for (;; it++) {
        const int s = it & 1;
        const uint32_t parity = (it >> 1) & 1u;
        bool ok = mbar_wait(&sm.bar[s], parity, a.ctl);
        if (!__syncthreads_and(ok)) break;  // every TMA this CTA issued has landed or timed out
        const unsigned long long t = sm.tile[s];
        if (t >= g.ntiles) { clean = true; break; }
        const TileInfo ti = tile_info(g, t);
        const uint8_t *stage = sm.stage[s];

        // block-row table for whole-row tiles
        if (!g.chunked) {
            if (tid < ti.nbr) {
                uint32_t nrows;
                unsigned long long rs = brow_start(g, ti.rho0 + tid, nrows);
                uint32_t n0;
                unsigned long long r0 = brow_start(g, ti.rho0, n0);
                sm.br_rel[tid] = (uint32_t)((rs - r0) * g.Z);
                sm.br_rows[tid] = (uint8_t)nrows;
            }
        } else if (tid == 0) {
            uint32_t nrows;
            brow_start(g, ti.rho0, nrows);
            sm.br_rows[0] = (uint8_t)nrows;
        }
        __syncthreads();

        const uint32_t nunits = (ti.nblk + 7) >> 3;
        // ---- pass A: statistics -> header byte per block
        for (uint32_t u = warp; u < nunits; u += kWarps) {
            const uint32_t b = u * 8 + jb;
            const bool active = b < ti.nblk;
            uint32_t wA[4] = {0, 0, 0, 0}, wB[4] = {0, 0, 0, 0};
            SegLoc L = seg_locate<true>(g, ti, sm.br_rel, sm.br_rows, stage, sm.mis[s], active ? b : 0, r);
            if (active && r < L.nrows) { load8<VEC>(L.pA, wA); if (L.ncols < 8) mask_cols(wA, L.ncols); }
            if (active && r + 4 < L.nrows) { load8<VEC>(L.pB, wB); if (L.ncols < 8) mask_cols(wB, L.ncols); }

            uint32_t choice = 3;
            if (BINS == BINS_MONO) {
                // choice = interval of the smallest value >= bin0 (counts of
                // cuLSZ_kernel.cu:906-935 are equal exactly when an interval is empty)
                uint32_t mn = 0xffffffffu;
                const uint32_t b0 = a.c.binc[0];
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    mn = min(mn, (wA[i] & 0xffffu) - b0); mn = min(mn, (wA[i] >> 16) - b0);
                    mn = min(mn, (wB[i] & 0xffffu) - b0); mn = min(mn, (wB[i] >> 16) - b0);
                }
                mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, 8));
                mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, 16));
                const uint32_t v = mn + b0;  // smallest value >= bin0 (if any)
                const bool any = mn < 0x80000000u;
                choice = (any && v < a.c.binc[1]) ? 0u : (any && v < a.c.binc[2]) ? 1u : (any && v < a.c.binc[3]) ? 2u : 3u;
            } else if (BINS == BINS_GENERAL) {
                uint32_t cnt = 0;  // four 8-bit counters
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    uint32_t w = i < 4 ? wA[i] : wB[i - 4];
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        uint32_t v = h ? (w >> 16) : (w & 0xffffu);
                        cnt += (v < a.c.binc[0]) | ((v < a.c.binc[1]) << 8) | ((v < a.c.binc[2]) << 16) |
                               ((uint32_t)(v < a.c.binc[3]) << 24);
                    }
                }
                cnt += __shfl_xor_sync(0xffffffffu, cnt, 8);
                cnt += __shfl_xor_sync(0xffffffffu, cnt, 16);
                uint32_t c0 = cnt & 0xff, c1 = (cnt >> 8) & 0xff, c2 = (cnt >> 16) & 0xff, c3 = cnt >> 24;
                choice = 0;
                if (c1 == c0) { choice = 1; if (c2 == c1) { choice = 2; if (c3 == c2) choice = 3; } }
            }
            bool pool = false;
            if (POOL) {
                uint32_t zc = 0;
#pragma unroll
                for (int i = 0; i < 4; i++) zc += zero_halves(wA[i]) + zero_halves(wB[i]);
                zc += __shfl_xor_sync(0xffffffffu, zc, 8);
                zc += __shfl_xor_sync(0xffffffffu, zc, 16);
                pool = (int)zc >= a.c.pool_min;
            }
            const uint32_t m = a.c.magic[choice];
            uint32_t orv = 0;
            if (pool) {
                uint32_t p0, p1, p2, p3;
                pool_row(wA, p0, p1);
                pool_row(wB, p2, p3);
                orv = quant2(p0, m) | quant2(p1, m) | quant2(p2, m) | quant2(p3, m);
            } else {
#pragma unroll
                for (int i = 0; i < 4; i++) orv |= quant2(wA[i], m) | quant2(wB[i], m);
            }
            orv |= __shfl_xor_sync(0xffffffffu, orv, 8);
            orv |= __shfl_xor_sync(0xffffffffu, orv, 16);
            const uint32_t rate = bitlen((orv & 0xffffu) | (orv >> 16));
            if (active && r == 0) sm.hdr[b] = (uint8_t)((pool ? 0x80u : 0u) | (choice << 5) | rate);
        }
        __syncthreads();

        // ---- tile size, look-back, stream offset
        if (warp == 0) {
            uint32_t agg = tile_scan(sm.hdr, sm.off, ti.nblk);
            bool lok;
            unsigned long long excl = tile_prefix(a.state, t, a.epoch, agg, a.ctl, lok);
            if (lane == 0) {
                sm.base = excl;
                sm.agg = agg;
                sm.flag_ok = lok ? 1u : 0u;
                if (lok && g.R + excl + agg > a.cap) {
                    raise_error(a.ctl, DEV_ERR_CAPACITY);
                    sm.flag_ok = 0;
                }
                if (lok && t == g.ntiles - 1 && sm.flag_ok) {
                    a.ctl->total = excl + agg;
                    a.ctl->stream_len = g.R + excl + agg;
                    if (a.sizes_out) {
                        a.sizes_out[0] = g.R + excl + agg;
                        a.sizes_out[1] = excl + agg;
                    }
                }
            }
        }
        __syncthreads();
        if (!sm.flag_ok) break;

        // ---- headers of this tile (and the zero pad after the last header)
        for (uint32_t b = tid; b < ti.nblk; b += kThreads) a.out[ti.k0 + b] = sm.hdr[b];
        if (t == g.ntiles - 1 && tid < (uint32_t)(g.R - g.nb)) a.out[g.nb + tid] = 0;

        // ---- pass B: pack bit planes into the stream
        uint8_t *const pay = a.out + g.R + sm.base;
        for (uint32_t u = warp; u < nunits; u += kWarps) {
            const uint32_t b = u * 8 + jb;
            const bool active = b < ti.nblk;
            uint32_t wA[4] = {0, 0, 0, 0}, wB[4] = {0, 0, 0, 0};
            SegLoc L = seg_locate<true>(g, ti, sm.br_rel, sm.br_rows, stage, sm.mis[s], active ? b : 0, r);
            if (active && r < L.nrows) { load8<VEC>(L.pA, wA); if (L.ncols < 8) mask_cols(wA, L.ncols); }
            if (active && r + 4 < L.nrows) { load8<VEC>(L.pB, wB); if (L.ncols < 8) mask_cols(wB, L.ncols); }
            const uint32_t h = active ? sm.hdr[b] : 0u;
            const bool pool = (h & 0x80u) != 0;
            const uint32_t rate = h & 0x1fu;
            const uint32_t m = a.c.magic[(h >> 5) & 3u];
            // the 8 values this lane transposes ("virtual row"): plain blocks
            // use rows r and r+4 as they are
            uint32_t v0 = quant2(wA[0], m), v1 = quant2(wA[1], m), v2 = quant2(wA[2], m), v3 = quant2(wA[3], m);
            uint32_t u0 = quant2(wB[0], m), u1 = quant2(wB[1], m), u2 = quant2(wB[2], m), u3 = quant2(wB[3], m);
            if (__any_sync(0xffffffffu, active && pool)) {
                // pooled blocks: lane r=0 takes rows 0,1; r=1 rows 4,5; r=2 rows 2,3;
                // r=3 rows 6,7 (one pooled byte row pair each)
                uint32_t p0, p1, p2, p3;
                pool_row(wA, p0, p1);
                pool_row(wB, p2, p3);
                p0 = quant2(p0, m); p1 = quant2(p1, m); p2 = quant2(p2, m); p3 = quant2(p3, m);
                const bool even = (r & 1u) == 0;
                const uint32_t t0 = __shfl_xor_sync(0xffffffffu, even ? p2 : p0, 8);
                const uint32_t t1 = __shfl_xor_sync(0xffffffffu, even ? p3 : p1, 8);
                if (pool) {
                    v0 = even ? p0 : t0; v1 = even ? p1 : t1;
                    v2 = even ? t0 : p2; v3 = even ? t1 : p3;
                    u0 = u1 = u2 = u3 = 0;
                }
            }
            const uint32_t wrate = __reduce_max_sync(0xffffffffu, rate);
            uint8_t *const dst = pay + (active ? sm.off[b] : 0u);
            for (uint32_t hi = 0; hi < 2; hi++) {
                if (wrate <= 8u * hi) break;
                uint32_t aL, aH, bL = 0, bH = 0;
                lsc_row_planes(v0, v1, v2, v3, (int)hi, aL, aH);
                lsc_row_planes(u0, u1, u2, u3, (int)hi, bL, bH);
                uint32_t y1 = xpose4(aL, r), y2 = xpose4(bL, r), y3 = xpose4(aH, r), y4 = xpose4(bH, r);
                const uint32_t pl = 8u * hi + r;  // planes pl and pl + 4
                if (pool) {
                    y1 = __byte_perm(y1, 0, 0x3120);
                    y3 = __byte_perm(y3, 0, 0x3120);
                    if (active && pl < rate) *reinterpret_cast<uint32_t *>(dst + 4u * pl) = y1;
                    if (active && pl + 4u < rate) *reinterpret_cast<uint32_t *>(dst + 4u * (pl + 4u)) = y3;
                } else {
                    if (active && pl < rate) {
                        *reinterpret_cast<uint32_t *>(dst + 8u * pl) = y1;
                        *reinterpret_cast<uint32_t *>(dst + 8u * pl + 4u) = y2;
                    }
                    if (active && pl + 4u < rate) {
                        *reinterpret_cast<uint32_t *>(dst + 8u * (pl + 4u)) = y3;
                        *reinterpret_cast<uint32_t *>(dst + 8u * (pl + 4u) + 4u) = y4;
                    }
                }
            }
        }
        __syncthreads();  // stage s fully consumed
        if (tid == 0) {
            unsigned long long nt = aborted(a.ctl) ? g.ntiles : atomicAdd(&a.ctl->ticket, 1ull);
            enc_issue<VEC>(a, sm, s, nt);
        }
    }
    // Leaving early (error): the copy issued into the other stage must land
    // before the CTA's shared memory is released.  Bounded like every wait.
    if (!clean && tid == 0) {
        const int o = (it + 1) & 1;
        mbar_wait(&sm.bar[o], ((it + 1) >> 1) & 1u, a.ctl);
    }
    __syncthreads();
}

// ---------------------------------------------------------------- decoder
template <int VEC>
__global__ void __launch_bounds__(kThreads, 4) dec_kernel(const DecArgs a)
{
    __shared__ DecSmem sm;
    const Geom &g = a.g;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t jb = lane & 7, r = lane >> 3;

    for (;;) {
        if (tid == 0) sm.tile = aborted(a.ctl) ? g.ntiles : atomicAdd(&a.ctl->ticket, 1ull);
        __syncthreads();
        const unsigned long long t = sm.tile;
        if (t >= g.ntiles) break;
        const TileInfo ti = tile_info(g, t);
        unsigned long long row0 = 0;
        {
            uint32_t n0;
            row0 = brow_start(g, ti.rho0, n0);
        }
        if (!g.chunked) {
            if (tid < ti.nbr) {
                uint32_t nrows;
                unsigned long long rs = brow_start(g, ti.rho0 + tid, nrows);
                sm.br_rel[tid] = (uint32_t)((rs - row0) * g.Z);
                sm.br_rows[tid] = (uint8_t)nrows;
            }
        } else if (tid == 0) {
            uint32_t nrows;
            brow_start(g, ti.rho0, nrows);
            sm.br_rows[0] = (uint8_t)nrows;
        }
        for (uint32_t b = tid; b < ti.nblk; b += kThreads) sm.hdr[b] = a.in[ti.k0 + b];
        __syncthreads();
        if (warp == 0) {
            uint32_t agg = tile_scan(sm.hdr, sm.off, ti.nblk);
            bool lok;
            unsigned long long excl = tile_prefix(a.state, t, a.epoch, agg, a.ctl, lok);
            if (lane == 0) {
                sm.base = excl;
                sm.agg = agg;
                sm.flag_ok = lok ? 1u : 0u;
                if (lok && g.R + excl + agg > a.cap) {
                    raise_error(a.ctl, DEV_ERR_CAPACITY);
                    sm.flag_ok = 0;
                }
            }
        }
        __syncthreads();
        if (!sm.flag_ok) break;

        const uint8_t *const pay = a.in + g.R + sm.base;
        const unsigned long long ebase = row0 * g.Z;  // element index of the tile's first row
        const uint32_t nunits = (ti.nblk + 7) >> 3;
        for (uint32_t u = warp; u < nunits; u += kWarps) {
            const uint32_t b = u * 8 + jb;
            const bool active = b < ti.nblk;
            SegLoc L = seg_locate<false>(g, ti, sm.br_rel, sm.br_rows, nullptr, nullptr, active ? b : 0, r);
            const uint32_t h = active ? sm.hdr[b] : 0u;
            const bool pool = (h & 0x80u) != 0;
            const uint32_t rate = h & 0x1fu;
            const uint32_t bin = a.c.bins[(h >> 5) & 3u];
            const uint8_t *src = pay + (active ? sm.off[b] : 0u);
            const uint32_t wrate = __reduce_max_sync(0xffffffffu, rate);
            uint32_t pl_[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};  // [hi][aL, bL, aH, bH] after transpose back
            for (uint32_t hi = 0; hi < 2; hi++) {
                if (wrate <= 8u * hi) break;
                const uint32_t pl = 8u * hi + r;
                uint32_t y1 = 0, y2 = 0, y3 = 0, y4 = 0;
                if (pool) {
                    if (pl < rate) y1 = *reinterpret_cast<const uint32_t *>(src + 4u * pl);
                    if (pl + 4u < rate) y3 = *reinterpret_cast<const uint32_t *>(src + 4u * (pl + 4u));
                    y1 = __byte_perm(y1, 0, 0x3120);
                    y3 = __byte_perm(y3, 0, 0x3120);
                } else {
                    if (pl < rate) {
                        y1 = *reinterpret_cast<const uint32_t *>(src + 8u * pl);
                        y2 = *reinterpret_cast<const uint32_t *>(src + 8u * pl + 4u);
                    }
                    if (pl + 4u < rate) {
                        y3 = *reinterpret_cast<const uint32_t *>(src + 8u * (pl + 4u));
                        y4 = *reinterpret_cast<const uint32_t *>(src + 8u * (pl + 4u) + 4u);
                    }
                }
                pl_[hi][0] = xpose4(y1, r);
                pl_[hi][1] = xpose4(y2, r);
                pl_[hi][2] = xpose4(y3, r);
                pl_[hi][3] = xpose4(y4, r);
            }
            // rebuild the quantised values of this lane's virtual row(s)
            uint32_t wA[4], wB[4];
            lsc_row_values(pl_[0][0], pl_[0][2], pl_[1][0], pl_[1][2], wA[0], wA[1], wA[2], wA[3]);
            lsc_row_values(pl_[0][1], pl_[0][3], pl_[1][1], pl_[1][3], wB[0], wB[1], wB[2], wB[3]);
            if (__any_sync(0xffffffffu, active && pool)) {
                // wA of a pooled lane holds the 8 pooled values of its row pair:
                // 4 of the first row, then 4 of the second.  Even lanes keep the
                // first row and send the second; odd lanes the reverse.
                const bool even = (r & 1u) == 0;
                const uint32_t t0 = __shfl_xor_sync(0xffffffffu, even ? wA[2] : wA[0], 8);
                const uint32_t t1 = __shfl_xor_sync(0xffffffffu, even ? wA[3] : wA[1], 8);
                if (pool) {
                    uint32_t q[4];
                    q[0] = even ? wA[0] : t0; q[1] = even ? wA[1] : t1;  // row r
                    q[2] = even ? t0 : wA[2]; q[3] = even ? t1 : wA[3];  // row r+4
                    uint32_t e[8];
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        // de-quantise and repeat each pooled value over its two columns
                        uint32_t lo = (q[i] & 0xffffu) * bin, hi = (q[i] >> 16) * bin;
                        e[2 * i] = (lo & 0xffffu) | (lo << 16);
                        e[2 * i + 1] = (hi & 0xffffu) | (hi << 16);
                    }
                    wA[0] = e[0]; wA[1] = e[1]; wA[2] = e[2]; wA[3] = e[3];
                    wB[0] = e[4]; wB[1] = e[5]; wB[2] = e[6]; wB[3] = e[7];
                }
            }
            if (!pool && bin != 1u) {
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    uint32_t lo = (wA[i] & 0xffffu) * bin, hi = (wA[i] >> 16) * bin;
                    wA[i] = (lo & 0xffffu) | (hi << 16);
                    lo = (wB[i] & 0xffffu) * bin; hi = (wB[i] >> 16) * bin;
                    wB[i] = (lo & 0xffffu) | (hi << 16);
                }
            }
            if (active) {
                uint16_t *rowA = a.out + ebase + L.growA;
                if (r < L.nrows) store8<VEC>(rowA, wA, L.ncols);
                if (r + 4 < L.nrows) store8<VEC>(rowA + 4ull * g.Z, wB, L.ncols);
            }
        }
        __syncthreads();
    }
}

}  // namespace lsc
