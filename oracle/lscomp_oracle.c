/*
 * lscomp_oracle.c -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * A plain C (OpenMP) restatement of the lsCOMP 8x8-block codec of
 * hyfshishen/SC25-lsCOMP.  It exists for two jobs only:
 *   1. the parity checker the CUDA path is compared against (tests/ and
 *      __graft_entry__.smoke());
 *   2. the timed CPU baseline in bench.py ("cpu_baseline", kind "port").
 * The product library never links, loads or calls anything in oracle/.
 *
 * Every step follows the reference kernels line by line in *behaviour*
 * (the control flow here is scalar and per block, not per warp):
 *
 *   block geometry, block count        lsCOMP/src/cuLSZ_entry.cu:97-99
 *   block gather with zero padding     lsCOMP/src/cuLSZ_kernel.cu:877-896
 *   zero / bin counts, max, pair max   lsCOMP/src/cuLSZ_kernel.cu:898-917
 *   pooling decision (float compare)   lsCOMP/src/cuLSZ_kernel.cu:920-921
 *   progressive bin choice             lsCOMP/src/cuLSZ_kernel.cu:922-935
 *   rate and header byte               lsCOMP/src/cuLSZ_kernel.cu:937-957
 *   payload base = roundup4(nb)        lsCOMP/src/cuLSZ_kernel.cu:843,1040
 *   per-1024-block tile layout         lsCOMP/src/cuLSZ_kernel.cu:864-868,962-1041,1086-1097
 *   bit-plane packing                  lsCOMP/src/cuLSZ_kernel.cu:1100-1276
 *   reported compressed size           lsCOMP/src/cuLSZ_entry.cu:124-125
 *   decode (sizes, unpack, scatter)    lsCOMP/src/cuLSZ_kernel.cu:1322-1342,1440-1640
 *   uint32 twins                       lsCOMP/src/cuLSZ_kernel.cu:4-824, cuLSZ_entry.cu:18-91
 *
 * Quirks of the reference that are modelled explicitly:
 *   Q1  header pad bytes [nb, roundup4(nb)) are never written by the
 *       reference; here they are written as 0 (the reference output on a
 *       zeroed buffer).
 *   Q2  the reported size is payload + nb, not payload + roundup4(nb).
 *   Q3  with a single 1024-block tile (nb <= 1024) the reference never
 *       stores the grand total, so it reports nb.  ref_size_out carries the
 *       reference's value; stream_len_out is the true stream length.
 *   Q4  decode never writes rate-0 blocks; write_zero_blocks=1 writes the
 *       zeros the reference would leave in a zeroed buffer.
 *   Q7  uint32: pair sums wrap mod 2^32; a quotient >= 2^31 gives rate 32,
 *       whose bit 5 spills into the bin field of the header byte, while the
 *       tile aggregate still counts 32 planes.  The per-1024-block tile
 *       layout is modelled so the stream matches byte for byte.
 */
#include <stdint.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_OK 0
#define ORC_ERR_ARG -1
#define ORC_ERR_CAPACITY -2
#define ORC_ERR_NOMEM -3
#define ORC_ERR_RANGE -4

#define REF_TILE_BLOCKS 1024u /* 32 lanes x block_per_thread (cuLSZ_kernel.h:7) */

typedef struct {
    uint32_t X, Y, Z;
    uint32_t byb, bzb; /* ceil(Y/8), ceil(Z/8) */
    uint64_t nb;       /* X * byb * bzb */
    uint32_t bins[4];
    int pool_min; /* smallest zero count that pools; 65 = never */
} geom_t;

static int set_geom(geom_t *g, uint32_t X, uint32_t Y, uint32_t Z, const uint32_t bins[4], float p)
{
    if (!X || !Y || !Z) return ORC_ERR_ARG;
    for (int k = 0; k < 4; k++) {
        if (!bins[k]) return ORC_ERR_ARG;
        g->bins[k] = bins[k];
    }
    g->X = X; g->Y = Y; g->Z = Z;
    g->byb = (Y + 7) / 8;
    g->bzb = (Z + 7) / 8;
    g->nb = (uint64_t)X * g->byb * g->bzb;
    /* cuLSZ_kernel.cu:920-921: pooling iff (float)zero_count/64 > poolingTH.
       k/64 is exact in binary32, so the compare is evaluated once per k here. */
    g->pool_min = 65;
    for (int k = 0; k <= 64; k++) {
        float sparsity = (float)k / 64.0f;
        if (sparsity > p) { g->pool_min = k; break; }
    }
    return ORC_OK;
}

int lsc_oracle_pool_min_zeros(float p)
{
    for (int k = 0; k <= 64; k++) {
        float sparsity = (float)k / 64.0f;
        if (sparsity > p) return k;
    }
    return 65;
}

uint64_t lsc_oracle_block_count(uint32_t X, uint32_t Y, uint32_t Z)
{
    return (uint64_t)X * ((Y + 7) / 8) * ((Z + 7) / 8);
}

static inline int bitlen32(uint32_t m)
{
    int r = 0;
    while (m) { r++; m >>= 1; }
    return r;
}

/* cuLSZ_kernel.cu:868-896 -- block k -> (x, by, bz); out-of-range elements read as 0. */
#define DEFINE_GATHER(T, SUF)                                                         \
    static void gather_##SUF(const T *in, const geom_t *g, uint64_t k, uint32_t v[64]) \
    {                                                                                 \
        uint64_t per_slice = (uint64_t)g->byb * g->bzb;                               \
        uint64_t x = k / per_slice;                                                   \
        uint64_t rem = k % per_slice;                                                 \
        uint64_t by = rem / g->bzb, bz = rem % g->bzb;                                \
        for (int i = 0; i < 8; i++) {                                                 \
            uint64_t y = by * 8 + i;                                                  \
            for (int j = 0; j < 8; j++) {                                             \
                uint64_t z = bz * 8 + j;                                              \
                v[i * 8 + j] = (y < g->Y && z < g->Z)                                 \
                                   ? (uint32_t)in[(x * g->Y + y) * g->Z + z]          \
                                   : 0u;                                              \
            }                                                                         \
        }                                                                             \
    }
DEFINE_GATHER(uint16_t, u16)
DEFINE_GATHER(uint32_t, u32)

/* cuLSZ_kernel.cu:898-957 -- statistics, pooling, bin choice, rate, header byte.
   declared = bytes the tile aggregate counts (pass 1), written = bytes pass 2
   emits (from the stored header byte); they differ only for a uint32 rate 32. */
static uint8_t block_header(const uint32_t v[64], const geom_t *g, uint32_t *declared, uint32_t *written)
{
    uint32_t zc = 0, cnt[4] = {0, 0, 0, 0}, max1 = 0, max2 = 0;
    for (int i = 0; i < 64; i++) {
        uint32_t val = v[i];
        zc += (val == 0);
        for (int b = 0; b < 4; b++) cnt[b] += (val < g->bins[b]);
        if (val > max1) max1 = val;
        if (i & 1) {
            uint32_t pm = (uint32_t)(v[i - 1] + v[i]) / 2u; /* uint arithmetic, wraps for uint32 data */
            if (pm > max2) max2 = pm;
        }
    }
    int pool = (int)zc >= g->pool_min;
    uint32_t c = 0;
    if (cnt[1] == cnt[0]) {
        c = 1;
        if (cnt[2] == cnt[1]) {
            c = 2;
            if (cnt[3] == cnt[2]) c = 3;
        }
    }
    uint32_t m = (pool ? max2 : max1) / g->bins[c];
    /* 32 - __clz((int)m): a quotient >= 2^31 is a negative int, clz 0, rate 32 */
    int rate = (m & 0x80000000u) ? 32 : bitlen32(m);
    uint32_t hb = (pool ? 0x80u : 0u) | (c << 5) | (uint32_t)rate;
    uint8_t byte = (uint8_t)hb;
    *declared = (uint32_t)rate * (pool ? 4u : 8u);
    *written = (uint32_t)(byte & 0x1f) * ((byte >> 7) ? 4u : 8u);
    return byte;
}

/* cuLSZ_kernel.cu:1100-1276 -- bit planes, least significant plane first;
   within a byte the first element sits in the most significant bit. */
static void pack_block(const uint32_t v[64], uint8_t hb, const geom_t *g, uint8_t *out)
{
    int pool = hb >> 7;
    uint32_t c = (hb & 0x60) >> 5;
    int rate = hb & 0x1f;
    if (!rate) return;
    uint32_t bin = g->bins[c];
    if (pool) {
        uint32_t pq[32];
        for (int i = 0; i < 32; i++) pq[i] = ((uint32_t)(v[2 * i] + v[2 * i + 1]) / 2u) / bin;
        for (int i = 0; i < rate; i++)
            for (int b = 0; b < 4; b++) {
                uint32_t byte = 0;
                for (int k = 0; k < 8; k++) byte |= ((pq[8 * b + k] >> i) & 1u) << (7 - k);
                out[4 * i + b] = (uint8_t)byte;
            }
    } else {
        uint32_t q[64];
        for (int i = 0; i < 64; i++) q[i] = v[i] / bin;
        for (int i = 0; i < rate; i++)
            for (int r = 0; r < 8; r++) {
                uint32_t byte = 0;
                for (int k = 0; k < 8; k++) byte |= ((q[8 * r + k] >> i) & 1u) << (7 - k);
                out[8 * i + r] = (uint8_t)byte;
            }
    }
}

/* cuLSZ_kernel.cu:1467-1627 -- rebuild quantised values and multiply by the bin. */
static void unpack_block(const uint8_t *in, uint8_t hb, const geom_t *g, uint32_t out[64])
{
    int pool = hb >> 7;
    uint32_t c = (hb & 0x60) >> 5;
    int rate = hb & 0x1f;
    uint32_t bin = g->bins[c];
    if (pool) {
        for (int m = 0; m < 32; m++) {
            uint32_t q = 0;
            for (int i = 0; i < rate; i++) q |= (uint32_t)((in[4 * i + m / 8] >> (7 - m % 8)) & 1) << i;
            out[2 * m] = out[2 * m + 1] = q * bin;
        }
    } else {
        for (int e = 0; e < 64; e++) {
            uint32_t q = 0;
            for (int i = 0; i < rate; i++) q |= (uint32_t)((in[8 * i + e / 8] >> (7 - e % 8)) & 1) << i;
            out[e] = q * bin;
        }
    }
}

static void set_threads(int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
}

int lsc_oracle_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Compression.  Writes the whole stream [0, stream_len) into out (pad and
   unwritten gaps as 0).  ref_size_out receives the value the reference's
   host API would report (Q2, Q3, 32-bit total for uint32). */
#define DEFINE_COMPRESS(T, SUF, IS32)                                                                 \
    int lsc_oracle_compress_##SUF(const T *in, uint32_t X, uint32_t Y, uint32_t Z,                    \
                                  const uint32_t bins[4], float p, uint8_t *out, size_t out_cap,      \
                                  size_t *stream_len_out, size_t *ref_size_out, int nthreads)         \
    {                                                                                                 \
        geom_t g;                                                                                     \
        int st = set_geom(&g, X, Y, Z, bins, p);                                                      \
        if (st) return st;                                                                            \
        set_threads(nthreads);                                                                        \
        uint64_t nb = g.nb, R = (nb + 3) / 4 * 4;                                                     \
        uint32_t *decl = (uint32_t *)malloc(nb * sizeof(uint32_t));                                   \
        uint32_t *wrt = (uint32_t *)malloc(nb * sizeof(uint32_t));                                    \
        uint64_t ntile = (nb + REF_TILE_BLOCKS - 1) / REF_TILE_BLOCKS;                                \
        uint64_t *tile_base = (uint64_t *)malloc((ntile + 1) * sizeof(uint64_t));                     \
        uint8_t *hdr = (uint8_t *)malloc(nb ? nb : 1);                                                \
        if (!decl || !wrt || !tile_base || !hdr) {                                                    \
            free(decl); free(wrt); free(tile_base); free(hdr);                                        \
            return ORC_ERR_NOMEM;                                                                     \
        }                                                                                             \
        int64_t k;                                                                                    \
        _Pragma("omp parallel for schedule(static)") for (k = 0; k < (int64_t)nb; k++)                \
        {                                                                                             \
            uint32_t v[64];                                                                           \
            gather_##SUF(in, &g, (uint64_t)k, v);                                                     \
            hdr[k] = block_header(v, &g, &decl[k], &wrt[k]);                                          \
        }                                                                                             \
        /* tile aggregates use declared sizes (pass 1); offsets inside a tile use     \
           the sizes pass 2 derives from the header bytes (cuLSZ_kernel.cu:1086-1097) */ \
        tile_base[0] = R;                                                                             \
        for (uint64_t t = 0; t < ntile; t++) {                                                        \
            uint64_t s = 0, e = (t + 1) * REF_TILE_BLOCKS;                                            \
            if (e > nb) e = nb;                                                                       \
            for (uint64_t j = t * REF_TILE_BLOCKS; j < e; j++) s += decl[j];                          \
            tile_base[t + 1] = tile_base[t] + s;                                                      \
        }                                                                                             \
        uint64_t total = tile_base[ntile] - R;                                                        \
        uint64_t slen = R + total;                                                                    \
        if (IS32 && slen > 0xffffffffull) { st = ORC_ERR_RANGE; goto done; }                          \
        if (slen > out_cap) { st = ORC_ERR_CAPACITY; goto done; }                                     \
        memset(out, 0, slen);                                                                         \
        memcpy(out, hdr, nb);                                                                         \
        int64_t t;                                                                                    \
        _Pragma("omp parallel for schedule(dynamic, 16)") for (t = 0; t < (int64_t)ntile; t++)        \
        {                                                                                             \
            uint64_t off = tile_base[t], e = ((uint64_t)t + 1) * REF_TILE_BLOCKS;                     \
            if (e > nb) e = nb;                                                                       \
            for (uint64_t j = (uint64_t)t * REF_TILE_BLOCKS; j < e; j++) {                            \
                if (wrt[j]) {                                                                         \
                    uint32_t v[64];                                                                   \
                    gather_##SUF(in, &g, j, v);                                                       \
                    pack_block(v, hdr[j], &g, out + off);                                             \
                }                                                                                     \
                off += wrt[j];                                                                        \
            }                                                                                         \
        }                                                                                             \
        if (stream_len_out) *stream_len_out = (size_t)slen;                                           \
        if (ref_size_out) {                                                                           \
            /* cuLSZ_entry.cu:124-125; Q3: one tile never stores the total */                        \
            uint64_t rep = (ntile > 1) ? total : 0;                                                   \
            if (IS32) rep &= 0xffffffffull;                                                           \
            *ref_size_out = (size_t)(rep + nb);                                                       \
        }                                                                                             \
    done:                                                                                             \
        free(decl); free(wrt); free(tile_base); free(hdr);                                            \
        return st;                                                                                    \
    }
DEFINE_COMPRESS(uint16_t, u16, 0)
DEFINE_COMPRESS(uint32_t, u32, 1)

/* Decompression.  cmp_len is the number of readable stream bytes; a stream
   whose headers point past it is rejected (the reference does not check). */
#define DEFINE_DECOMPRESS(T, SUF)                                                                   \
    int lsc_oracle_decompress_##SUF(const uint8_t *cmp, size_t cmp_len, uint32_t X, uint32_t Y,     \
                                    uint32_t Z, const uint32_t bins[4], float p, T *out,            \
                                    int write_zero_blocks, int nthreads)                            \
    {                                                                                               \
        geom_t g;                                                                                   \
        int st = set_geom(&g, X, Y, Z, bins, p);                                                    \
        if (st) return st;                                                                          \
        set_threads(nthreads);                                                                      \
        uint64_t nb = g.nb, R = (nb + 3) / 4 * 4;                                                   \
        if (cmp_len < nb) return ORC_ERR_CAPACITY;                                                  \
        uint64_t *off = (uint64_t *)malloc((nb + 1) * sizeof(uint64_t));                            \
        if (!off) return ORC_ERR_NOMEM;                                                             \
        /* cuLSZ_kernel.cu:1333-1339: sizes from the header bytes, rate = byte & 0x1f */            \
        off[0] = R;                                                                                 \
        for (uint64_t k = 0; k < nb; k++) {                                                         \
            uint8_t b = cmp[k];                                                                     \
            off[k + 1] = off[k] + (uint64_t)(b & 0x1f) * ((b >> 7) ? 4u : 8u);                      \
        }                                                                                           \
        if (off[nb] > cmp_len) { free(off); return ORC_ERR_CAPACITY; }                              \
        uint64_t per_slice = (uint64_t)g.byb * g.bzb;                                               \
        int64_t k;                                                                                  \
        _Pragma("omp parallel for schedule(static)") for (k = 0; k < (int64_t)nb; k++)              \
        {                                                                                           \
            uint8_t b = cmp[k];                                                                     \
            if (!(b & 0x1f) && !write_zero_blocks) continue; /* Q4 */                               \
            uint32_t v[64];                                                                         \
            if (b & 0x1f) unpack_block(cmp + off[k], b, &g, v);                                     \
            else memset(v, 0, sizeof(v));                                                           \
            uint64_t x = (uint64_t)k / per_slice, rem = (uint64_t)k % per_slice;                    \
            uint64_t by = rem / g.bzb, bz = rem % g.bzb;                                            \
            for (int i = 0; i < 8; i++) {                                                           \
                uint64_t y = by * 8 + i;                                                            \
                if (y >= g.Y) break;                                                                \
                for (int j = 0; j < 8; j++) {                                                       \
                    uint64_t z = bz * 8 + j;                                                        \
                    if (z < g.Z) out[(x * g.Y + y) * g.Z + z] = (T)v[i * 8 + j];                    \
                }                                                                                   \
            }                                                                                       \
        }                                                                                           \
        free(off);                                                                                  \
        return ORC_OK;                                                                              \
    }
DEFINE_DECOMPRESS(uint16_t, u16)
DEFINE_DECOMPRESS(uint32_t, u32)

/* Per-block header bytes and declared sizes only (pass 1), for tests that
   look at one stage at a time. */
int lsc_oracle_headers_u16(const uint16_t *in, uint32_t X, uint32_t Y, uint32_t Z,
                           const uint32_t bins[4], float p, uint8_t *hdr, uint32_t *sizes)
{
    geom_t g;
    int st = set_geom(&g, X, Y, Z, bins, p);
    if (st) return st;
    for (uint64_t k = 0; k < g.nb; k++) {
        uint32_t v[64], d, w;
        gather_u16(in, &g, k, v);
        hdr[k] = block_header(v, &g, &d, &w);
        if (sizes) sizes[k] = d;
    }
    return ORC_OK;
}
