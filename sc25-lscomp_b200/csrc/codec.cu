// codec.cu -- host side of the uint16 codec: argument checks, tile geometry,
// workspace (scan state + launch control block), kernel selection and the
// C ABI declared in include/lscomp.h.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <atomic>
#include <mutex>
#include "lscomp.h"
#include "codec_kernels.cuh"

using namespace lsc;

namespace {

std::atomic<uint64_t> g_launches{0};

constexpr uint32_t kEpochMax = (1u << 20) - 1;

}  // namespace

struct lscomp_workspace {
    int device = 0;
    int sm_count = 0;
    LaunchCtl *ctl = nullptr;          // device
    LaunchCtl *h_ctl = nullptr;        // pinned host mirror for status reads
    unsigned long long *state = nullptr;   // look-back words, then per-tile offsets
    uint64_t state_cap = 0;            // entries of each of the two arrays
    uint32_t epoch = 0;
    std::mutex mu;
};

namespace {

int cuda_status(cudaError_t e)
{
    if (e == cudaSuccess) return LSCOMP_OK;
    if (e == cudaErrorMemoryAllocation) return LSCOMP_ERR_NOMEM;
    return LSCOMP_ERR_CUDA;
}

int dev_status(uint32_t e)
{
    switch (e) {
    case DEV_OK: return LSCOMP_OK;
    case DEV_ERR_TIMEOUT: return LSCOMP_ERR_TIMEOUT;
    case DEV_ERR_CAPACITY: return LSCOMP_ERR_CAPACITY;
    case DEV_ERR_CORRUPT: return LSCOMP_ERR_CORRUPT;
    case DEV_ERR_RANGE: return LSCOMP_ERR_RANGE;
    default: return LSCOMP_ERR_CUDA;
    }
}

// smallest zero count k (0..64) with (float)k/64 > p, 65 if none
// (lsCOMP/src/cuLSZ_kernel.cu:920-921; k/64 is exact in binary32)
int pool_min_zeros(float p)
{
    for (int k = 0; k <= 64; k++) {
        float sparsity = (float)k / 64.0f;
        if (sparsity > p) return k;
    }
    return 65;
}

// ceil(2^64 / b) for b >= 2: with 2^64 - 1 = q b + r (0 <= r < b), 2^64 / b
// = q + (r + 1) / b and 0 < r + 1 <= b, so the ceiling is always q + 1
unsigned long long magic64(uint32_t b)
{
    if (b < 2) return 0;
    return ~0ull / b + 1;
}

bool make_geom(uint32_t X, uint32_t Y, uint32_t Z, uint32_t tile_blocks, Geom &g)
{
    if (!X || !Y || !Z) return false;
    g.X = X; g.Y = Y; g.Z = Z;
    g.byb = (Y + 7) / 8;
    g.bzb = (Z + 7) / 8;
    g.nrows_b = (unsigned long long)X * g.byb;
    g.nb = g.nrows_b * g.bzb;
    g.R = (g.nb + 3) / 4 * 4;
    g.N = (unsigned long long)X * Y * Z;
    if (g.bzb <= tile_blocks) {
        g.chunked = 0;
        g.G = tile_blocks / g.bzb;
        g.ntiles = (g.nrows_b + g.G - 1) / g.G;
        g.nc = 1;
        g.W = g.bzb;
        g.inv_bzb = (65536u + g.bzb - 1) / g.bzb;
    } else {
        g.chunked = 1;
        g.G = 1;
        g.nc = (g.bzb + tile_blocks - 1) / tile_blocks;
        g.W = (g.bzb + g.nc - 1) / g.nc;
        g.ntiles = g.nrows_b * g.nc;
        g.inv_bzb = 0;
    }
    g.byb_magic = magic64(g.byb);
    g.nc_magic = magic64(g.nc);
    return true;
}

bool make_codec(const uint32_t bins[4], float p, bool wide, Codec &c, int &layout)
{
    if (!bins) return false;
    for (int k = 0; k < 4; k++) {
        if (bins[k] == 0) return false;
        c.bins[k] = bins[k];
        c.magic[k] = bins[k] == 1 ? 0u : (uint32_t)((0x100000000ull + bins[k] - 1) / bins[k]);
        c.magic64[k] = magic64(bins[k]);
        c.binc[k] = (!wide && bins[k] > 65536u) ? 65536u : bins[k];
    }
    c.pool_min = pool_min_zeros(p);
    if (bins[0] == 1 && bins[1] == 1 && bins[2] == 1 && bins[3] == 1)
        layout = BINS_IDENT;
    else if (bins[0] == bins[1] && bins[1] == bins[2] && bins[2] == bins[3])
        layout = BINS_EQUAL;
    else if (bins[0] <= bins[1] && bins[1] <= bins[2] && bins[2] <= bins[3])
        layout = BINS_MONO;
    else
        layout = BINS_GENERAL;
    return true;
}

// widest access every row segment of the stack allows (bytes)
int vec_class(const void *p, uint32_t Z, size_t es)
{
    uintptr_t a = reinterpret_cast<uintptr_t>(p);
    if (es == 2) {
        if ((Z % 8u) == 0 && (a % 16u) == 0) return 16;
        if ((Z % 2u) == 0 && (a % 4u) == 0) return 4;
        return 2;
    }
    if ((Z % 4u) == 0 && (a % 16u) == 0) return 16;
    return 4;
}

// Ensure the workspace holds `ntiles` scan slots and hand out a fresh epoch.
int ws_prepare(lscomp_workspace *ws, uint64_t ntiles, cudaStream_t st)
{
    if (ntiles > ws->state_cap) {
        uint64_t cap = ntiles + ntiles / 4 + 1024;
        unsigned long long *p = nullptr;
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_status(e);
        if (ws->state) cudaFree(ws->state);
        ws->state = nullptr;
        ws->state_cap = 0;
        e = cudaMalloc(&p, 2 * cap * sizeof(unsigned long long));
        if (e != cudaSuccess) return cuda_status(e);
        e = cudaMemsetAsync(p, 0, 2 * cap * sizeof(unsigned long long), st);
        if (e != cudaSuccess) { cudaFree(p); return cuda_status(e); }
        ws->state = p;
        ws->state_cap = cap;
        ws->epoch = 0;
    }
    if (ws->epoch >= kEpochMax) {
        cudaError_t e = cudaMemsetAsync(ws->state, 0, ws->state_cap * sizeof(unsigned long long), st);
        if (e != cudaSuccess) return cuda_status(e);
        ws->epoch = 0;
    }
    ws->epoch++;
    cudaError_t e = cudaMemsetAsync(ws->ctl, 0, sizeof(LaunchCtl), st);
    return cuda_status(e);
}

template <typename K>
int ctas_per_sm(K kernel, size_t smem)
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, kThreads, smem) != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}

template <typename T, int VEC, int BINS, bool POOL, int GRP, int WPG>
int launch_enc_w(const EncArgs<T> &a, int sm_count, cudaStream_t st)
{
    auto k = enc_kernel<T, VEC, BINS, POOL, GRP, WPG>;
    const size_t smem = sizeof(EncSmem);
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    // persistent: one CTA per SM (the CTA holds ~200 KB of rings)
    unsigned long long grid = (unsigned long long)sm_count;
    if (grid > a.g.ntiles) grid = a.g.ntiles;
    k<<<(unsigned)grid, EncShape<GRP, WPG>::kThreads, smem, st>>>(a);
    g_launches.fetch_add(1);
    return cuda_status(cudaGetLastError());
}

// Compute warps per encoder CTA: LSC_ENC_GROUPS groups of LSC_ENC_WPG warps.
template <typename T, int VEC, int BINS, bool POOL>
int launch_enc_t(const EncArgs<T> &a, int sm_count, cudaStream_t st)
{
    return launch_enc_w<T, VEC, BINS, POOL, LSC_ENC_GROUPS, LSC_ENC_WPG>(a, sm_count, st);
}

template <typename T, int VEC>
int launch_enc_v(const EncArgs<T> &a, int layout, bool pool, int sm, cudaStream_t st)
{
    if (layout == BINS_IDENT)
        return pool ? launch_enc_t<T, VEC, BINS_IDENT, true>(a, sm, st)
                    : launch_enc_t<T, VEC, BINS_IDENT, false>(a, sm, st);
    if (layout == BINS_EQUAL)
        return pool ? launch_enc_t<T, VEC, BINS_EQUAL, true>(a, sm, st)
                    : launch_enc_t<T, VEC, BINS_EQUAL, false>(a, sm, st);
    if (layout == BINS_MONO)
        return pool ? launch_enc_t<T, VEC, BINS_MONO, true>(a, sm, st)
                    : launch_enc_t<T, VEC, BINS_MONO, false>(a, sm, st);
    return pool ? launch_enc_t<T, VEC, BINS_GENERAL, true>(a, sm, st)
                : launch_enc_t<T, VEC, BINS_GENERAL, false>(a, sm, st);
}

template <typename T, int VEC>
int launch_dec_t(const DecArgs<T> &a, int sm_count, cudaStream_t st)
{
    // 1) per-tile stream offsets from the header bytes
    const unsigned long long nseg = (a.g.ntiles + kSegTiles - 1) / kSegTiles;
    unsigned long long grid = (unsigned long long)sm_count * 4;
    if (grid > nseg) grid = nseg;
    dec_offsets_kernel<T><<<(unsigned)grid, kThreads, 0, st>>>(a);
    g_launches.fetch_add(1);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e);
    // 2) every tile independently
    if (a.g.ntiles > 0x7fffffffull) return LSCOMP_ERR_ARG;
    dec_kernel<T, VEC><<<(unsigned)a.g.ntiles, kThreads, 0, st>>>(a);
    g_launches.fetch_add(1);
    return cuda_status(cudaGetLastError());
}

int read_ctl(lscomp_workspace *ws, cudaStream_t st)
{
    cudaError_t e = cudaMemcpyAsync(ws->h_ctl, ws->ctl, sizeof(LaunchCtl), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return cuda_status(e);
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_status(e);
    return dev_status(ws->h_ctl->error);
}

template <typename T>
int compress_async_t(lscomp_workspace *ws, const T *d_in, uint32_t x, uint32_t y, uint32_t z, const uint32_t bins[4],
                     float pooling, uint8_t *d_out, uint64_t cap, uint64_t *d_sizes, void *stream)
{
    if (!ws || !d_in || !d_out) return LSCOMP_ERR_ARG;
    // the stream is written in 4-byte words
    if (reinterpret_cast<uintptr_t>(d_in) % sizeof(T) || reinterpret_cast<uintptr_t>(d_out) % 4u) return LSCOMP_ERR_ARG;
    EncArgs<T> a;
    int layout = 0;
    if (!make_geom(x, y, z, Elem<T>::kTileBlocks, a.g) || !make_codec(bins, pooling, sizeof(T) == 4, a.c, layout))
        return LSCOMP_ERR_ARG;
    if (cap < a.g.R) return LSCOMP_ERR_CAPACITY;
    cudaStream_t st = (cudaStream_t)stream;
    std::lock_guard<std::mutex> lk(ws->mu);
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != ws->device) cudaSetDevice(ws->device);
    int s = ws_prepare(ws, a.g.ntiles, st);
    if (!s) {
        a.in = d_in;
        a.out = d_out;
        a.cap = cap;
        a.ctl = ws->ctl;
        a.state = ws->state;
        a.epoch = ws->epoch;
        a.sizes_out = reinterpret_cast<unsigned long long *>(d_sizes);
        const bool pool = a.c.pool_min <= 64;
        switch (vec_class(d_in, z, sizeof(T))) {
        case 16: s = launch_enc_v<T, 16>(a, layout, pool, ws->sm_count, st); break;
        case 4: s = launch_enc_v<T, 4>(a, layout, pool, ws->sm_count, st); break;
        default:
            if (sizeof(T) == 2) s = launch_enc_v<T, 2>(a, layout, pool, ws->sm_count, st);
            else s = LSCOMP_ERR_ARG;
            break;
        }
    }
    if (prev != ws->device) cudaSetDevice(prev);
    return s;
}

template <typename T>
int compress_sync_t(lscomp_workspace *ws, const T *d_in, uint32_t x, uint32_t y, uint32_t z, const uint32_t bins[4],
                    float pooling, uint8_t *d_out, uint64_t cap, uint64_t *stream_len, uint64_t *ref_size,
                    void *stream)
{
    int s = compress_async_t<T>(ws, d_in, x, y, z, bins, pooling, d_out, cap, nullptr, stream);
    if (s) return s;
    std::lock_guard<std::mutex> lk(ws->mu);
    s = read_ctl(ws, (cudaStream_t)stream);
    if (s) return s;
    uint64_t nb = (uint64_t)x * ((y + 7) / 8) * ((z + 7) / 8);
    uint64_t total = ws->h_ctl->total;
    if (sizeof(T) == 4) total &= 0xffffffffull;  // the reference reports a 32-bit total for uint32
    if (stream_len) *stream_len = ws->h_ctl->stream_len;
    if (ref_size) *ref_size = total + nb;
    return LSCOMP_OK;
}

template <typename T>
int decompress_async_t(lscomp_workspace *ws, const uint8_t *d_in, uint64_t cmp_len, uint32_t x, uint32_t y,
                       uint32_t z, const uint32_t bins[4], float pooling, T *d_out, void *stream)
{
    if (!ws || !d_in || !d_out) return LSCOMP_ERR_ARG;
    // the stream is read in 4-byte words
    if (reinterpret_cast<uintptr_t>(d_out) % sizeof(T) || reinterpret_cast<uintptr_t>(d_in) % 4u) return LSCOMP_ERR_ARG;
    DecArgs<T> a;
    int layout = 0;
    if (!make_geom(x, y, z, Elem<T>::kTileBlocks, a.g) || !make_codec(bins, pooling, sizeof(T) == 4, a.c, layout))
        return LSCOMP_ERR_ARG;
    if (cmp_len < a.g.nb) return LSCOMP_ERR_CAPACITY;
    cudaStream_t st = (cudaStream_t)stream;
    std::lock_guard<std::mutex> lk(ws->mu);
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != ws->device) cudaSetDevice(ws->device);
    int s = ws_prepare(ws, a.g.ntiles, st);
    if (!s) {
        a.in = d_in;
        a.out = d_out;
        a.cap = cmp_len;
        a.ctl = ws->ctl;
        a.state = ws->state;
        a.tile_off = ws->state + ws->state_cap;
        a.epoch = ws->epoch;
        switch (vec_class(d_out, z, sizeof(T))) {
        case 16: s = launch_dec_t<T, 16>(a, ws->sm_count, st); break;
        case 4: s = launch_dec_t<T, 4>(a, ws->sm_count, st); break;
        default:
            if (sizeof(T) == 2) s = launch_dec_t<T, 2>(a, ws->sm_count, st);
            else s = LSCOMP_ERR_ARG;
            break;
        }
    }
    if (prev != ws->device) cudaSetDevice(prev);
    return s;
}

}  // namespace


extern "C" {

int lscomp_version(void) { return 100; }

const char *lscomp_status_string(int s)
{
    switch (s) {
    case LSCOMP_OK: return "ok";
    case LSCOMP_ERR_ARG: return "invalid argument";
    case LSCOMP_ERR_CAPACITY: return "buffer too small for the stream";
    case LSCOMP_ERR_CUDA: return "CUDA runtime error";
    case LSCOMP_ERR_TIMEOUT: return "bounded wait in kernel timed out";
    case LSCOMP_ERR_CORRUPT: return "stream inconsistent with the geometry";
    case LSCOMP_ERR_RANGE: return "value range not representable";
    case LSCOMP_ERR_NOMEM: return "out of memory";
    case LSCOMP_ERR_TOO_LARGE: return "stack too large for the fixed scratch area";
    default: return "unknown status";
    }
}

uint64_t lscomp_block_count(uint32_t x, uint32_t y, uint32_t z)
{
    return (uint64_t)x * ((y + 7) / 8) * ((z + 7) / 8);
}

uint64_t lscomp_max_stream_bytes_u16(uint32_t x, uint32_t y, uint32_t z)
{
    uint64_t nb = lscomp_block_count(x, y, z);
    return (nb + 3) / 4 * 4 + 128ull * nb;
}

uint64_t lscomp_max_stream_bytes_u32(uint32_t x, uint32_t y, uint32_t z)
{
    uint64_t nb = lscomp_block_count(x, y, z);
    return (nb + 3) / 4 * 4 + 248ull * nb;  // 31 planes of 8 bytes
}

uint64_t lscomp_launch_count(void) { return g_launches.load(); }

int lscomp_workspace_create(lscomp_workspace **out, int device)
{
    if (!out) return LSCOMP_ERR_ARG;
    *out = nullptr;
    int dev = device;
    if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return LSCOMP_ERR_CUDA;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(dev) != cudaSuccess) return LSCOMP_ERR_CUDA;
    lscomp_workspace *ws = new (std::nothrow) lscomp_workspace();
    if (!ws) return LSCOMP_ERR_NOMEM;
    ws->device = dev;
    int st = LSCOMP_OK;
    if (cudaDeviceGetAttribute(&ws->sm_count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) st = LSCOMP_ERR_CUDA;
    if (!st) st = cuda_status(cudaMalloc(&ws->ctl, sizeof(LaunchCtl)));
    if (!st) st = cuda_status(cudaMemset(ws->ctl, 0, sizeof(LaunchCtl)));
    if (!st) st = cuda_status(cudaMallocHost(&ws->h_ctl, sizeof(LaunchCtl)));
    cudaSetDevice(prev);
    if (st) {
        lscomp_workspace_destroy(ws);
        return st;
    }
    *out = ws;
    return LSCOMP_OK;
}

int lscomp_workspace_destroy(lscomp_workspace *ws)
{
    if (!ws) return LSCOMP_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(ws->device);
    if (ws->state) cudaFree(ws->state);
    if (ws->ctl) cudaFree(ws->ctl);
    if (ws->h_ctl) cudaFreeHost(ws->h_ctl);
    cudaSetDevice(prev);
    delete ws;
    return LSCOMP_OK;
}

int lscomp_workspace_check(lscomp_workspace *ws, void *stream)
{
    if (!ws) return LSCOMP_ERR_ARG;
    std::lock_guard<std::mutex> lk(ws->mu);
    return read_ctl(ws, (cudaStream_t)stream);
}

int lscomp_compress_u16_async(lscomp_workspace *ws, const uint16_t *d_in, uint32_t x, uint32_t y, uint32_t z,
                              const uint32_t bins[4], float pooling, uint8_t *d_out, uint64_t cap,
                              uint64_t *d_sizes, void *stream)
{
    return compress_async_t<uint16_t>(ws, d_in, x, y, z, bins, pooling, d_out, cap, d_sizes, stream);
}

int lscomp_compress_u32_async(lscomp_workspace *ws, const uint32_t *d_in, uint32_t x, uint32_t y, uint32_t z,
                              const uint32_t bins[4], float pooling, uint8_t *d_out, uint64_t cap,
                              uint64_t *d_sizes, void *stream)
{
    return compress_async_t<uint32_t>(ws, d_in, x, y, z, bins, pooling, d_out, cap, d_sizes, stream);
}

int lscomp_compress_u16(lscomp_workspace *ws, const uint16_t *d_in, uint32_t x, uint32_t y, uint32_t z,
                        const uint32_t bins[4], float pooling, uint8_t *d_out, uint64_t cap,
                        uint64_t *stream_len, uint64_t *ref_size, void *stream)
{
    return compress_sync_t<uint16_t>(ws, d_in, x, y, z, bins, pooling, d_out, cap, stream_len, ref_size, stream);
}

int lscomp_compress_u32(lscomp_workspace *ws, const uint32_t *d_in, uint32_t x, uint32_t y, uint32_t z,
                        const uint32_t bins[4], float pooling, uint8_t *d_out, uint64_t cap,
                        uint64_t *stream_len, uint64_t *ref_size, void *stream)
{
    return compress_sync_t<uint32_t>(ws, d_in, x, y, z, bins, pooling, d_out, cap, stream_len, ref_size, stream);
}

int lscomp_decompress_u16_async(lscomp_workspace *ws, const uint8_t *d_in, uint64_t cmp_len, uint32_t x,
                                uint32_t y, uint32_t z, const uint32_t bins[4], float pooling, uint16_t *d_out,
                                void *stream)
{
    return decompress_async_t<uint16_t>(ws, d_in, cmp_len, x, y, z, bins, pooling, d_out, stream);
}

int lscomp_decompress_u32_async(lscomp_workspace *ws, const uint8_t *d_in, uint64_t cmp_len, uint32_t x,
                                uint32_t y, uint32_t z, const uint32_t bins[4], float pooling, uint32_t *d_out,
                                void *stream)
{
    return decompress_async_t<uint32_t>(ws, d_in, cmp_len, x, y, z, bins, pooling, d_out, stream);
}

int lscomp_decompress_u16(lscomp_workspace *ws, const uint8_t *d_in, uint64_t cmp_len, uint32_t x, uint32_t y,
                          uint32_t z, const uint32_t bins[4], float pooling, uint16_t *d_out, void *stream)
{
    int s = decompress_async_t<uint16_t>(ws, d_in, cmp_len, x, y, z, bins, pooling, d_out, stream);
    if (s) return s;
    std::lock_guard<std::mutex> lk(ws->mu);
    return read_ctl(ws, (cudaStream_t)stream);
}

int lscomp_decompress_u32(lscomp_workspace *ws, const uint8_t *d_in, uint64_t cmp_len, uint32_t x, uint32_t y,
                          uint32_t z, const uint32_t bins[4], float pooling, uint32_t *d_out, void *stream)
{
    int s = decompress_async_t<uint32_t>(ws, d_in, cmp_len, x, y, z, bins, pooling, d_out, stream);
    if (s) return s;
    std::lock_guard<std::mutex> lk(ws->mu);
    return read_ctl(ws, (cudaStream_t)stream);
}

}  // extern "C"

// ---------------------------------------------------------------- allocation-free compression
// lscomp_compress_u16_noalloc: the uint16 encoder with its scan scratch (the
// launch control block and one look-back word per tile) taken from a
// file-scope device array instead of a workspace allocation.
//
// Who needs it: callers that must not allocate device memory at call time --
// for example detector acquisition loops that run with a fixed, pre-reserved
// memory budget (a cudaMalloc there can fail once the budget is used up, and
// it synchronises the device in the middle of a streaming pipeline), or
// processes in which another allocator already owns the device memory.  The
// caller still provides the input and the output buffers; nothing else is
// allocated: no cudaMalloc, no cudaFree, no library allocator.
//
// Limits and sharing: the array is kNoAllocScratchBytes per device, held by
// every GPU that loads this library until the process exits.  It bounds the
// stack to kNoAllocMaxTiles tiles (about 67 M 8x8 blocks for 16-bit data);
// larger stacks are refused with LSCOMP_ERR_TOO_LARGE before any GPU work.
// All calls on a device share the one array, which keeps the previous call's
// contents: the control block is cleared on every call (cudaMemsetAsync,
// which allocates nothing), and the look-back words carry a per-call epoch so
// stale ones are never mistaken for fresh.  Calls that overlap on the GPU
// race on the shared array; this function serialises its own calls within a
// process and returns only after its kernel has finished.  The first call on
// a device looks up the array's device address (cudaGetSymbolAddress) with
// that device current; make that first call before any stream capture.
namespace {
constexpr size_t kNoAllocScratchBytes = 2u << 20;  // 2 MiB per device
constexpr size_t kNoAllocCtlBytes = 256;           // LaunchCtl, padded
constexpr uint64_t kNoAllocMaxTiles = (kNoAllocScratchBytes - kNoAllocCtlBytes) / sizeof(unsigned long long);
constexpr int kNoAllocMaxDevices = 64;
static_assert(sizeof(LaunchCtl) <= kNoAllocCtlBytes, "control block fits its slot");
}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {
struct NoAllocDevice {
    unsigned char *scratch = nullptr;  // device address of g_noalloc_scratch on this device
    int sm_count = 0;
    uint32_t epoch = 0;
};
std::mutex g_noalloc_mu;
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];
}  // namespace

extern "C" int lscomp_compress_u16_noalloc(const uint16_t *d_in, uint32_t x, uint32_t y, uint32_t z,
                                           const uint32_t bins[4], float pooling, uint8_t *d_out, uint64_t cap,
                                           uint64_t *stream_len, uint64_t *ref_size, void *stream)
{
    if (!d_in || !d_out) return LSCOMP_ERR_ARG;
    if (reinterpret_cast<uintptr_t>(d_in) % 2u || reinterpret_cast<uintptr_t>(d_out) % 4u) return LSCOMP_ERR_ARG;
    EncArgs<uint16_t> a;
    int layout = 0;
    if (!make_geom(x, y, z, Elem<uint16_t>::kTileBlocks, a.g) || !make_codec(bins, pooling, false, a.c, layout))
        return LSCOMP_ERR_ARG;
    if (a.g.ntiles > kNoAllocMaxTiles) return LSCOMP_ERR_TOO_LARGE;
    if (cap < a.g.R) return LSCOMP_ERR_CAPACITY;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) return LSCOMP_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;

    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    NoAllocDevice &d = g_noalloc_dev[dev];
    if (!d.scratch) {
        // one-time set-up on this device, with the device current: the host
        // symbol is only a stand-in, the kernel needs the device address
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_status(e);
        if (cudaDeviceGetAttribute(&d.sm_count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return LSCOMP_ERR_CUDA;
        d.scratch = static_cast<unsigned char *>(p);
    }
    unsigned long long *state = reinterpret_cast<unsigned long long *>(d.scratch + kNoAllocCtlBytes);
    if (d.epoch >= kEpochMax) {
        // epochs wrapped: clear the look-back words once
        cudaError_t e = cudaMemsetAsync(state, 0, kNoAllocMaxTiles * sizeof(unsigned long long), st);
        if (e != cudaSuccess) return cuda_status(e);
        d.epoch = 0;
    }
    d.epoch++;
    cudaError_t e = cudaMemsetAsync(d.scratch, 0, sizeof(LaunchCtl), st);
    if (e != cudaSuccess) return cuda_status(e);

    a.in = d_in;
    a.out = d_out;
    a.cap = cap;
    a.ctl = reinterpret_cast<LaunchCtl *>(d.scratch);
    a.state = state;
    a.epoch = d.epoch;
    a.sizes_out = nullptr;
    const bool pool = a.c.pool_min <= 64;
    int s;
    switch (vec_class(d_in, z, 2)) {
    case 16: s = launch_enc_v<uint16_t, 16>(a, layout, pool, d.sm_count, st); break;
    case 4: s = launch_enc_v<uint16_t, 4>(a, layout, pool, d.sm_count, st); break;
    default: s = launch_enc_v<uint16_t, 2>(a, layout, pool, d.sm_count, st); break;
    }
    if (s) return s;
    LaunchCtl h;  // plain host memory: the copy allocates nothing
    e = cudaMemcpyAsync(&h, d.scratch, sizeof(LaunchCtl), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_status(e);
    s = dev_status(h.error);
    if (s) return s;
    if (stream_len) *stream_len = h.stream_len;
    if (ref_size) *ref_size = h.total + a.g.nb;
    return LSCOMP_OK;
}
