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
#include "codec_host.h"

using namespace lsc;

using namespace lsc_host;

namespace {


template <typename T>
int compress_async_t(lscomp_workspace *ws, const T *d_in, uint32_t x, uint32_t y, uint32_t z, const uint32_t bins[4],
                     float pooling, uint8_t *d_out, uint64_t cap, uint64_t *d_sizes, void *stream)
{
    if (!ws || !d_in || !d_out) return LSCOMP_ERR_ARG;
    // the stream is written in 4-byte words
    if (reinterpret_cast<uintptr_t>(d_in) % sizeof(T) || reinterpret_cast<uintptr_t>(d_out) % 4u) return LSCOMP_ERR_ARG;
    Geom g0;
    Codec c;
    int layout = 0;
    if (!make_geom(x, y, z, Elem<T>::kTileBlocks, g0) || !make_codec(bins, pooling, sizeof(T) == 4, c, layout))
        return LSCOMP_ERR_ARG;
    if (cap < g0.R) return LSCOMP_ERR_CAPACITY;
    const int vec = vec_class(d_in, z, sizeof(T));
    if (sizeof(T) == 4 && vec == 2) return LSCOMP_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    std::lock_guard<std::mutex> lk(ws->mu);
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != ws->device) cudaSetDevice(ws->device);
    const bool pool = c.pool_min <= 64;
    // one complete call with configuration cfg (the tuner runs it too)
    auto run = [&](const TuneCfg &cfg) -> int {
        EncArgs<T> a = {};
        make_geom(x, y, z, cfg.tile_blocks, a.g);
        int s = ws_prepare(ws, a.g.ntiles, st);
        if (s) return s;
        a.c = c;
        a.in = d_in;
        a.out = d_out;
        a.cap = cap;
        a.ctl = ws->ctl;
        a.state = ws->state;
        a.epoch = ws->epoch;
        a.sizes_out = reinterpret_cast<unsigned long long *>(d_sizes);
        return launch_enc_any<T, false>(a, vec, layout, pool, cfg.shape, ws->sm_count, st);
    };
    const TuneKey key{(uint8_t)sizeof(T), (uint8_t)layout, (uint8_t)pool, kTuneCompress, (uint8_t)vec, g0.bzb};
    const bool may_tune = g0.ntiles >= (uint64_t)kTuneMinTilesPerSm * ws->sm_count;
    const TuneCfg cfg = tune_choose(ws, key, TuneCfg{-1, (uint32_t)Elem<T>::kTileBlocks}, may_tune, st, run);
    const int s = run(cfg);
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
    Geom g0;
    Codec c;
    int layout = 0;
    if (!make_geom(x, y, z, Elem<T>::kTileBlocks, g0) || !make_codec(bins, pooling, sizeof(T) == 4, c, layout))
        return LSCOMP_ERR_ARG;
    if (cmp_len < g0.nb) return LSCOMP_ERR_CAPACITY;
    const int vec = vec_class(d_out, z, sizeof(T));
    if (sizeof(T) == 4 && vec == 2) return LSCOMP_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    std::lock_guard<std::mutex> lk(ws->mu);
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != ws->device) cudaSetDevice(ws->device);
    auto run = [&](const TuneCfg &cfg) -> int {
        DecArgs<T> a = {};
        make_geom(x, y, z, cfg.tile_blocks, a.g);
        int s = ws_prepare(ws, a.g.ntiles, st);
        if (s) return s;
        a.c = c;
        a.in = d_in;
        a.out = d_out;
        a.cap = cmp_len;
        a.ctl = ws->ctl;
        a.state = ws->state;
        a.tile_off = ws->state + ws->state_cap;
        a.epoch = ws->epoch;
        switch (vec) {
        case 16: return launch_dec_t<T, 16>(a, ws->sm_count, st);
        case 4: return launch_dec_t<T, 4>(a, ws->sm_count, st);
        default:
            if constexpr (sizeof(T) == 2) return launch_dec_t<T, 2>(a, ws->sm_count, st);
            return LSCOMP_ERR_ARG;
        }
    };
    const TuneKey key{(uint8_t)sizeof(T), (uint8_t)layout, (uint8_t)(c.pool_min <= 64), kTuneDecompress, (uint8_t)vec,
                      g0.bzb};
    const bool may_tune = g0.ntiles >= (uint64_t)kTuneMinTilesPerSm * ws->sm_count;
    const TuneCfg cfg = tune_choose(ws, key, TuneCfg{-1, (uint32_t)Elem<T>::kTileBlocks}, may_tune, st, run);
    const int s = run(cfg);
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
    pipe_destroy(ws);
    if (ws->state) cudaFree(ws->state);
    if (ws->ctl) cudaFree(ws->ctl);
    if (ws->h_ctl) cudaFreeHost(ws->h_ctl);
    if (ws->d_stacks) cudaFree(ws->d_stacks);
    if (ws->h_stacks) cudaFreeHost(ws->h_stacks);
    if (ws->d_bsizes) cudaFree(ws->d_bsizes);
    if (ws->h_bsizes) cudaFreeHost(ws->h_bsizes);
    if (ws->d_tile_stack) cudaFree(ws->d_tile_stack);
    cudaSetDevice(prev);
    delete ws;
    return LSCOMP_OK;
}

int lscomp_workspace_set_tuning(lscomp_workspace *ws, int allow)
{
    if (!ws) return LSCOMP_ERR_ARG;
    std::lock_guard<std::mutex> lk(ws->mu);
    ws->no_tune = allow == 0;
    return LSCOMP_OK;
}

int lscomp_workspace_stall_next(lscomp_workspace *ws, uint64_t wait_ns)
{
    if (!ws || wait_ns < 1000000ull || wait_ns > 2000000000ull) return LSCOMP_ERR_ARG;
    std::lock_guard<std::mutex> lk(ws->mu);
    ws->stall_wait_ns = wait_ns;
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
    EncArgs<uint16_t> a = {};
    int layout = 0;
    if (!make_geom(x, y, z, Elem<uint16_t>::kTileBlocks, a.g) || !make_codec(bins, pooling, false, a.c, layout))
        return LSCOMP_ERR_ARG;
    if (a.g.ntiles > kNoAllocMaxTiles) return LSCOMP_ERR_TOO_LARGE;
    const bool pool = a.c.pool_min <= 64;
    const int vec = vec_class(d_in, z, 2);
    // a configuration the tuner chose for this key earlier is used when its
    // tiles fit the scratch area; no tuning runs here
    TuneCfg cfg{-1, (uint32_t)Elem<uint16_t>::kTileBlocks};
    {
        TuneCfg t;
        Geom gt;
        const TuneKey key{2, (uint8_t)layout, (uint8_t)pool, kTuneCompress, (uint8_t)vec, a.g.bzb};
        if (tune_lookup(key, t) && make_geom(x, y, z, t.tile_blocks, gt) && gt.ntiles <= kNoAllocMaxTiles) {
            cfg = t;
            a.g = gt;
        }
    }
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
    int s = launch_enc_any<uint16_t, false>(a, vec, layout, pool, cfg.shape, d.sm_count, st);
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
