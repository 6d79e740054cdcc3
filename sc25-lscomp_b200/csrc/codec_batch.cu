// codec_batch.cu -- batch compression (include/lscomp.h,
// lscomp_compress_batch_u16 / _u32): many stacks of any shapes in one
// persistent launch of the encoder.
//
// The stacks' tiles are numbered one after the other (stack order) and
// claimed from one ticket counter, so every SM stays busy however small the
// stacks are; a tile's look-back state is indexed by its number in the
// batch, and the first tile of each stack publishes an inclusive prefix at
// once, so no look-back walk crosses into the previous stack.  Each stack's
// stream is exactly the one lscomp_compress_u16/_u32 writes for it alone.
#include <string.h>
#include <algorithm>
#include <mutex>
#include <vector>
#include "codec_host.h"

using namespace lsc;
using namespace lsc_host;

namespace {

// The stack of every tile of the batch: one CTA per stack.
__global__ void tile_stack_kernel(const BatchStack *stacks, uint32_t n, uint32_t *map)
{
    for (uint32_t s = blockIdx.x; s < n; s += gridDim.x) {
        const unsigned long long t0 = stacks[s].tile0, nt = stacks[s].g.ntiles;
        for (unsigned long long t = threadIdx.x; t < nt; t += blockDim.x) map[t0 + t] = s;
    }
}

// Grow the workspace's batch buffers (only when a batch is larger than any
// before it on this workspace).
int batch_reserve(lscomp_workspace *ws, uint32_t n, uint64_t ntiles, cudaStream_t st)
{
    if (n > ws->stacks_cap) {
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_status(e);
        if (ws->d_stacks) cudaFree(ws->d_stacks);
        if (ws->h_stacks) cudaFreeHost(ws->h_stacks);
        if (ws->d_bsizes) cudaFree(ws->d_bsizes);
        if (ws->h_bsizes) cudaFreeHost(ws->h_bsizes);
        ws->d_stacks = nullptr;
        ws->h_stacks = nullptr;
        ws->d_bsizes = ws->h_bsizes = nullptr;
        ws->stacks_cap = 0;
        const uint32_t cap = n + n / 4 + 16;
        e = cudaMalloc(&ws->d_stacks, cap * sizeof(BatchStack));
        if (e == cudaSuccess) e = cudaMallocHost(&ws->h_stacks, cap * sizeof(BatchStack));
        if (e == cudaSuccess) e = cudaMalloc(&ws->d_bsizes, 2ull * cap * sizeof(unsigned long long));
        if (e == cudaSuccess) e = cudaMallocHost(&ws->h_bsizes, 2ull * cap * sizeof(unsigned long long));
        if (e != cudaSuccess) return cuda_status(e);
        ws->stacks_cap = cap;
    }
    if (ntiles > ws->tile_stack_cap) {
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_status(e);
        if (ws->d_tile_stack) cudaFree(ws->d_tile_stack);
        ws->d_tile_stack = nullptr;
        ws->tile_stack_cap = 0;
        const uint64_t cap = ntiles + ntiles / 4 + 1024;
        e = cudaMalloc(&ws->d_tile_stack, cap * sizeof(uint32_t));
        if (e != cudaSuccess) return cuda_status(e);
        ws->tile_stack_cap = cap;
    }
    return LSCOMP_OK;
}

// Per-stack geometry with tiles of at most tile_blocks blocks and each
// stack's first tile over the batch; false if a stack's dims are invalid.
inline bool batch_geoms(const lscomp_stack *stacks, uint32_t n, uint32_t tile_blocks, std::vector<Geom> &geom,
                        std::vector<unsigned long long> &tile0, unsigned long long &total)
{
    geom.resize(n);
    tile0.resize(n);
    total = 0;
    for (uint32_t s = 0; s < n; s++) {
        if (!make_geom(stacks[s].x, stacks[s].y, stacks[s].z, tile_blocks, geom[s])) return false;
        tile0[s] = total;
        total += geom[s].ntiles;
    }
    return true;
}

// Per-stack codecs (per_stack: bins[4 s .. 4 s + 3] and pooling[s] for stack
// s; else bins[0..3] and pooling[0] for all) and the bins layout and pooling
// flag one launch must be instantiated for to serve all of them: a common
// layout if there is one, else the increasing-bins kernel when every stack's
// bins increase (lossless and equal bins are special cases of it), else the
// general one.
inline bool batch_codecs(const uint32_t *bins, const float *pooling, bool per_stack, uint32_t n, bool wide,
                         std::vector<Codec> &codec, int &layout, bool &pool)
{
    if (!bins || !pooling) return false;
    codec.resize(n);
    layout = -1;
    bool mono = true;
    pool = false;
    for (uint32_t s = 0; s < n; s++) {
        int l = 0;
        if (per_stack || s == 0) {
            if (!make_codec(bins + (per_stack ? 4ull * s : 0), pooling[per_stack ? s : 0], wide, codec[s], l)) return false;
        } else {
            codec[s] = codec[0];
            l = layout;
        }
        if (s == 0) layout = l;
        else if (l != layout) layout = -2;  // mixed
        if (l == BINS_GENERAL) mono = false;
        if (codec[s].pool_min <= 64) pool = true;
    }
    if (layout == -2) layout = mono ? BINS_MONO : BINS_GENERAL;
    return true;
}

template <typename T>
int compress_batch_t(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t *bins,
                     const float *pooling, bool per_stack, uint64_t *stream_len, uint64_t *ref_size, void *stream)
{
    if (!ws || (n && !stacks)) return LSCOMP_ERR_ARG;
    if (n == 0) return LSCOMP_OK;
    std::vector<Codec> codec;
    int layout = 0;
    bool pool = false;
    if (!batch_codecs(bins, pooling, per_stack, n, sizeof(T) == 4, codec, layout, pool)) return LSCOMP_ERR_ARG;
    const Codec &c = codec[0];
    // every stack checked as lscomp_compress_* checks it; the narrowest
    // row access any stack allows is used for all
    std::vector<Geom> geom;
    std::vector<unsigned long long> tile0;
    unsigned long long total = 0;
    int vec = 16;
    for (uint32_t s = 0; s < n; s++) {
        const lscomp_stack &q = stacks[s];
        if (!q.d_in || !q.d_out) return LSCOMP_ERR_ARG;
        if (reinterpret_cast<uintptr_t>(q.d_in) % sizeof(T) || reinterpret_cast<uintptr_t>(q.d_out) % 4u)
            return LSCOMP_ERR_ARG;
        Geom g;
        if (!make_geom(q.x, q.y, q.z, Elem<T>::kTileBlocks, g)) return LSCOMP_ERR_ARG;
        if (q.cap < g.R) return LSCOMP_ERR_CAPACITY;
        const int v = vec_class(q.d_in, q.z, sizeof(T));
        if (sizeof(T) == 4 && v == 2) return LSCOMP_ERR_ARG;
    }
    // every stack is read with its own row access width (Geom::vec); the
    // launch is instantiated once for all widths
    vec = sizeof(T) == 2 ? 2 : 4;
    cudaStream_t st = (cudaStream_t)stream;
    std::lock_guard<std::mutex> lk(ws->mu);
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != ws->device) cudaSetDevice(ws->device);
    // one complete call with configuration cfg.  The descriptors are rebuilt
    // only when the tile size changes; the tuner synchronises the stream
    // before it changes configuration, so no pending copy reads the pinned
    // descriptors while they are rewritten.
    uint32_t built = 0;
    auto run = [&](const TuneCfg &cfg) -> int {
        int r = LSCOMP_OK;
        if (cfg.tile_blocks != built) {
            if (!batch_geoms(stacks, n, cfg.tile_blocks, geom, tile0, total)) return LSCOMP_ERR_ARG;
            r = batch_reserve(ws, n, total, st);
            if (r) return r;
            for (uint32_t s = 0; s < n; s++) {
                BatchStack &b = ws->h_stacks[s];
                b.g = geom[s];
                b.g.vec = (uint32_t)vec_class(stacks[s].d_in, stacks[s].z, sizeof(T));
                b.c = codec[s];
                b.in = stacks[s].d_in;
                b.out = stacks[s].d_out;
                b.cap = stacks[s].cap;
                b.tile0 = tile0[s];
                b.sizes = ws->d_bsizes + 2ull * s;
            }
            r = cuda_status(
                cudaMemcpyAsync(ws->d_stacks, ws->h_stacks, n * sizeof(BatchStack), cudaMemcpyHostToDevice, st));
            if (r) return r;
            const uint32_t grid = n < 4096u ? n : 4096u;
            tile_stack_kernel<<<grid, 256, 0, st>>>(ws->d_stacks, n, ws->d_tile_stack);
            g_launches.fetch_add(1);
            r = cuda_status(cudaGetLastError());
            if (r) return r;
            built = cfg.tile_blocks;
        }
        r = ws_prepare(ws, total, st);
        if (r) return r;
        EncArgs<T> a;
        memset(&a, 0, sizeof(a));
        a.g = geom[0];  // not read by batch launches
        a.c = c;
        a.ctl = ws->ctl;
        a.state = ws->state;
        a.epoch = ws->epoch;
        a.stacks = ws->d_stacks;
        a.tile_stack = ws->d_tile_stack;
        a.ntiles_all = total;
        return launch_enc_any<T, true>(a, vec, layout, pool, cfg.shape, ws->sm_count, st);
    };
    const TuneKey key{(uint8_t)sizeof(T), (uint8_t)layout, (uint8_t)pool, kTuneBatch, (uint8_t)vec, 0};
    const TuneCfg cfg = tune_choose(ws, key, TuneCfg{-1, (uint32_t)Elem<T>::kTileBlocks}, true, st, run);
    int r = run(cfg);
    if (!r)
        r = cuda_status(cudaMemcpyAsync(ws->h_bsizes, ws->d_bsizes, 2ull * n * sizeof(unsigned long long),
                                        cudaMemcpyDeviceToHost, st));
    if (!r) r = read_ctl(ws, st);  // synchronises the stream
    if (!r) {
        for (uint32_t s = 0; s < n; s++) {
            uint64_t total_s = ws->h_bsizes[2ull * s + 1];
            if (sizeof(T) == 4) total_s &= 0xffffffffull;  // the reference reports a 32-bit total for uint32
            if (stream_len) stream_len[s] = ws->h_bsizes[2ull * s];
            if (ref_size) ref_size[s] = total_s + geom[s].nb;
        }
    }
    if (prev != ws->device) cudaSetDevice(prev);
    return r;
}

// ---------------------------------------------------------------- stream sizes
// The exact stream length of every stack of a batch without writing any
// stream: pass A of the encoder (every block's header byte, the same
// block_header as enc_compute, so the same sizes) summed per stack.  One CTA
// per tile at a time, rows read straight from global memory with each
// stack's row access width; a tile's sum goes to its stack's counter with
// one atomic add.
template <typename T, int BINS, bool POOL>
__global__ void __launch_bounds__(kThreads) size_kernel(const BatchStack *stacks, const uint32_t *tile_stack,
                                                        unsigned long long ntiles, unsigned long long *payload,
                                                        LaunchCtl *ctl)
{
    __shared__ BatchStack bs;
    __shared__ uint32_t sum_s, bad_s, stk_s;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5, jb = lane & 7u, r = lane >> 3;
    for (unsigned long long gt = blockIdx.x; gt < ntiles; gt += gridDim.x) {
        if (tid == 0) {
            stk_s = tile_stack[gt];
            bs = stacks[stk_s];
            sum_s = 0;
            bad_s = 0;
        }
        __syncthreads();
        const Geom &g = bs.g;
        const TileInfo ti = tile_info(g, gt - bs.tile0);
        const T *in = static_cast<const T *>(bs.in);
        const uint32_t nunits = (ti.nblk + 7u) >> 3;
        uint32_t sum = 0, bad = 0;
        for (uint32_t u = warp; u < nunits; u += kWarps) {
            const uint32_t b = u * 8u + jb;
            const bool active = b < ti.nblk;
            const unsigned long long rho = g.chunked ? ti.rho0 : ti.rho0 + (active ? b / g.bzb : 0u);
            const uint32_t bz = g.chunked ? ti.c0 + b : (active ? b % g.bzb : 0u);
            uint32_t nrows;
            const unsigned long long e0 = (brow_start(g, rho, nrows) + r) * g.Z + 8ull * bz;
            const uint32_t left = g.Z - 8u * bz, ncols = left < 8u ? left : 8u;
            Row<T> A, B;
#pragma unroll
            for (int i = 0; i < Elem<T>::kWords; i++) A.w[i] = B.w[i] = 0;
            for (uint32_t half = 0; half < 2u; half++) {
                Row<T> &v = half ? B : A;
                if (!active || r + 4u * half >= nrows) continue;
                const T *p = in + e0 + 4ull * half * g.Z;
                if (g.vec == 16) load_cols<T, 16>(p, ncols, v);
                else if (sizeof(T) == 4 || g.vec == 4) load_cols<T, 4>(p, ncols, v);
                else load_cols<T, 2>(p, ncols, v);
            }
            uint32_t rb;
            const uint32_t h =
                block_header<T, BINS == BINS_IDENT ? BINS_EQUAL : BINS, POOL, BINS == BINS_IDENT>(A, B, bs.c, rb);
            if (active && r == 0) {
                sum += (h & 0x1fu) << (3u - ((h >> 7) & 1u));  // rate planes of 8 bytes, or 4 when pooled
                bad |= rb;
            }
        }
        sum = __reduce_add_sync(0xffffffffu, sum);
        bad = __reduce_or_sync(0xffffffffu, bad);
        if (lane == 0) {
            atomicAdd(&sum_s, sum);
            atomicOr(&bad_s, bad);
        }
        __syncthreads();
        if (tid == 0) {
            atomicAdd(&payload[stk_s], (unsigned long long)sum_s);
            if (bad_s) raise_error(ctl, DEV_ERR_RANGE);
        }
        __syncthreads();
    }
}

template <typename T, int BINS>
void launch_size_p(bool pool, unsigned grid, const BatchStack *stacks, const uint32_t *map, unsigned long long ntiles,
                   unsigned long long *payload, LaunchCtl *ctl, cudaStream_t st)
{
    if (pool) size_kernel<T, BINS, true><<<grid, kThreads, 0, st>>>(stacks, map, ntiles, payload, ctl);
    else size_kernel<T, BINS, false><<<grid, kThreads, 0, st>>>(stacks, map, ntiles, payload, ctl);
}

template <typename T>
int stream_sizes_t(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t *bins,
                   const float *pooling, uint64_t *stream_len, void *stream)
{
    if (!ws || !stream_len || (n && !stacks)) return LSCOMP_ERR_ARG;
    if (n == 0) return LSCOMP_OK;
    std::vector<Codec> codec;
    int layout = 0;
    bool pool = false;
    if (!batch_codecs(bins, pooling, true, n, sizeof(T) == 4, codec, layout, pool)) return LSCOMP_ERR_ARG;
    std::vector<Geom> geom;
    std::vector<unsigned long long> tile0;
    unsigned long long total = 0;
    if (!batch_geoms(stacks, n, Elem<T>::kTileBlocks, geom, tile0, total)) return LSCOMP_ERR_ARG;
    for (uint32_t s = 0; s < n; s++) {
        if (!stacks[s].d_in || reinterpret_cast<uintptr_t>(stacks[s].d_in) % sizeof(T)) return LSCOMP_ERR_ARG;
        geom[s].vec = (uint32_t)vec_class(stacks[s].d_in, stacks[s].z, sizeof(T));
    }
    cudaStream_t st = (cudaStream_t)stream;
    std::lock_guard<std::mutex> lk(ws->mu);
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != ws->device) cudaSetDevice(ws->device);
    int r = batch_reserve(ws, n, total, st);
    if (!r) r = ws_prepare(ws, 1, st);  // clears the control block
    if (!r) {
        for (uint32_t s = 0; s < n; s++) {
            BatchStack &b = ws->h_stacks[s];
            memset(&b, 0, sizeof(b));
            b.g = geom[s];
            b.c = codec[s];
            b.in = stacks[s].d_in;
            b.tile0 = tile0[s];
        }
        r = cuda_status(cudaMemcpyAsync(ws->d_stacks, ws->h_stacks, n * sizeof(BatchStack), cudaMemcpyHostToDevice, st));
    }
    if (!r) r = cuda_status(cudaMemsetAsync(ws->d_bsizes, 0, n * sizeof(unsigned long long), st));
    if (!r) {
        const uint32_t mgrid = n < 4096u ? n : 4096u;
        tile_stack_kernel<<<mgrid, 256, 0, st>>>(ws->d_stacks, n, ws->d_tile_stack);
        g_launches.fetch_add(1);
        r = cuda_status(cudaGetLastError());
    }
    if (!r) {
        unsigned long long grid = (unsigned long long)ws->sm_count * 8;
        if (grid > total) grid = total;
        const unsigned gr = (unsigned)grid;
        switch (layout) {
        case BINS_IDENT: launch_size_p<T, BINS_IDENT>(pool, gr, ws->d_stacks, ws->d_tile_stack, total, ws->d_bsizes, ws->ctl, st); break;
        case BINS_EQUAL: launch_size_p<T, BINS_EQUAL>(pool, gr, ws->d_stacks, ws->d_tile_stack, total, ws->d_bsizes, ws->ctl, st); break;
        case BINS_MONO: launch_size_p<T, BINS_MONO>(pool, gr, ws->d_stacks, ws->d_tile_stack, total, ws->d_bsizes, ws->ctl, st); break;
        default: launch_size_p<T, BINS_GENERAL>(pool, gr, ws->d_stacks, ws->d_tile_stack, total, ws->d_bsizes, ws->ctl, st); break;
        }
        g_launches.fetch_add(1);
        r = cuda_status(cudaGetLastError());
    }
    if (!r)
        r = cuda_status(cudaMemcpyAsync(ws->h_bsizes, ws->d_bsizes, n * sizeof(unsigned long long),
                                        cudaMemcpyDeviceToHost, st));
    if (!r) r = read_ctl(ws, st);  // synchronises the stream
    if (!r)
        for (uint32_t s = 0; s < n; s++) stream_len[s] = geom[s].R + ws->h_bsizes[s];
    if (prev != ws->device) cudaSetDevice(prev);
    return r;
}

// ---------------------------------------------------------------- batch decompression
// Many streams decoded by three launches: the stack of every tile, the
// offsets kernel over every stack's segments, then one CTA per tile of every
// stack.  stacks[i]: d_in =
// stream, cap = its readable bytes, d_out = the decoded values (X*Y*Z of the
// call's type), bins[4 i ..] and pooling[i] its settings.
template <typename T>
int decompress_batch_t(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t *bins,
                       const float *pooling, void *stream)
{
    if (!ws || (n && (!stacks || !bins || !pooling))) return LSCOMP_ERR_ARG;
    if (n == 0) return LSCOMP_OK;
    std::vector<Codec> codec;
    int layout = 0;
    bool pool = false;
    if (!batch_codecs(bins, pooling, true, n, sizeof(T) == 4, codec, layout, pool)) return LSCOMP_ERR_ARG;
    std::vector<Geom> geom;
    std::vector<unsigned long long> tile0;
    unsigned long long total = 0;
    if (!batch_geoms(stacks, n, Elem<T>::kTileBlocks, geom, tile0, total)) return LSCOMP_ERR_ARG;
    int vec = 16;
    std::vector<unsigned long long> seg0(n + 1, 0);
    for (uint32_t s = 0; s < n; s++) {
        const lscomp_stack &q = stacks[s];
        if (!q.d_in || !q.d_out) return LSCOMP_ERR_ARG;
        // the stream is read in 4-byte words, the values stored as T
        if (reinterpret_cast<uintptr_t>(q.d_in) % 4u || reinterpret_cast<uintptr_t>(q.d_out) % sizeof(T))
            return LSCOMP_ERR_ARG;
        if (q.cap < geom[s].nb) return LSCOMP_ERR_CAPACITY;
        const int v = vec_class(q.d_out, q.z, sizeof(T));
        if (sizeof(T) == 4 && v == 2) return LSCOMP_ERR_ARG;
        geom[s].vec = (uint32_t)v;  // every stack is written with its own row access width
        seg0[s + 1] = seg0[s] + (geom[s].ntiles + kSegTiles - 1) / kSegTiles;
    }
    vec = sizeof(T) == 2 ? 2 : 4;
    if (total > 0x7fffffffull) return LSCOMP_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    std::lock_guard<std::mutex> lk(ws->mu);
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != ws->device) cudaSetDevice(ws->device);
    // look-back words: one per segment; tile offsets: ntiles + 1 per stack
    const unsigned long long need = std::max<unsigned long long>(seg0[n], total + n);
    int r = ws_prepare(ws, need, st);
    if (!r) r = batch_reserve(ws, n, total, st);
    if (!r) {
        for (uint32_t s = 0; s < n; s++) {
            BatchStack &b = ws->h_stacks[s];
            b.g = geom[s];
            b.c = codec[s];
            b.in = stacks[s].d_in;
            b.out = stacks[s].d_out;
            b.cap = stacks[s].cap;
            b.tile0 = tile0[s];
            b.sizes = nullptr;
        }
        for (uint32_t s = 0; s <= n; s++) ws->h_bsizes[s] = seg0[s];  // pinned staging of the segment table
        r = cuda_status(cudaMemcpyAsync(ws->d_stacks, ws->h_stacks, n * sizeof(BatchStack), cudaMemcpyHostToDevice, st));
        if (!r)
            r = cuda_status(cudaMemcpyAsync(ws->d_bsizes, ws->h_bsizes, (n + 1ull) * sizeof(unsigned long long),
                                            cudaMemcpyHostToDevice, st));
    }
    if (!r) {
        DecArgs<T> a;
        memset(&a, 0, sizeof(a));
        a.ctl = ws->ctl;
        a.state = ws->state;
        a.tile_off = ws->state + ws->state_cap;
        a.epoch = ws->epoch;
        a.stacks = ws->d_stacks;
        a.nstacks = n;
        a.seg0 = ws->d_bsizes;
        a.tile_stack = ws->d_tile_stack;
        const uint32_t mgrid = n < 4096u ? n : 4096u;
        tile_stack_kernel<<<mgrid, 256, 0, st>>>(ws->d_stacks, n, ws->d_tile_stack);
        g_launches.fetch_add(1);
        r = cuda_status(cudaGetLastError());
        unsigned long long grid = (unsigned long long)ws->sm_count * 4;
        if (grid > seg0[n]) grid = seg0[n];
        if (!r) {
            dec_offsets_batch_kernel<T><<<(unsigned)grid, kThreads, 0, st>>>(a);
            g_launches.fetch_add(1);
            r = cuda_status(cudaGetLastError());
        }
        if (!r) {
            switch (vec) {
            case 16: dec_kernel<T, 16, true><<<(unsigned)total, kThreads, 0, st>>>(a); break;
            case 4: dec_kernel<T, 4, true><<<(unsigned)total, kThreads, 0, st>>>(a); break;
            default:
                if constexpr (sizeof(T) == 2) dec_kernel<T, 2, true><<<(unsigned)total, kThreads, 0, st>>>(a);
                break;
            }
            g_launches.fetch_add(1);
            r = cuda_status(cudaGetLastError());
        }
    }
    if (!r) r = read_ctl(ws, st);  // synchronises the stream
    if (prev != ws->device) cudaSetDevice(prev);
    return r;
}

// the single-stack asynchronous call for one stack descriptor
template <typename T>
int compress_async_t_dispatch(lscomp_workspace *ws, const lscomp_stack &q, const uint32_t bins[4], float pooling,
                              void *stream)
{
    if constexpr (sizeof(T) == 2)
        return lscomp_compress_u16_async(ws, static_cast<const uint16_t *>(q.d_in), q.x, q.y, q.z, bins, pooling,
                                         q.d_out, q.cap, nullptr, stream);
    else
        return lscomp_compress_u32_async(ws, static_cast<const uint32_t *>(q.d_in), q.x, q.y, q.z, bins, pooling,
                                         q.d_out, q.cap, nullptr, stream);
}

// ---------------------------------------------------------------- graph plans
// A plan is one batch compression with everything fixed (the stacks'
// buffers and shapes, bins, pooling threshold, launch configuration),
// captured once as a CUDA graph: clear the control block and the look-back
// words, run the encoder, copy the per-stack sizes and the control block to
// pinned host memory.  A replay is one graph launch and one synchronisation;
// the host computes nothing per call.  The plan owns its scratch (look-back
// words at a fixed epoch, cleared by the graph itself), so plans and
// workspace calls do not share state.
struct PlanImpl {
    std::mutex mu;
    int device = 0;
    int es = 2;
    uint32_t n = 0;
    TuneCfg cfg{-1, 0};
    uint64_t ntiles = 0;
    std::vector<uint64_t> nb;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    LaunchCtl *ctl = nullptr, *h_ctl = nullptr;
    unsigned long long *state = nullptr;
    BatchStack *d_stacks = nullptr;
    uint32_t *d_tile_stack = nullptr;
    unsigned long long *d_sizes = nullptr, *h_sizes = nullptr;
};

void plan_free(PlanImpl *p)
{
    if (!p) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(p->device);
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    if (p->ctl) cudaFree(p->ctl);
    if (p->h_ctl) cudaFreeHost(p->h_ctl);
    if (p->state) cudaFree(p->state);
    if (p->d_stacks) cudaFree(p->d_stacks);
    if (p->d_tile_stack) cudaFree(p->d_tile_stack);
    if (p->d_sizes) cudaFree(p->d_sizes);
    if (p->h_sizes) cudaFreeHost(p->h_sizes);
    cudaSetDevice(prev);
    delete p;
}

constexpr uint32_t kPlanEpoch = 1;  // the graph clears the look-back words before every replay

template <typename T>
int plan_create_t(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t *bins,
                  const float *pooling, bool per_stack, void *stream, PlanImpl **out)
{
    if (!out) return LSCOMP_ERR_ARG;
    *out = nullptr;
    if (!ws || !stacks || n == 0 || !bins || !pooling) return LSCOMP_ERR_ARG;
    // one ordinary call first: it checks every argument, tunes the key when
    // tuning is on, and leaves the streams written
    int r = n == 1 ? compress_async_t_dispatch<T>(ws, stacks[0], bins, pooling[0], stream)
                   : compress_batch_t<T>(ws, stacks, n, bins, pooling, per_stack, nullptr, nullptr, stream);
    if (!r && n == 1) r = lscomp_workspace_check(ws, stream);
    if (r) return r;
    std::vector<Codec> codec;
    int layout = 0;
    bool pool = false;
    batch_codecs(bins, pooling, per_stack, n, sizeof(T) == 4, codec, layout, pool);
    const Codec &c = codec[0];
    // one stack: the single-stack kernel at the stack's row access width;
    // several: the batch kernel, every stack at its own width (Geom::vec)
    int vec = n == 1 ? vec_class(stacks[0].d_in, stacks[0].z, sizeof(T)) : (sizeof(T) == 2 ? 2 : 4);
    Geom g0;
    make_geom(stacks[0].x, stacks[0].y, stacks[0].z, Elem<T>::kTileBlocks, g0);
    TuneCfg cfg{-1, (uint32_t)Elem<T>::kTileBlocks};
    const TuneKey key{(uint8_t)sizeof(T), (uint8_t)layout, (uint8_t)pool, n == 1 ? kTuneCompress : kTuneBatch,
                      (uint8_t)vec, n == 1 ? g0.bzb : 0u};
    tune_lookup(key, cfg);

    PlanImpl *p = new (std::nothrow) PlanImpl();
    if (!p) return LSCOMP_ERR_NOMEM;
    p->device = ws->device;
    p->es = (int)sizeof(T);
    p->n = n;
    p->cfg = cfg;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(p->device);
    std::vector<Geom> geom;
    std::vector<unsigned long long> tile0;
    unsigned long long total = 0;
    batch_geoms(stacks, n, cfg.tile_blocks, geom, tile0, total);
    p->ntiles = total;
    p->nb.resize(n);
    for (uint32_t s = 0; s < n; s++) p->nb[s] = geom[s].nb;
    cudaStream_t cs = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&p->ctl, sizeof(LaunchCtl));
    if (e == cudaSuccess) e = cudaMallocHost(&p->h_ctl, sizeof(LaunchCtl));
    if (e == cudaSuccess) e = cudaMalloc(&p->state, total * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&p->d_sizes, 2ull * n * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMallocHost(&p->h_sizes, 2ull * n * sizeof(unsigned long long));
    if (e == cudaSuccess && n > 1) {
        std::vector<BatchStack> h(n);
        for (uint32_t s = 0; s < n; s++) {
            h[s].g = geom[s];
            h[s].g.vec = (uint32_t)vec_class(stacks[s].d_in, stacks[s].z, sizeof(T));
            h[s].c = codec[s];
            h[s].in = stacks[s].d_in;
            h[s].out = stacks[s].d_out;
            h[s].cap = stacks[s].cap;
            h[s].tile0 = tile0[s];
            h[s].sizes = p->d_sizes + 2ull * s;
        }
        e = cudaMalloc(&p->d_stacks, n * sizeof(BatchStack));
        if (e == cudaSuccess) e = cudaMalloc(&p->d_tile_stack, total * sizeof(uint32_t));
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(p->d_stacks, h.data(), n * sizeof(BatchStack), cudaMemcpyHostToDevice, cs);
        if (e == cudaSuccess) {
            const uint32_t grid = n < 4096u ? n : 4096u;
            tile_stack_kernel<<<grid, 256, 0, cs>>>(p->d_stacks, n, p->d_tile_stack);
            g_launches.fetch_add(1);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(cs);
    }
    r = cuda_status(e);
    if (!r) {
        EncArgs<T> a;
        memset(&a, 0, sizeof(a));
        a.g = geom[0];
        a.c = c;
        a.ctl = p->ctl;
        a.state = p->state;
        a.epoch = kPlanEpoch;
        if (n == 1) {
            a.in = static_cast<const T *>(stacks[0].d_in);
            a.out = stacks[0].d_out;
            a.cap = stacks[0].cap;
            a.sizes_out = p->d_sizes;
        } else {
            a.stacks = p->d_stacks;
            a.tile_stack = p->d_tile_stack;
            a.ntiles_all = total;
        }
        e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed);
        if (e == cudaSuccess) {
            cudaMemsetAsync(p->ctl, 0, sizeof(LaunchCtl), cs);
            cudaMemsetAsync(p->state, 0, total * sizeof(unsigned long long), cs);
            const int lr = n == 1 ? launch_enc_any<T, false>(a, vec, layout, pool, cfg.shape, ws->sm_count, cs)
                                  : launch_enc_any<T, true>(a, vec, layout, pool, cfg.shape, ws->sm_count, cs);
            cudaMemcpyAsync(p->h_sizes, p->d_sizes, 2ull * n * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            cs);
            cudaMemcpyAsync(p->h_ctl, p->ctl, sizeof(LaunchCtl), cudaMemcpyDeviceToHost, cs);
            e = cudaStreamEndCapture(cs, &p->graph);
            if (e == cudaSuccess && lr) e = cudaErrorLaunchFailure;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&p->exec, p->graph, 0);
        r = cuda_status(e);
    }
    if (cs) cudaStreamDestroy(cs);
    cudaSetDevice(prev);
    if (r) {
        plan_free(p);
        return r;
    }
    *out = p;
    return LSCOMP_OK;
}

int plan_run(PlanImpl *p, void *stream, uint64_t *stream_len, uint64_t *ref_size)
{
    if (!p) return LSCOMP_ERR_ARG;
    std::lock_guard<std::mutex> lk(p->mu);
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != p->device) cudaSetDevice(p->device);
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaGraphLaunch(p->exec, st);
    if (e == cudaSuccess) {
        g_launches.fetch_add(1);
        e = cudaStreamSynchronize(st);
    }
    int r = cuda_status(e);
    if (!r) r = dev_status(p->h_ctl->error);
    if (!r) {
        for (uint32_t s = 0; s < p->n; s++) {
            uint64_t total_s = p->h_sizes[2ull * s + 1];
            if (p->es == 4) total_s &= 0xffffffffull;  // the reference reports a 32-bit total for uint32
            if (stream_len) stream_len[s] = p->h_sizes[2ull * s];
            if (ref_size) ref_size[s] = total_s + p->nb[s];
        }
    }
    if (prev != p->device) cudaSetDevice(prev);
    return r;
}

}  // namespace

extern "C" {

int lscomp_compress_batch_u16(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t bins[4],
                              float pooling, uint64_t *stream_len, uint64_t *ref_size, void *stream)
{
    return compress_batch_t<uint16_t>(ws, stacks, n, bins, &pooling, false, stream_len, ref_size, stream);
}

int lscomp_compress_batch_u32(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t bins[4],
                              float pooling, uint64_t *stream_len, uint64_t *ref_size, void *stream)
{
    return compress_batch_t<uint32_t>(ws, stacks, n, bins, &pooling, false, stream_len, ref_size, stream);
}

int lscomp_compress_batch_ex_u16(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t *bins,
                                 const float *pooling, uint64_t *stream_len, uint64_t *ref_size, void *stream)
{
    return compress_batch_t<uint16_t>(ws, stacks, n, bins, pooling, true, stream_len, ref_size, stream);
}

int lscomp_compress_batch_ex_u32(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t *bins,
                                 const float *pooling, uint64_t *stream_len, uint64_t *ref_size, void *stream)
{
    return compress_batch_t<uint32_t>(ws, stacks, n, bins, pooling, true, stream_len, ref_size, stream);
}

int lscomp_stream_sizes_batch_u16(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t *bins,
                                  const float *pooling, uint64_t *stream_len, void *stream)
{
    return stream_sizes_t<uint16_t>(ws, stacks, n, bins, pooling, stream_len, stream);
}

int lscomp_stream_sizes_batch_u32(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t *bins,
                                  const float *pooling, uint64_t *stream_len, void *stream)
{
    return stream_sizes_t<uint32_t>(ws, stacks, n, bins, pooling, stream_len, stream);
}

int lscomp_decompress_batch_u16(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t *bins,
                                const float *pooling, void *stream)
{
    return decompress_batch_t<uint16_t>(ws, stacks, n, bins, pooling, stream);
}

int lscomp_decompress_batch_u32(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t *bins,
                                const float *pooling, void *stream)
{
    return decompress_batch_t<uint32_t>(ws, stacks, n, bins, pooling, stream);
}

int lscomp_plan_create_u16(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t bins[4],
                           float pooling, void *stream, lscomp_plan **plan)
{
    return plan_create_t<uint16_t>(ws, stacks, n, bins, &pooling, false, stream, reinterpret_cast<PlanImpl **>(plan));
}

int lscomp_plan_create_u32(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t bins[4],
                           float pooling, void *stream, lscomp_plan **plan)
{
    return plan_create_t<uint32_t>(ws, stacks, n, bins, &pooling, false, stream, reinterpret_cast<PlanImpl **>(plan));
}

int lscomp_plan_create_ex_u16(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t *bins,
                              const float *pooling, void *stream, lscomp_plan **plan)
{
    return plan_create_t<uint16_t>(ws, stacks, n, bins, pooling, true, stream, reinterpret_cast<PlanImpl **>(plan));
}

int lscomp_plan_create_ex_u32(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t *bins,
                              const float *pooling, void *stream, lscomp_plan **plan)
{
    return plan_create_t<uint32_t>(ws, stacks, n, bins, pooling, true, stream, reinterpret_cast<PlanImpl **>(plan));
}

int lscomp_plan_run(lscomp_plan *plan, void *stream, uint64_t *stream_len, uint64_t *ref_size)
{
    return plan_run(reinterpret_cast<PlanImpl *>(plan), stream, stream_len, ref_size);
}

int lscomp_plan_destroy(lscomp_plan *plan)
{
    plan_free(reinterpret_cast<PlanImpl *>(plan));
    return LSCOMP_OK;
}

}  // extern "C"
