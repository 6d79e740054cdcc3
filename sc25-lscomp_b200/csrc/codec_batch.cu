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

template <typename T>
int compress_batch_t(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t bins[4],
                     float pooling, uint64_t *stream_len, uint64_t *ref_size, void *stream)
{
    if (!ws || (n && !stacks)) return LSCOMP_ERR_ARG;
    if (n == 0) return LSCOMP_OK;
    Codec c;
    int layout = 0;
    if (!make_codec(bins, pooling, sizeof(T) == 4, c, layout)) return LSCOMP_ERR_ARG;
    // every stack checked as lscomp_compress_* checks it; the narrowest
    // row access any stack allows is used for all
    std::vector<Geom> geom(n);
    std::vector<unsigned long long> tile0(n);
    unsigned long long total = 0;
    int vec = 16;
    for (uint32_t s = 0; s < n; s++) {
        const lscomp_stack &q = stacks[s];
        if (!q.d_in || !q.d_out) return LSCOMP_ERR_ARG;
        if (reinterpret_cast<uintptr_t>(q.d_in) % sizeof(T) || reinterpret_cast<uintptr_t>(q.d_out) % 4u)
            return LSCOMP_ERR_ARG;
        if (!make_geom(q.x, q.y, q.z, Elem<T>::kTileBlocks, geom[s])) return LSCOMP_ERR_ARG;
        if (q.cap < geom[s].R) return LSCOMP_ERR_CAPACITY;
        const int v = vec_class(q.d_in, q.z, sizeof(T));
        if (v < vec) vec = v;
        tile0[s] = total;
        total += geom[s].ntiles;
    }
    if (sizeof(T) == 4 && vec == 2) return LSCOMP_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    std::lock_guard<std::mutex> lk(ws->mu);
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != ws->device) cudaSetDevice(ws->device);
    int r = ws_prepare(ws, total, st);
    if (!r) r = batch_reserve(ws, n, total, st);
    if (!r) {
        for (uint32_t s = 0; s < n; s++) {
            BatchStack &b = ws->h_stacks[s];
            b.g = geom[s];
            b.in = stacks[s].d_in;
            b.out = stacks[s].d_out;
            b.cap = stacks[s].cap;
            b.tile0 = tile0[s];
            b.sizes = ws->d_bsizes + 2ull * s;
        }
        r = cuda_status(cudaMemcpyAsync(ws->d_stacks, ws->h_stacks, n * sizeof(BatchStack), cudaMemcpyHostToDevice, st));
    }
    if (!r) {
        const uint32_t grid = n < 4096u ? n : 4096u;
        tile_stack_kernel<<<grid, 256, 0, st>>>(ws->d_stacks, n, ws->d_tile_stack);
        g_launches.fetch_add(1);
        r = cuda_status(cudaGetLastError());
    }
    if (!r) {
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
        const bool pool = c.pool_min <= 64;
        switch (vec) {
        case 16: r = launch_enc_v<T, 16, true>(a, layout, pool, ws->sm_count, st); break;
        case 4: r = launch_enc_v<T, 4, true>(a, layout, pool, ws->sm_count, st); break;
        default:
            if (sizeof(T) == 2) r = launch_enc_v<T, 2, true>(a, layout, pool, ws->sm_count, st);
            else r = LSCOMP_ERR_ARG;
            break;
        }
    }
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

}  // namespace

extern "C" {

int lscomp_compress_batch_u16(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t bins[4],
                              float pooling, uint64_t *stream_len, uint64_t *ref_size, void *stream)
{
    return compress_batch_t<uint16_t>(ws, stacks, n, bins, pooling, stream_len, ref_size, stream);
}

int lscomp_compress_batch_u32(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t bins[4],
                              float pooling, uint64_t *stream_len, uint64_t *ref_size, void *stream)
{
    return compress_batch_t<uint32_t>(ws, stacks, n, bins, pooling, stream_len, ref_size, stream);
}

}  // extern "C"
