// host_pipe.cu -- compression and decompression straight from and to host
// memory (include/lscomp.h, lscomp_compress_host_* / lscomp_decompress_host_*).
//
// The stack is cut into chunks of whole frames.  Chunks go through two
// device slots, so the copy of one chunk to the device, the kernel of the
// next and the copy of a third back to the host run at the same time: one
// copy stream per direction plus the caller's stream for the kernels, with
// events between them.  The stream of a stack is the concatenation of its
// chunks' streams taken apart: block order is frame-major, so chunk c's
// header bytes are the global header bytes [k0_c, k0_c + nb_c) and its
// payload follows the payload of every earlier chunk.  Compression learns a
// chunk's payload size when its kernel finishes (the control block copied to
// pinned memory) and places the payload then; decompression uploads the
// whole header first and sums every chunk's payload on the device, so all
// chunk offsets are known before the first payload byte moves.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>
#include <algorithm>
#include <mutex>
#include <vector>
#include "codec_host.h"

using namespace lsc;
using namespace lsc_host;

namespace lsc_host {

constexpr uint64_t kPipeChunkBytes = 128ull << 20;  // input bytes per chunk (whole frames, at least one)
constexpr uint32_t kPipeMaxChunks = 4096;           // chunks per call at most (one pinned status slot each)

struct PipeState {
    std::mutex mu;
    cudaStream_t up = nullptr, down = nullptr;  // host->device and device->host copy streams
    cudaEvent_t ev_up[2] = {}, ev_run[2] = {}, ev_down[2] = {};
    uint8_t *buf_a[2] = {}, *buf_b[2] = {};     // per slot: chunk input / stream (a), stream / output (b)
    uint64_t buf_cap = 0;                        // bytes of each of the four buffers
    uint8_t *d_hdr = nullptr;                    // decompression: the whole header
    uint64_t hdr_cap = 0;
    unsigned long long *d_sums = nullptr, *h_sums = nullptr;  // decompression: payload bytes per chunk
    LaunchCtl *h_ctl = nullptr;                  // pinned status of each chunk
};

void pipe_destroy(lscomp_workspace *ws)
{
    PipeState *p = static_cast<PipeState *>(ws->pipe);
    if (!p) return;
    if (p->up) cudaStreamDestroy(p->up);
    if (p->down) cudaStreamDestroy(p->down);
    for (int s = 0; s < 2; s++) {
        if (p->ev_up[s]) cudaEventDestroy(p->ev_up[s]);
        if (p->ev_run[s]) cudaEventDestroy(p->ev_run[s]);
        if (p->ev_down[s]) cudaEventDestroy(p->ev_down[s]);
        if (p->buf_a[s]) cudaFree(p->buf_a[s]);
        if (p->buf_b[s]) cudaFree(p->buf_b[s]);
    }
    if (p->d_hdr) cudaFree(p->d_hdr);
    if (p->d_sums) cudaFree(p->d_sums);
    if (p->h_sums) cudaFreeHost(p->h_sums);
    if (p->h_ctl) cudaFreeHost(p->h_ctl);
    delete p;
    ws->pipe = nullptr;
}

}  // namespace lsc_host

namespace {

// The workspace's pipeline state (streams, events, pinned status), created
// on first use under the workspace lock; the caller then holds its own lock.
int pipe_state(lscomp_workspace *ws, PipeState *&out)
{
    std::lock_guard<std::mutex> g(ws->mu);
    PipeState *p = static_cast<PipeState *>(ws->pipe);
    if (!p) {
        p = new (std::nothrow) PipeState();
        if (!p) return LSCOMP_ERR_NOMEM;
        ws->pipe = p;
        cudaError_t e = cudaStreamCreateWithFlags(&p->up, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->down, cudaStreamNonBlocking);
        for (int s = 0; s < 2 && e == cudaSuccess; s++) {
            e = cudaEventCreateWithFlags(&p->ev_up[s], cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->ev_run[s], cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->ev_down[s], cudaEventDisableTiming);
        }
        if (e == cudaSuccess) e = cudaMallocHost(&p->h_ctl, kPipeMaxChunks * sizeof(LaunchCtl));
        if (e == cudaSuccess) e = cudaMalloc(&p->d_sums, kPipeMaxChunks * sizeof(unsigned long long));
        if (e == cudaSuccess) e = cudaMallocHost(&p->h_sums, kPipeMaxChunks * sizeof(unsigned long long));
        if (e != cudaSuccess) {
            pipe_destroy(ws);
            return cuda_status(e);
        }
    }
    out = p;
    return LSCOMP_OK;
}

// Slot buffers of at least `need` bytes each (the pipeline lock held; every
// earlier use of the buffers has finished, since each call ends with its
// streams synchronised).
int pipe_reserve(PipeState *p, uint64_t need)
{
    if (need <= p->buf_cap) return LSCOMP_OK;
    for (int s = 0; s < 2; s++) {
        if (p->buf_a[s]) cudaFree(p->buf_a[s]);
        if (p->buf_b[s]) cudaFree(p->buf_b[s]);
        p->buf_a[s] = p->buf_b[s] = nullptr;
    }
    p->buf_cap = 0;
    cudaError_t e = cudaSuccess;
    for (int s = 0; s < 2 && e == cudaSuccess; s++) {
        e = cudaMalloc(&p->buf_a[s], need);
        if (e == cudaSuccess) e = cudaMalloc(&p->buf_b[s], need);
    }
    if (e != cudaSuccess) return cuda_status(e);
    p->buf_cap = need;
    return LSCOMP_OK;
}

// Chunking: frames per chunk and the number of chunks (at most
// kPipeMaxChunks, so every chunk has its own pinned status slot).
void chunking(uint64_t chunk_bytes, uint32_t x, uint64_t frame_bytes, uint32_t &fpc, uint32_t &nchunks)
{
    uint64_t f = (chunk_bytes ? chunk_bytes : kPipeChunkBytes) / (frame_bytes ? frame_bytes : 1);
    if (f < 1) f = 1;
    if (f > x) f = x;
    uint64_t n = (x + f - 1) / f;
    if (n > kPipeMaxChunks) {
        f = (x + kPipeMaxChunks - 1) / kPipeMaxChunks;
        n = (x + f - 1) / f;
    }
    fpc = (uint32_t)f;
    nchunks = (uint32_t)n;
}

uint64_t max_stream(uint64_t nb, size_t es) { return (nb + 3) / 4 * 4 + (es == 2 ? 128ull : 248ull) * nb; }

template <typename T>
int compress_chunk(lscomp_workspace *ws, const void *d_in, uint32_t nf, uint32_t y, uint32_t z, const uint32_t bins[4],
                   float p, uint8_t *d_out, uint64_t cap, cudaStream_t st)
{
    if constexpr (sizeof(T) == 2)
        return lscomp_compress_u16_async(ws, static_cast<const uint16_t *>(d_in), nf, y, z, bins, p, d_out, cap,
                                         nullptr, st);
    else
        return lscomp_compress_u32_async(ws, static_cast<const uint32_t *>(d_in), nf, y, z, bins, p, d_out, cap,
                                         nullptr, st);
}

template <typename T>
int decompress_chunk(lscomp_workspace *ws, const uint8_t *d_in, uint64_t len, uint32_t nf, uint32_t y, uint32_t z,
                     const uint32_t bins[4], float p, void *d_out, cudaStream_t st)
{
    if constexpr (sizeof(T) == 2)
        return lscomp_decompress_u16_async(ws, d_in, len, nf, y, z, bins, p, static_cast<uint16_t *>(d_out), st);
    else
        return lscomp_decompress_u32_async(ws, d_in, len, nf, y, z, bins, p, static_cast<uint32_t *>(d_out), st);
}

template <typename T>
int compress_host_t(lscomp_workspace *ws, const T *h_in, uint32_t x, uint32_t y, uint32_t z, const uint32_t bins[4],
                    float pooling, uint8_t *h_out, uint64_t cap, uint64_t *stream_len, uint64_t *ref_size,
                    void *stream)
{
    if (!ws || !h_in || !h_out || !bins || !x || !y || !z) return LSCOMP_ERR_ARG;
    const uint64_t byb = (y + 7) / 8, bzb = (z + 7) / 8, bpf = byb * bzb;  // blocks per frame
    const uint64_t nb = (uint64_t)x * bpf, R = (nb + 3) / 4 * 4;
    if (cap < R) return LSCOMP_ERR_CAPACITY;
    const uint64_t frame_bytes = (uint64_t)y * z * sizeof(T);
    uint32_t fpc, nchunks;
    chunking(ws->host_chunk_bytes, x, frame_bytes, fpc, nchunks);
    const uint64_t need = std::max<uint64_t>(fpc * frame_bytes, max_stream(fpc * bpf, sizeof(T)));
    cudaStream_t st = (cudaStream_t)stream;
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != ws->device) cudaSetDevice(ws->device);
    PipeState *p = nullptr;
    std::unique_lock<std::mutex> lk;
    int r = pipe_state(ws, p);
    if (!r) {
        lk = std::unique_lock<std::mutex>(p->mu);
        r = pipe_reserve(p, need);
    }
    uint64_t payload = 0;  // bytes of the payload placed so far
    // host side of chunk c once its kernel has finished: status, then the
    // header bytes and the payload copied to their places in h_out
    auto place = [&](uint32_t c) -> int {
        const int s = (int)(c & 1u);
        const uint32_t f0 = c * fpc, nf = std::min<uint32_t>(fpc, x - f0);
        const uint64_t nb_c = (uint64_t)nf * bpf, R_c = (nb_c + 3) / 4 * 4;
        cudaError_t e = cudaEventSynchronize(p->ev_run[s]);
        if (e != cudaSuccess) return cuda_status(e);
        const LaunchCtl &h = p->h_ctl[c];
        if (h.error) return dev_status(h.error);
        const uint64_t pay = h.total;
        if (R + payload + pay > cap) return LSCOMP_ERR_CAPACITY;
        e = cudaStreamWaitEvent(p->down, p->ev_run[s], 0);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(h_out + (uint64_t)f0 * bpf, p->buf_b[s], nb_c, cudaMemcpyDeviceToHost, p->down);
        if (e == cudaSuccess && pay)
            e = cudaMemcpyAsync(h_out + R + payload, p->buf_b[s] + R_c, pay, cudaMemcpyDeviceToHost, p->down);
        if (e == cudaSuccess) e = cudaEventRecord(p->ev_down[s], p->down);
        payload += pay;
        return cuda_status(e);
    };
    for (uint32_t c = 0; !r && c < nchunks; c++) {
        const int s = (int)(c & 1u);
        const uint32_t f0 = c * fpc, nf = std::min<uint32_t>(fpc, x - f0);
        // slot s: its input is free once chunk c-2's kernel has run, its
        // stream buffer once chunk c-2's copies down have run
        cudaError_t e = cudaStreamWaitEvent(p->up, p->ev_run[s], 0);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(p->buf_a[s], reinterpret_cast<const uint8_t *>(h_in) + (uint64_t)f0 * frame_bytes,
                                (uint64_t)nf * frame_bytes, cudaMemcpyHostToDevice, p->up);
        if (e == cudaSuccess) e = cudaEventRecord(p->ev_up[s], p->up);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(st, p->ev_up[s], 0);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(st, p->ev_down[s], 0);
        r = cuda_status(e);
        if (!r) r = compress_chunk<T>(ws, p->buf_a[s], nf, y, z, bins, pooling, p->buf_b[s], p->buf_cap, st);
        if (!r) r = cuda_status(cudaMemcpyAsync(&p->h_ctl[c], ws->ctl, sizeof(LaunchCtl), cudaMemcpyDeviceToHost, st));
        if (!r) r = cuda_status(cudaEventRecord(p->ev_run[s], st));
        if (!r && c > 0) r = place(c - 1);
    }
    if (!r) r = place(nchunks - 1);
    // every copy of this call has finished before the call returns
    const cudaError_t e1 = cudaStreamSynchronize(st);
    const cudaError_t e2 = p ? cudaStreamSynchronize(p->up) : cudaSuccess;
    const cudaError_t e3 = p ? cudaStreamSynchronize(p->down) : cudaSuccess;
    if (!r && e1 != cudaSuccess) r = cuda_status(e1);
    if (!r && e2 != cudaSuccess) r = cuda_status(e2);
    if (!r && e3 != cudaSuccess) r = cuda_status(e3);
    if (!r) {
        for (uint64_t k = nb; k < R; k++) h_out[k] = 0;  // header pad
        uint64_t total = payload;
        if (sizeof(T) == 4) total &= 0xffffffffull;  // the reference reports a 32-bit total for uint32
        if (stream_len) *stream_len = R + payload;
        if (ref_size) *ref_size = total + nb;
    }
    if (prev != ws->device) cudaSetDevice(prev);
    return r;
}

// payload bytes of each chunk's blocks (chunk c: header bytes
// [c * bpc, min((c + 1) * bpc, nb)))
__global__ void chunk_sums_kernel(const uint8_t *hdr, unsigned long long nb, unsigned long long bpc,
                                  unsigned long long *sums)
{
    __shared__ unsigned long long part[32];
    const unsigned long long k0 = blockIdx.x * bpc;
    const unsigned long long k1 = min(k0 + bpc, nb);
    unsigned long long s = 0;
    for (unsigned long long k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
        const uint32_t h = hdr[k];
        s += (h & 0x1fu) << (3u - (h >> 7));  // rate planes of 8 bytes, or 4 when pooled
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < blockDim.x / 32 ? part[threadIdx.x] : 0ull;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) sums[blockIdx.x] = s;
    }
}

template <typename T>
int decompress_host_t(lscomp_workspace *ws, const uint8_t *h_in, uint64_t cmp_len, uint32_t x, uint32_t y, uint32_t z,
                      const uint32_t bins[4], float pooling, T *h_out, void *stream)
{
    if (!ws || !h_in || !h_out || !bins || !x || !y || !z) return LSCOMP_ERR_ARG;
    const uint64_t byb = (y + 7) / 8, bzb = (z + 7) / 8, bpf = byb * bzb;
    const uint64_t nb = (uint64_t)x * bpf, R = (nb + 3) / 4 * 4;
    if (cmp_len < nb) return LSCOMP_ERR_CAPACITY;
    const uint64_t frame_bytes = (uint64_t)y * z * sizeof(T);
    uint32_t fpc, nchunks;
    chunking(ws->host_chunk_bytes, x, frame_bytes, fpc, nchunks);
    const uint64_t need = std::max<uint64_t>(fpc * frame_bytes, max_stream(fpc * bpf, sizeof(T)));
    cudaStream_t st = (cudaStream_t)stream;
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != ws->device) cudaSetDevice(ws->device);
    PipeState *p = nullptr;
    std::unique_lock<std::mutex> lk;
    int r = pipe_state(ws, p);
    if (!r) {
        lk = std::unique_lock<std::mutex>(p->mu);
        r = pipe_reserve(p, need);
    }
    // the whole header up, every chunk's payload size down
    if (!r && nb > p->hdr_cap) {
        if (p->d_hdr) cudaFree(p->d_hdr);
        p->d_hdr = nullptr;
        p->hdr_cap = 0;
        r = cuda_status(cudaMalloc(&p->d_hdr, nb));
        if (!r) p->hdr_cap = nb;
    }
    if (!r) r = cuda_status(cudaMemcpyAsync(p->d_hdr, h_in, nb, cudaMemcpyHostToDevice, p->up));
    if (!r) {
        chunk_sums_kernel<<<nchunks, 512, 0, p->up>>>(p->d_hdr, nb, (unsigned long long)fpc * bpf, p->d_sums);
        g_launches.fetch_add(1);
        r = cuda_status(cudaGetLastError());
    }
    if (!r)
        r = cuda_status(cudaMemcpyAsync(p->h_sums, p->d_sums, nchunks * sizeof(unsigned long long),
                                        cudaMemcpyDeviceToHost, p->up));
    if (!r) r = cuda_status(cudaStreamSynchronize(p->up));
    std::vector<uint64_t> off(nchunks + 1, 0);
    for (uint32_t c = 0; !r && c < nchunks; c++) off[c + 1] = off[c] + p->h_sums[c];
    if (!r && R + off[nchunks] > cmp_len) r = LSCOMP_ERR_CAPACITY;
    for (uint32_t c = 0; !r && c < nchunks; c++) {
        const int s = (int)(c & 1u);
        const uint32_t f0 = c * fpc, nf = std::min<uint32_t>(fpc, x - f0);
        const uint64_t nb_c = (uint64_t)nf * bpf, R_c = (nb_c + 3) / 4 * 4, pay = off[c + 1] - off[c];
        // chunk stream [header | pad | payload] into slot s's buffer a, free
        // once chunk c-2's kernel has run
        cudaError_t e = cudaStreamWaitEvent(p->up, p->ev_run[s], 0);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(p->buf_a[s], p->d_hdr + (uint64_t)f0 * bpf, nb_c, cudaMemcpyDeviceToDevice, p->up);
        if (e == cudaSuccess && R_c > nb_c) e = cudaMemsetAsync(p->buf_a[s] + nb_c, 0, R_c - nb_c, p->up);
        if (e == cudaSuccess && pay)
            e = cudaMemcpyAsync(p->buf_a[s] + R_c, h_in + R + off[c], pay, cudaMemcpyHostToDevice, p->up);
        if (e == cudaSuccess) e = cudaEventRecord(p->ev_up[s], p->up);
        // the kernel writes buffer b, free once chunk c-2's copy down has run
        if (e == cudaSuccess) e = cudaStreamWaitEvent(st, p->ev_up[s], 0);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(st, p->ev_down[s], 0);
        r = cuda_status(e);
        if (!r) r = decompress_chunk<T>(ws, p->buf_a[s], R_c + pay, nf, y, z, bins, pooling, p->buf_b[s], st);
        if (!r) r = cuda_status(cudaMemcpyAsync(&p->h_ctl[c], ws->ctl, sizeof(LaunchCtl), cudaMemcpyDeviceToHost, st));
        if (!r) r = cuda_status(cudaEventRecord(p->ev_run[s], st));
        if (!r) {
            e = cudaStreamWaitEvent(p->down, p->ev_run[s], 0);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(reinterpret_cast<uint8_t *>(h_out) + (uint64_t)f0 * frame_bytes, p->buf_b[s],
                                    (uint64_t)nf * frame_bytes, cudaMemcpyDeviceToHost, p->down);
            if (e == cudaSuccess) e = cudaEventRecord(p->ev_down[s], p->down);
            r = cuda_status(e);
        }
    }
    const cudaError_t e1 = cudaStreamSynchronize(st);
    const cudaError_t e2 = p ? cudaStreamSynchronize(p->up) : cudaSuccess;
    const cudaError_t e3 = p ? cudaStreamSynchronize(p->down) : cudaSuccess;
    if (!r && e1 != cudaSuccess) r = cuda_status(e1);
    if (!r && e2 != cudaSuccess) r = cuda_status(e2);
    if (!r && e3 != cudaSuccess) r = cuda_status(e3);
    for (uint32_t c = 0; !r && c < nchunks; c++)
        if (p->h_ctl[c].error) r = dev_status(p->h_ctl[c].error);
    if (prev != ws->device) cudaSetDevice(prev);
    return r;
}

}  // namespace

extern "C" {

int lscomp_workspace_set_host_chunk(lscomp_workspace *ws, uint64_t bytes)
{
    if (!ws) return LSCOMP_ERR_ARG;
    ws->host_chunk_bytes = bytes;
    return LSCOMP_OK;
}

int lscomp_compress_host_u16(lscomp_workspace *ws, const uint16_t *h_in, uint32_t x, uint32_t y, uint32_t z,
                             const uint32_t bins[4], float pooling, uint8_t *h_out, uint64_t cap,
                             uint64_t *stream_len, uint64_t *ref_size, void *stream)
{
    return compress_host_t<uint16_t>(ws, h_in, x, y, z, bins, pooling, h_out, cap, stream_len, ref_size, stream);
}

int lscomp_compress_host_u32(lscomp_workspace *ws, const uint32_t *h_in, uint32_t x, uint32_t y, uint32_t z,
                             const uint32_t bins[4], float pooling, uint8_t *h_out, uint64_t cap,
                             uint64_t *stream_len, uint64_t *ref_size, void *stream)
{
    return compress_host_t<uint32_t>(ws, h_in, x, y, z, bins, pooling, h_out, cap, stream_len, ref_size, stream);
}

int lscomp_decompress_host_u16(lscomp_workspace *ws, const uint8_t *h_in, uint64_t cmp_len, uint32_t x, uint32_t y,
                               uint32_t z, const uint32_t bins[4], float pooling, uint16_t *h_out, void *stream)
{
    return decompress_host_t<uint16_t>(ws, h_in, cmp_len, x, y, z, bins, pooling, h_out, stream);
}

int lscomp_decompress_host_u32(lscomp_workspace *ws, const uint8_t *h_in, uint64_t cmp_len, uint32_t x, uint32_t y,
                               uint32_t z, const uint32_t bins[4], float pooling, uint32_t *h_out, void *stream)
{
    return decompress_host_t<uint32_t>(ws, h_in, cmp_len, x, y, z, bins, pooling, h_out, stream);
}

}  // extern "C"
