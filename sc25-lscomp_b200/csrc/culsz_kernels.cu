// culsz_kernels.cu -- the four __global__ kernels of the reference's public
// kernel header (include/cuLSZ_kernel.h, lsCOMP/include/cuLSZ_kernel.h:9-36)
// for callers that launch them directly with the reference's launch
// contract: one CTA of 32 threads per 1024 8x8 blocks (block_per_thread =
// 32 blocks per thread), and three zeroed scratch arrays of grid + 1
// entries.  The stream is the reference's, byte for byte; the block math is
// this library's (block_header, block_pack, dec_values in
// codec_kernels.cuh), applied to one CTA's 1024 blocks at a time:
//
//   * the CTA claims its run of 1024 blocks from a ticket in flag[grid], so
//     every run a CTA waits for belongs to a CTA that is already running;
//   * pass A: the header byte of every block (rows read straight from the
//     input, edges filled with zeros), written to the stream; the block
//     sizes are scanned across the warp;
//   * the run's payload offset comes from a decoupled look-back over the
//     caller's scratch: flag[i] = 1 when locOffset[i] holds run i's payload
//     bytes, 2 when cmpOffset[i] holds the bytes of runs 0..i (values are
//     written before their flag with release/acquire ordering); every wait
//     is bounded, and a wait that runs out (or a value range the 5-bit rate
//     field cannot carry) sets the sign bit of flag[grid], which ends every
//     other CTA's wait and claim;
//   * pass B: the rows again (now in L2), quantised and packed as bit planes
//     straight to their stream offsets; the last run writes the total
//     payload to cmpOffset[grid] and zeroes the header pad.
// Decompression mirrors it: header bytes, sizes, the same look-back for the
// run's payload offset, then every block's rows rebuilt and written (blocks
// of rate 0 as zeros).
#include <cuda_runtime.h>
#include <stdint.h>
#include "cuLSZ_kernel.h"
#include "codec_kernels.cuh"

namespace {

using namespace lsc;

constexpr uint32_t kRun = 32u * block_per_thread;  // 8x8 blocks per CTA (1024)
constexpr uint32_t kUnits = kRun / 8;              // 8-block units per CTA
constexpr int kAborted = (int)0x80000000;          // sign bit of flag[grid]

__device__ __forceinline__ int ld_acquire_i32(const volatile int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_i32(volatile int *p, int v)
{
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// The codec of the launch's bins and pooling threshold, as make_codec
// builds it on the host (codec_host.h); false if a bin is 0.
__device__ bool device_codec(const uint4 qb, float p, bool wide, Codec &c)
{
    const uint32_t b[4] = {qb.x, qb.y, qb.z, qb.w};
    bool ok = true;
    for (int k = 0; k < 4; k++) {
        const uint32_t v = b[k] ? b[k] : 1u;
        ok = ok && b[k] != 0u;
        c.bins[k] = v;
        c.magic[k] = v == 1u ? 0u : (uint32_t)((0x100000000ull + v - 1) / v);
        c.magic64[k] = v < 2u ? 0ull : ~0ull / v + 1;
        c.binc[k] = (!wide && v > 65536u) ? 65536u : v;
        c.qsm[k] = lsc_small_quant_magic(v);
    }
    c.pool_min = 65;
    for (int k = 0; k <= 64; k++)
        if ((float)k / 64.0f > p) {  // lsCOMP/src/cuLSZ_kernel.cu:920-921
            c.pool_min = k;
            break;
        }
    return ok;
}

// Rows r and r+4 of block b (block index order, z fastest) from global
// memory; values outside the stack are 0.
template <typename T>
__device__ __forceinline__ void block_rows(const T *in, uint3 d, uint32_t byb, uint32_t bzb, uint32_t b, bool active,
                                           uint32_t r, Row<T> &A, Row<T> &B, unsigned long long &e0, uint32_t &nrows,
                                           uint32_t &ncols)
{
    const uint32_t per = byb * bzb;
    const uint32_t x = b / per, rem = b - x * per, by = rem / bzb, bz = rem - by * bzb;
    const uint32_t ry = d.y - 8u * by, cz = d.z - 8u * bz;
    nrows = ry < 8u ? ry : 8u;
    ncols = cz < 8u ? cz : 8u;
    e0 = ((unsigned long long)x * d.y + 8ull * by + r) * d.z + 8ull * bz;  // row r's first element
#pragma unroll
    for (int i = 0; i < Elem<T>::kWords; i++) A.w[i] = B.w[i] = 0;
    if (!active) return;
    if (r < nrows) load_cols<T>(in + e0, ncols, A);
    if (r + 4 < nrows) load_cols<T>(in + e0 + 4ull * d.z, ncols, B);
}

// Claim the next run (lane 0's ticket, to the whole warp); -1 when none is
// left or the launch was aborted.
__device__ __forceinline__ int claim(volatile int *flag, uint32_t grid)
{
    int t = 0;
    if ((threadIdx.x & 31u) == 0) t = atomicAdd(const_cast<int *>(&flag[grid]), 1);
    t = __shfl_sync(0xffffffffu, t, 0);
    return (t < 0 || (uint32_t)t >= grid) ? -1 : t;
}

__device__ __forceinline__ void abort_launch(volatile int *flag, uint32_t grid)
{
    atomicOr(const_cast<int *>(&flag[grid]), kAborted);
}

// Exclusive scan of the 1024 block sizes of the run (size of block i from
// header byte hdr[i]) into off[]; returns the run's total in every lane.
__device__ __forceinline__ uint32_t run_scan(const uint8_t *hdr, uint32_t *off)
{
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t sum = 0;
    for (uint32_t i = 0; i < 32u; i++) {
        const uint32_t h = hdr[lane * 32u + i];
        sum += (h & 0x1fu) << (3u - (h >> 7));  // rate planes of 8 bytes, or 4 when pooled
    }
    uint32_t inc = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= (uint32_t)o) inc += v;
    }
    uint32_t run = inc - sum;
    for (uint32_t i = 0; i < 32u; i++) {
        const uint32_t h = hdr[lane * 32u + i];
        off[lane * 32u + i] = run;
        run += (h & 0x1fu) << (3u - (h >> 7));
    }
    return __shfl_sync(0xffffffffu, inc, 31);
}

// Payload bytes of runs 0 .. t-1 by decoupled look-back over the caller's
// scratch, then run t's own entries published.  ok = false when a wait ran
// out or the launch was aborted.
template <typename OffT>
__device__ unsigned long long run_prefix(volatile OffT *cmpOffset, volatile OffT *locOffset, volatile int *flag,
                                         uint32_t grid, uint32_t t, uint32_t agg, bool &ok)
{
    const uint32_t lane = threadIdx.x & 31u;
    ok = true;
    if (t > 0 && lane == 0) {
        locOffset[t] = (OffT)agg;
        st_release_i32(&flag[t], 1);
    }
    unsigned long long excl = 0;
    long long end = (long long)t - 1;
    const unsigned long long t0 = global_ns();
    uint32_t spins = 0;
    while (end >= 0) {
        const long long idx = end - (long long)lane;
        int f = 2;
        unsigned long long v = 0;
        if (idx >= 0) {
            f = ld_acquire_i32(&flag[idx]);
            v = f == 2 ? (unsigned long long)cmpOffset[idx] : (f == 1 ? (unsigned long long)locOffset[idx] : 0ull);
        }
        const uint32_t missing = __ballot_sync(0xffffffffu, f != 1 && f != 2);
        const uint32_t incl = __ballot_sync(0xffffffffu, f == 2);
        const uint32_t upto = incl ? ((incl & (0u - incl)) << 1) - 1u : 0xffffffffu;  // lanes up to the first inclusive
        if ((missing & upto) == 0) {
            unsigned long long part = ((upto >> lane) & 1u) ? v : 0ull;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
            excl += part;
            if (incl) break;
            end -= 32;
            continue;
        }
        if ((++spins & 63u) == 0) {
            bool stop = false;
            if (lane == 0) stop = ld_acquire_i32(&flag[grid]) < 0 || global_ns() - t0 > kWaitLimitNs;
            if (__shfl_sync(0xffffffffu, stop, 0)) {
                if (lane == 0) abort_launch(flag, grid);
                ok = false;
                return 0;
            }
        }
        __nanosleep(64);
    }
    if (lane == 0) {
        cmpOffset[t] = (OffT)(excl + agg);
        st_release_i32(&flag[t], 2);
    }
    return excl;
}

template <typename T, typename OffT>
__device__ void compress_runs(const T *in, unsigned char *out, volatile OffT *cmpOffset, volatile OffT *locOffset,
                              volatile int *flag, uint32_t nb, uint3 d, uint4 qb, float p)
{
    __shared__ uint8_t hdr[kRun];
    __shared__ uint32_t off[kRun];
    const uint32_t grid = gridDim.x, lane = threadIdx.x & 31u, jb = lane & 7u, r = lane >> 3;
    const uint32_t byb = (d.y + 7u) / 8u, bzb = (d.z + 7u) / 8u;
    const unsigned long long R = (nb + 3ull) / 4ull * 4ull;
    Codec c;
    if (!device_codec(qb, p, sizeof(T) == 4, c) || (reinterpret_cast<uintptr_t>(out) & 3u) ||
        (reinterpret_cast<uintptr_t>(in) & (sizeof(T) - 1))) {
        if (lane == 0) abort_launch(flag, grid);
        return;
    }
    const XSel xs = xsel(r);
    for (;;) {
        const int t = claim(flag, grid);
        if (t < 0) return;
        const uint32_t k0 = (uint32_t)t * kRun;
        // pass A: header bytes (lsCOMP/src/cuLSZ_kernel.cu:877-957)
        uint32_t bad = 0;
        for (uint32_t u = 0; u < kUnits; u++) {
            const uint32_t i = u * 8u + jb, b = k0 + i;
            const bool active = b < nb;
            Row<T> A, B;
            unsigned long long e0;
            uint32_t nrows, ncols;
            block_rows<T>(in, d, byb, bzb, active ? b : 0u, active, r, A, B, e0, nrows, ncols);
            uint32_t rb;
            const uint32_t h = block_header<T, BINS_GENERAL, true, false>(A, B, c, rb);
            if (r == 0) {
                hdr[i] = active ? (uint8_t)h : 0u;
                if (active) out[b] = (uint8_t)h;
            }
            bad |= active ? rb : 0u;
        }
        __syncwarp();
        if (__any_sync(0xffffffffu, bad != 0)) {  // a quotient that needs 32 planes (uint32)
            if (lane == 0) abort_launch(flag, grid);
            return;
        }
        const uint32_t agg = run_scan(hdr, off);
        bool ok;
        const unsigned long long base = R + run_prefix<OffT>(cmpOffset, locOffset, flag, grid, (uint32_t)t, agg, ok);
        if (!ok) return;
        // pass B: bit planes to the stream (lsCOMP/src/cuLSZ_kernel.cu:1100-1276)
        for (uint32_t u = 0; u < kUnits; u++) {
            const uint32_t i = u * 8u + jb, b = k0 + i;
            const bool active = b < nb;
            Row<T> A, B;
            unsigned long long e0;
            uint32_t nrows, ncols;
            block_rows<T>(in, d, byb, bzb, active ? b : 0u, active, r, A, B, e0, nrows, ncols);
            block_pack<T, false, false>(A, B, hdr[i], active, r, xs, c, out + base + (active ? off[i] : 0u));
        }
        if ((uint32_t)t == grid - 1) {
            if (lane == 0) cmpOffset[grid] = (OffT)(base - R + agg);  // the payload of the whole stream
            if (lane < (uint32_t)(R - nb)) out[nb + lane] = 0;         // header pad
        }
        __syncwarp();
    }
}

template <typename T, typename OffT>
__device__ void decompress_runs(T *outv, const unsigned char *in, volatile OffT *cmpOffset, volatile OffT *locOffset,
                                volatile int *flag, uint32_t nb, uint3 d, uint4 qb, float p)
{
    constexpr int NG = Elem<T>::kGroups;
    __shared__ uint8_t hdr[kRun];
    __shared__ uint32_t off[kRun];
    const uint32_t grid = gridDim.x, lane = threadIdx.x & 31u, jb = lane & 7u, r = lane >> 3;
    const uint32_t byb = (d.y + 7u) / 8u, bzb = (d.z + 7u) / 8u;
    const unsigned long long R = (nb + 3ull) / 4ull * 4ull;
    Codec c;
    if (!device_codec(qb, p, sizeof(T) == 4, c) || (reinterpret_cast<uintptr_t>(in) & 3u) ||
        (reinterpret_cast<uintptr_t>(outv) & (sizeof(T) - 1))) {
        if (lane == 0) abort_launch(flag, grid);
        return;
    }
    for (;;) {
        const int t = claim(flag, grid);
        if (t < 0) return;
        const uint32_t k0 = (uint32_t)t * kRun;
        for (uint32_t i = lane; i < kRun; i += 32u) hdr[i] = k0 + i < nb ? in[k0 + i] : 0u;
        __syncwarp();
        const uint32_t agg = run_scan(hdr, off);
        bool ok;
        const unsigned long long base = R + run_prefix<OffT>(cmpOffset, locOffset, flag, grid, (uint32_t)t, agg, ok);
        if (!ok) return;
        for (uint32_t u = 0; u < kUnits; u++) {
            const uint32_t i = u * 8u + jb, b = k0 + i;
            const bool active = b < nb;
            const uint32_t h = hdr[i];
            uint32_t Y[NG][4], Z;
            dec_load<T>(in + base + (active ? off[i] : 0u), h, r, Y, Z);
            const uint32_t wrate = __reduce_max_sync(0xffffffffu, h & 0x1fu);
            Row<T> A, B;
            dec_values<T>(Y, Z, h, active, r, c.bins[(h >> 5) & 3u], wrate, A, B);
            if (!active) continue;
            const uint32_t per = byb * bzb;
            const uint32_t x = b / per, rem = b - x * per, by = rem / bzb, bz = rem - by * bzb;
            const uint32_t ry = d.y - 8u * by, cz = d.z - 8u * bz;
            const uint32_t nrows = ry < 8u ? ry : 8u, ncols = cz < 8u ? cz : 8u;
            T *row = outv + ((unsigned long long)x * d.y + 8ull * by + r) * d.z + 8ull * bz;
            if (r < nrows) store8<sizeof(T)>(row, A, ncols);
            if (r + 4 < nrows) store8<sizeof(T)>(row + 4ull * d.z, B, ncols);
        }
        __syncwarp();
    }
}

}  // namespace

__global__ void cuLSZ_compression_kernel_uint32_bsize64(const uint32_t *const __restrict__ oriData,
                                                        unsigned char *const __restrict__ cmpBytes,
                                                        volatile unsigned int *const __restrict__ cmpOffset,
                                                        volatile unsigned int *const __restrict__ locOffset,
                                                        volatile int *const __restrict__ flag, uint blockNum,
                                                        const uint3 dims, const uint4 quantBins, const float poolingTH)
{
    compress_runs<uint32_t, unsigned int>(oriData, cmpBytes, cmpOffset, locOffset, flag, blockNum, dims, quantBins,
                                          poolingTH);
}

__global__ void cuLSZ_decompression_kernel_uint32_bsize64(uint32_t *const __restrict__ decData,
                                                          const unsigned char *const __restrict__ cmpBytes,
                                                          volatile unsigned int *const __restrict__ cmpOffset,
                                                          volatile unsigned int *const __restrict__ locOffset,
                                                          volatile int *const __restrict__ flag, uint blockNum,
                                                          const uint3 dims, const uint4 quantBins,
                                                          const float poolingTH)
{
    decompress_runs<uint32_t, unsigned int>(decData, cmpBytes, cmpOffset, locOffset, flag, blockNum, dims, quantBins,
                                            poolingTH);
}

__global__ void cuLSZ_compression_kernel_uint16_bsize64(const uint16_t *const __restrict__ oriData,
                                                        unsigned char *const __restrict__ cmpBytes,
                                                        volatile size_t *const __restrict__ cmpOffset,
                                                        volatile size_t *const __restrict__ locOffset,
                                                        volatile int *const __restrict__ flag, uint blockNum,
                                                        const uint3 dims, const uint4 quantBins, const float poolingTH)
{
    compress_runs<uint16_t, size_t>(oriData, cmpBytes, cmpOffset, locOffset, flag, blockNum, dims, quantBins,
                                    poolingTH);
}

__global__ void cuLSZ_decompression_kernel_uint16_bsize64(uint16_t *const __restrict__ decData,
                                                          const unsigned char *const __restrict__ cmpBytes,
                                                          volatile size_t *const __restrict__ cmpOffset,
                                                          volatile size_t *const __restrict__ locOffset,
                                                          volatile int *const __restrict__ flag, uint blockNum,
                                                          const uint3 dims, const uint4 quantBins,
                                                          const float poolingTH)
{
    decompress_runs<uint16_t, size_t>(decData, cmpBytes, cmpOffset, locOffset, flag, blockNum, dims, quantBins,
                                      poolingTH);
}
