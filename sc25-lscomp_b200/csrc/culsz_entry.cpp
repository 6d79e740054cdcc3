// culsz_entry.cpp -- the reference's host API (lsCOMP/include/cuLSZ_entry.h:8-11)
// implemented on top of the C ABI in include/lscomp.h.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <map>
#include <mutex>
#include <utility>
#include "cuLSZ_entry.h"
#include "lscomp.h"

namespace {

std::mutex g_mu;
std::map<std::pair<int, cudaStream_t>, lscomp_workspace *> g_ws;

// One workspace per (device, stream): calls on one stream are ordered, so
// its scan state can be reused without a device-side reset.
lscomp_workspace *workspace_for(cudaStream_t stream)
{
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_mu);
    auto key = std::make_pair(dev, stream);
    auto it = g_ws.find(key);
    if (it != g_ws.end()) return it->second;
    lscomp_workspace *ws = nullptr;
    int s = lscomp_workspace_create(&ws, dev);
    if (s) {
        fprintf(stderr, "lscomp: workspace allocation failed: %s\n", lscomp_status_string(s));
        exit(s);
    }
    g_ws[key] = ws;
    return ws;
}

// Same failure behaviour as the reference's check(): message, then exit
// with the status (lsCOMP/src/cuLSZ_entry.cu:9-15).
void check(int status, const char *what)
{
    if (status == LSCOMP_OK) return;
    fprintf(stderr, "lscomp error in %s: %s (status %d)\n", what, lscomp_status_string(status), status);
    exit(status);
}

}  // namespace

// lsCOMP/src/cuLSZ_entry.cu:93-131.  The reference gives the kernel no
// capacity; the worst-case stream length is assumed available, as the
// reference also assumes implicitly.
void cuLSZ_compression_uint16_bsize64(uint16_t *d_oriData, unsigned char *d_cmpBytes, size_t *cmpSize, uint3 dims,
                                      uint4 quantBins, float poolingTH, cudaStream_t stream)
{
    const uint32_t bins[4] = {quantBins.x, quantBins.y, quantBins.z, quantBins.w};
    lscomp_workspace *ws = workspace_for(stream);
    uint64_t cap = lscomp_max_stream_bytes_u16(dims.x, dims.y, dims.z);
    uint64_t stream_len = 0, ref_size = 0;
    check(lscomp_compress_u16(ws, d_oriData, dims.x, dims.y, dims.z, bins, poolingTH, d_cmpBytes, cap, &stream_len,
                              &ref_size, stream),
          "cuLSZ_compression_uint16_bsize64");
    if (cmpSize) *cmpSize = (size_t)ref_size;
}

// lsCOMP/src/cuLSZ_entry.cu:133-166.  cmpSize is not used by the reference;
// here the readable length is taken as the worst-case stream length, like the
// compression side.
void cuLSZ_decompression_uint16_bsize64(uint16_t *d_decData, unsigned char *d_cmpBytes, size_t cmpSize, uint3 dims,
                                        uint4 quantBins, float poolingTH, cudaStream_t stream)
{
    (void)cmpSize;
    const uint32_t bins[4] = {quantBins.x, quantBins.y, quantBins.z, quantBins.w};
    lscomp_workspace *ws = workspace_for(stream);
    uint64_t cap = lscomp_max_stream_bytes_u16(dims.x, dims.y, dims.z);
    check(lscomp_decompress_u16(ws, d_cmpBytes, cap, dims.x, dims.y, dims.z, bins, poolingTH, d_decData, stream),
          "cuLSZ_decompression_uint16_bsize64");
}

// lsCOMP/src/cuLSZ_entry.cu:18-56.  *cmpSize = 32-bit payload total + nb, as
// the reference computes it.
void cuLSZ_compression_uint32_bsize64(uint32_t *d_oriData, unsigned char *d_cmpBytes, size_t *cmpSize, uint3 dims,
                                      uint4 quantBins, float poolingTH, cudaStream_t stream)
{
    const uint32_t bins[4] = {quantBins.x, quantBins.y, quantBins.z, quantBins.w};
    lscomp_workspace *ws = workspace_for(stream);
    uint64_t cap = lscomp_max_stream_bytes_u32(dims.x, dims.y, dims.z);
    uint64_t stream_len = 0, ref_size = 0;
    check(lscomp_compress_u32(ws, d_oriData, dims.x, dims.y, dims.z, bins, poolingTH, d_cmpBytes, cap, &stream_len,
                              &ref_size, stream),
          "cuLSZ_compression_uint32_bsize64");
    if (cmpSize) *cmpSize = (size_t)ref_size;
}

// lsCOMP/src/cuLSZ_entry.cu:58-91
void cuLSZ_decompression_uint32_bsize64(uint32_t *d_decData, unsigned char *d_cmpBytes, size_t cmpSize, uint3 dims,
                                        uint4 quantBins, float poolingTH, cudaStream_t stream)
{
    (void)cmpSize;
    const uint32_t bins[4] = {quantBins.x, quantBins.y, quantBins.z, quantBins.w};
    lscomp_workspace *ws = workspace_for(stream);
    uint64_t cap = lscomp_max_stream_bytes_u32(dims.x, dims.y, dims.z);
    check(lscomp_decompress_u32(ws, d_cmpBytes, cap, dims.x, dims.y, dims.z, bins, poolingTH, d_decData, stream),
          "cuLSZ_decompression_uint32_bsize64");
}
