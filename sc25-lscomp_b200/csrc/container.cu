// container.cu -- the self-describing container around an lsCOMP stream
// (include/lscomp.h, lscomp_container_*).
//
// The reference's stream carries neither the stack's dimensions nor the
// bins, pooling threshold or element type, and its size travels out of
// band (lsCOMP/src/cuLSZ_entry.cu:124-125).  A container is a 64-byte
// header followed by the stream, byte for byte unchanged:
//
//   0  "LSCZ"            8  x  12 y  16 z           (uint32, z fastest)
//   4  version (u16) = 1, 6 element bytes (u16: 2 or 4)
//   20 bins[4] (uint32)  36 pooling threshold (IEEE binary32)
//   40 stream length (u64)  48 reference-reported size (u64)
//   56 CRC-32 (IEEE 802.3) of bytes 0..55   60 zero
//
// All fields little-endian.  The header is 64 bytes so that a body placed
// right after a 16-byte-aligned header stays 16-byte aligned.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>
#include "lscomp.h"

namespace {

constexpr uint32_t kHdr = 64;
constexpr uint16_t kVersion = 1;

void put32(uint8_t *p, uint32_t v)
{
    for (int i = 0; i < 4; i++) p[i] = (uint8_t)(v >> (8 * i));
}

void put64(uint8_t *p, uint64_t v)
{
    for (int i = 0; i < 8; i++) p[i] = (uint8_t)(v >> (8 * i));
}

uint32_t get32(const uint8_t *p)
{
    uint32_t v = 0;
    for (int i = 0; i < 4; i++) v |= (uint32_t)p[i] << (8 * i);
    return v;
}

uint64_t get64(const uint8_t *p)
{
    uint64_t v = 0;
    for (int i = 0; i < 8; i++) v |= (uint64_t)p[i] << (8 * i);
    return v;
}

// CRC-32 with the reflected polynomial 0xEDB88320 (the IEEE 802.3 / zlib
// checksum), bit by bit: the header is 56 bytes.
uint32_t crc32(const uint8_t *p, size_t n)
{
    uint32_t c = 0xffffffffu;
    for (size_t i = 0; i < n; i++) {
        c ^= p[i];
        for (int k = 0; k < 8; k++) c = (c >> 1) ^ (0xEDB88320u & (0u - (c & 1u)));
    }
    return ~c;
}

int status_of(cudaError_t e)
{
    if (e == cudaSuccess) return LSCOMP_OK;
    if (e == cudaErrorMemoryAllocation) return LSCOMP_ERR_NOMEM;
    return LSCOMP_ERR_CUDA;
}

}  // namespace

extern "C" {

uint32_t lscomp_container_header_bytes(void) { return kHdr; }

int lscomp_container_write_header(uint8_t *hdr, uint32_t elem_bytes, uint32_t x, uint32_t y, uint32_t z,
                                  const uint32_t bins[4], float pooling, uint64_t stream_len, uint64_t ref_size)
{
    if (!hdr || !bins || (elem_bytes != 2 && elem_bytes != 4) || !x || !y || !z) return LSCOMP_ERR_ARG;
    memset(hdr, 0, kHdr);
    memcpy(hdr, "LSCZ", 4);
    hdr[4] = (uint8_t)kVersion;
    hdr[5] = (uint8_t)(kVersion >> 8);
    hdr[6] = (uint8_t)elem_bytes;
    put32(hdr + 8, x);
    put32(hdr + 12, y);
    put32(hdr + 16, z);
    for (int k = 0; k < 4; k++) put32(hdr + 20 + 4 * k, bins[k]);
    uint32_t pb;
    memcpy(&pb, &pooling, 4);
    put32(hdr + 36, pb);
    put64(hdr + 40, stream_len);
    put64(hdr + 48, ref_size);
    put32(hdr + 56, crc32(hdr, 56));
    return LSCOMP_OK;
}

int lscomp_container_read_header(const uint8_t *hdr, uint64_t len, lscomp_container_info *info)
{
    if (!hdr || !info) return LSCOMP_ERR_ARG;
    if (len < kHdr || memcmp(hdr, "LSCZ", 4) != 0) return LSCOMP_ERR_CORRUPT;
    if ((uint32_t)(hdr[4] | (hdr[5] << 8)) != kVersion) return LSCOMP_ERR_CORRUPT;
    if (get32(hdr + 56) != crc32(hdr, 56)) return LSCOMP_ERR_CORRUPT;
    lscomp_container_info in;
    in.elem_bytes = hdr[6] | (hdr[7] << 8);
    in.x = get32(hdr + 8);
    in.y = get32(hdr + 12);
    in.z = get32(hdr + 16);
    for (int k = 0; k < 4; k++) in.bins[k] = get32(hdr + 20 + 4 * k);
    const uint32_t pb = get32(hdr + 36);
    memcpy(&in.pooling, &pb, 4);
    in.stream_len = get64(hdr + 40);
    in.ref_size = get64(hdr + 48);
    if ((in.elem_bytes != 2 && in.elem_bytes != 4) || !in.x || !in.y || !in.z) return LSCOMP_ERR_CORRUPT;
    const uint64_t nb = lscomp_block_count(in.x, in.y, in.z);
    if (in.stream_len < (nb + 3) / 4 * 4) return LSCOMP_ERR_CORRUPT;
    if (len != kHdr && len < kHdr + in.stream_len) return LSCOMP_ERR_CORRUPT;  // len = kHdr: header only
    *info = in;
    return LSCOMP_OK;
}

int lscomp_compress_container(lscomp_workspace *ws, uint32_t elem_bytes, const void *d_in, uint32_t x, uint32_t y,
                              uint32_t z, const uint32_t bins[4], float pooling, uint8_t *d_out, uint64_t cap,
                              uint64_t *container_len, void *stream)
{
    if (!d_out || cap < kHdr || ((uintptr_t)d_out & 3u)) return LSCOMP_ERR_ARG;
    uint64_t len = 0, ref = 0;
    int s;
    if (elem_bytes == 2)
        s = lscomp_compress_u16(ws, (const uint16_t *)d_in, x, y, z, bins, pooling, d_out + kHdr, cap - kHdr, &len,
                                &ref, stream);
    else if (elem_bytes == 4)
        s = lscomp_compress_u32(ws, (const uint32_t *)d_in, x, y, z, bins, pooling, d_out + kHdr, cap - kHdr, &len,
                                &ref, stream);
    else
        return LSCOMP_ERR_ARG;
    if (s) return s;
    uint8_t hdr[kHdr];
    s = lscomp_container_write_header(hdr, elem_bytes, x, y, z, bins, pooling, len, ref);
    if (s) return s;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaMemcpyAsync(d_out, hdr, kHdr, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // hdr lives on this stack frame
    if (e != cudaSuccess) return status_of(e);
    if (container_len) *container_len = kHdr + len;
    return LSCOMP_OK;
}

int lscomp_decompress_container(lscomp_workspace *ws, const uint8_t *d_in, uint64_t len, void *d_out,
                                uint64_t out_cap, lscomp_container_info *info, void *stream)
{
    if (!d_in || !d_out || len < kHdr) return LSCOMP_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    uint8_t hdr[kHdr];
    cudaError_t e = cudaMemcpyAsync(hdr, d_in, kHdr, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return status_of(e);
    lscomp_container_info in;
    int s = lscomp_container_read_header(hdr, len, &in);
    if (s) return s;
    if (out_cap < (uint64_t)in.x * in.y * in.z * in.elem_bytes) return LSCOMP_ERR_CAPACITY;
    if (in.elem_bytes == 2)
        s = lscomp_decompress_u16(ws, d_in + kHdr, in.stream_len, in.x, in.y, in.z, in.bins, in.pooling,
                                  (uint16_t *)d_out, stream);
    else
        s = lscomp_decompress_u32(ws, d_in + kHdr, in.stream_len, in.x, in.y, in.z, in.bins, in.pooling,
                                  (uint32_t *)d_out, stream);
    if (!s && info) *info = in;
    return s;
}

}  // extern "C"
