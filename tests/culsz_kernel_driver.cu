// Test helper: launches the kernels of include/cuLSZ_kernel.h the way a
// caller of the reference's kernel header does (the reference's own host
// code, lsCOMP/src/cuLSZ_entry.cu:93-166, launches its kernels so): one
// 32-thread CTA per 1024 blocks, three zeroed scratch arrays of grid + 1
// entries, the payload size read from cmpOffset[grid].  Built and loaded by
// tests/test_kernel_header.py; C linkage for ctypes.
#include <cuda_runtime.h>
#include <stdint.h>
#include "cuLSZ_kernel.h"

template <typename T, typename OffT>
static int run(bool comp, T *data, unsigned char *cmp, size_t *cmpSize, unsigned x, unsigned y, unsigned z,
               const unsigned *bins, float p, int *flag_end)
{
    const uint3 dims = make_uint3(x, y, z);
    const uint4 qb = make_uint4(bins[0], bins[1], bins[2], bins[3]);
    const unsigned nb = x * ((y + 7) / 8) * ((z + 7) / 8);
    const unsigned grid = (nb + 32 * block_per_thread - 1) / (32 * block_per_thread);
    OffT *cmpOffset = nullptr, *locOffset = nullptr;
    int *flag = nullptr;
    cudaMalloc(&cmpOffset, sizeof(OffT) * (grid + 1));
    cudaMalloc(&locOffset, sizeof(OffT) * (grid + 1));
    cudaMalloc(&flag, sizeof(int) * (grid + 1));
    cudaMemset(cmpOffset, 0, sizeof(OffT) * (grid + 1));
    cudaMemset(locOffset, 0, sizeof(OffT) * (grid + 1));
    cudaMemset(flag, 0, sizeof(int) * (grid + 1));
    if (comp) {
        if constexpr (sizeof(T) == 2)
            cuLSZ_compression_kernel_uint16_bsize64<<<grid, 32, sizeof(OffT) * 2>>>(data, cmp, cmpOffset, locOffset,
                                                                                   flag, nb, dims, qb, p);
        else
            cuLSZ_compression_kernel_uint32_bsize64<<<grid, 32, sizeof(OffT) * 2>>>(data, cmp, cmpOffset, locOffset,
                                                                                   flag, nb, dims, qb, p);
    } else {
        if constexpr (sizeof(T) == 2)
            cuLSZ_decompression_kernel_uint16_bsize64<<<grid, 32, sizeof(OffT) * 2>>>(data, cmp, cmpOffset, locOffset,
                                                                                     flag, nb, dims, qb, p);
        else
            cuLSZ_decompression_kernel_uint32_bsize64<<<grid, 32, sizeof(OffT) * 2>>>(data, cmp, cmpOffset, locOffset,
                                                                                     flag, nb, dims, qb, p);
    }
    int st = (int)cudaGetLastError();
    OffT total = 0;
    if (!st) st = (int)cudaMemcpy(&total, cmpOffset + grid, sizeof(OffT), cudaMemcpyDeviceToHost);
    if (!st) st = (int)cudaMemcpy(flag_end, flag + grid, sizeof(int), cudaMemcpyDeviceToHost);
    if (cmpSize) *cmpSize = (size_t)total + nb;
    cudaFree(cmpOffset);
    cudaFree(locOffset);
    cudaFree(flag);
    return st;
}

extern "C" {
int kdrv_compress_u16(uint16_t *d_in, unsigned char *d_cmp, size_t *cmpSize, unsigned x, unsigned y, unsigned z,
                      const unsigned *bins, float p, int *flag_end)
{
    return run<uint16_t, size_t>(true, d_in, d_cmp, cmpSize, x, y, z, bins, p, flag_end);
}
int kdrv_decompress_u16(uint16_t *d_out, unsigned char *d_cmp, unsigned x, unsigned y, unsigned z,
                        const unsigned *bins, float p, int *flag_end)
{
    return run<uint16_t, size_t>(false, d_out, d_cmp, nullptr, x, y, z, bins, p, flag_end);
}
int kdrv_compress_u32(uint32_t *d_in, unsigned char *d_cmp, size_t *cmpSize, unsigned x, unsigned y, unsigned z,
                      const unsigned *bins, float p, int *flag_end)
{
    return run<uint32_t, unsigned int>(true, d_in, d_cmp, cmpSize, x, y, z, bins, p, flag_end);
}
int kdrv_decompress_u32(uint32_t *d_out, unsigned char *d_cmp, unsigned x, unsigned y, unsigned z,
                        const unsigned *bins, float p, int *flag_end)
{
    return run<uint32_t, unsigned int>(false, d_out, d_cmp, nullptr, x, y, z, bins, p, flag_end);
}
}
