/*
 * cuLSZ_kernel.h -- the reference's public kernel header
 * (lsCOMP/include/cuLSZ_kernel.h:1-39), for callers that launch the codec
 * kernels themselves instead of calling the host API (cuLSZ_entry.h).
 *
 * The declarations repeat the reference's names and signatures so such a
 * caller builds and links against liblscomp.so unchanged.  The kernels are
 * this library's own (csrc/culsz_kernels.cu), written for the reference's
 * launch contract and producing the reference's stream byte for byte:
 *
 *   grid  = ceil(blockNum / (32 * block_per_thread)) CTAs of 32 threads
 *           (one CTA per 1024 8x8 blocks, blockNum = X * ceil(Y/8) * ceil(Z/8));
 *   cmpOffset, locOffset, flag: caller-allocated scratch of grid + 1
 *           entries each, zeroed before every launch;
 *   after a compression launch cmpOffset[grid] holds the payload bytes, so
 *           the reference's reported size is cmpOffset[grid] + blockNum
 *           (lsCOMP/src/cuLSZ_entry.cu:124-125).  The reference leaves it 0
 *           for a one-CTA grid (blockNum <= 1024); these kernels write it for
 *           every grid.
 *
 * Differences a caller can observe, all on inputs where the reference's own
 * result is undefined: the zero pad between the header and the payload is
 * written, blocks of rate 0 are decoded as zeros, and every wait is bounded
 * (2 s): a kernel that would wait longer returns with flag[grid] marked
 * instead of spinning (the reference spins without a bound,
 * lsCOMP/src/cuLSZ_kernel.cu:1001-1004).  flag[grid] also serves as the
 * launch's CTA ticket, so CTAs process their 1024 blocks in claim order.
 *
 * The host API (cuLSZ_entry.h) does not use these kernels; it runs the
 * persistent B200 kernels behind include/lscomp.h.
 */
#ifndef CULSZ_INCLUDE_CULSZ_KERNEL_H
#define CULSZ_INCLUDE_CULSZ_KERNEL_H

#include <stdint.h>
#include <cuda_runtime.h>

static const int block_per_thread = 32;

__global__ void cuLSZ_compression_kernel_uint32_bsize64(const uint32_t* const __restrict__ oriData,
                                                        unsigned char* const __restrict__ cmpBytes,
                                                        volatile unsigned int* const __restrict__ cmpOffset,
                                                        volatile unsigned int* const __restrict__ locOffset,
                                                        volatile int* const __restrict__ flag,
                                                        uint blockNum, const uint3 dims,
                                                        const uint4 quantBins, const float poolingTH);
__global__ void cuLSZ_decompression_kernel_uint32_bsize64(uint32_t* const __restrict__ decData,
                                                        const unsigned char* const __restrict__ cmpBytes,
                                                        volatile unsigned int* const __restrict__ cmpOffset,
                                                        volatile unsigned int* const __restrict__ locOffset,
                                                        volatile int* const __restrict__ flag,
                                                        uint blockNum, const uint3 dims,
                                                        const uint4 quantBins, const float poolingTH);
__global__ void cuLSZ_compression_kernel_uint16_bsize64(const uint16_t* const __restrict__ oriData,
                                                        unsigned char* const __restrict__ cmpBytes,
                                                        volatile size_t* const __restrict__ cmpOffset,
                                                        volatile size_t* const __restrict__ locOffset,
                                                        volatile int* const __restrict__ flag,
                                                        uint blockNum, const uint3 dims,
                                                        const uint4 quantBins, const float poolingTH);
__global__ void cuLSZ_decompression_kernel_uint16_bsize64(uint16_t* const __restrict__ decData,
                                                        const unsigned char* const __restrict__ cmpBytes,
                                                        volatile size_t* const __restrict__ cmpOffset,
                                                        volatile size_t* const __restrict__ locOffset,
                                                        volatile int* const __restrict__ flag,
                                                        uint blockNum, const uint3 dims,
                                                        const uint4 quantBins, const float poolingTH);

#endif  // CULSZ_INCLUDE_CULSZ_KERNEL_H
