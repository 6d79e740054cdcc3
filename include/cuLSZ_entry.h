/*
 * cuLSZ_entry.h -- drop-in host API with the reference's exact C++
 * signatures (same mangled symbols), so programs written against
 * lsCOMP/include/cuLSZ_entry.h:8-11 relink against liblscomp unchanged.
 *
 * Differences from the reference, all deliberate:
 *   - scan scratch comes from a cached per-(device, stream) workspace
 *     instead of cudaMalloc/cudaMemset/cudaFree on every call
 *     (lsCOMP/src/cuLSZ_entry.cu:105-114,128-130);
 *   - *cmpSize is payload + nb for every size; the reference reports nb
 *     alone when nb <= 1024 (it never stores the total for a single tile);
 *   - the header pad bytes and rate-0 blocks are written as zeros;
 *   - errors print a message and exit with the status, as the reference's
 *     check() does for launch errors (lsCOMP/src/cuLSZ_entry.cu:9-15).
 */
#ifndef CULSZ_INCLUDE_CULSZ_ENTRY_H
#define CULSZ_INCLUDE_CULSZ_ENTRY_H

#include <stdint.h>
#include <stddef.h>
#include <cuda_runtime.h>

void cuLSZ_compression_uint32_bsize64(uint32_t* d_oriData, unsigned char* d_cmpBytes, size_t* cmpSize, uint3 dims, uint4 quantBins, float poolingSH, cudaStream_t stream=0);
void cuLSZ_decompression_uint32_bsize64(uint32_t* d_decData, unsigned char* d_cmpBytes, size_t cmpSize, uint3 dims, uint4 quantBins, float poolingSH, cudaStream_t stream=0);
void cuLSZ_compression_uint16_bsize64(uint16_t* d_oriData, unsigned char* d_cmpBytes, size_t* cmpSize, uint3 dims, uint4 quantBins, float poolingSH, cudaStream_t stream=0);
void cuLSZ_decompression_uint16_bsize64(uint16_t* d_decData, unsigned char* d_cmpBytes, size_t cmpSize, uint3 dims, uint4 quantBins, float poolingSH, cudaStream_t stream=0);

#endif // CULSZ_INCLUDE_CULSZ_ENTRY_H
