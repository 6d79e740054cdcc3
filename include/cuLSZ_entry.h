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

/* Stream capacity: these functions take none, like the reference's, and
   treat d_cmpBytes as holding the worst-case stream -- roundup4(nb) + 128 nb
   bytes for uint16, roundup4(nb) + 248 nb for uint32, nb = X ceil(Y/8)
   ceil(Z/8) (lscomp_max_stream_bytes_u16/_u32 in lscomp.h).  A caller that
   allocates less (the reference's CLIs allocate X Y Z sizeof(T) bytes,
   lsCOMP/example/lsCOMP_xpcs.cpp:137, which is smaller for incompressible
   data) is not protected from an overrun, exactly as with the reference;
   the C ABI's calls take the capacity and refuse instead of overrunning. */
void cuLSZ_compression_uint32_bsize64(uint32_t* d_oriData, unsigned char* d_cmpBytes, size_t* cmpSize, uint3 dims, uint4 quantBins, float poolingSH, cudaStream_t stream=0);
void cuLSZ_decompression_uint32_bsize64(uint32_t* d_decData, unsigned char* d_cmpBytes, size_t cmpSize, uint3 dims, uint4 quantBins, float poolingSH, cudaStream_t stream=0);
void cuLSZ_compression_uint16_bsize64(uint16_t* d_oriData, unsigned char* d_cmpBytes, size_t* cmpSize, uint3 dims, uint4 quantBins, float poolingSH, cudaStream_t stream=0);
void cuLSZ_decompression_uint16_bsize64(uint16_t* d_decData, unsigned char* d_cmpBytes, size_t cmpSize, uint3 dims, uint4 quantBins, float poolingSH, cudaStream_t stream=0);

#endif // CULSZ_INCLUDE_CULSZ_ENTRY_H
