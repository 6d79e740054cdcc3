// ref_driver.cu -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// C-linkage wrappers around the reference's own public host API
// (lsCOMP/include/cuLSZ_entry.h:8-11), compiled together with the
// unmodified reference sources into oracle/_ref/ so that Python tests and
// bench.py's reference arm can call the reference through ctypes.  Nothing
// here changes what the reference computes; the wrappers only forward the
// arguments and report cudaGetLastError().
#include <cstdint>
#include <cstddef>
#include <cuda_runtime.h>
#include "cuLSZ_entry.h"

extern "C" {

int ref_compress_u16(void *d_in, void *d_cmp, size_t *cmp_size, unsigned x, unsigned y, unsigned z,
                     const unsigned bins[4], float p, void *stream)
{
    uint3 dims = make_uint3(x, y, z);
    uint4 qb = make_uint4(bins[0], bins[1], bins[2], bins[3]);
    cuLSZ_compression_uint16_bsize64((uint16_t *)d_in, (unsigned char *)d_cmp, cmp_size, dims, qb, p,
                                     (cudaStream_t)stream);
    return (int)cudaGetLastError();
}

int ref_decompress_u16(void *d_out, void *d_cmp, size_t cmp_size, unsigned x, unsigned y, unsigned z,
                       const unsigned bins[4], float p, void *stream)
{
    uint3 dims = make_uint3(x, y, z);
    uint4 qb = make_uint4(bins[0], bins[1], bins[2], bins[3]);
    cuLSZ_decompression_uint16_bsize64((uint16_t *)d_out, (unsigned char *)d_cmp, cmp_size, dims, qb, p,
                                       (cudaStream_t)stream);
    return (int)cudaGetLastError();
}

int ref_compress_u32(void *d_in, void *d_cmp, size_t *cmp_size, unsigned x, unsigned y, unsigned z,
                     const unsigned bins[4], float p, void *stream)
{
    uint3 dims = make_uint3(x, y, z);
    uint4 qb = make_uint4(bins[0], bins[1], bins[2], bins[3]);
    cuLSZ_compression_uint32_bsize64((uint32_t *)d_in, (unsigned char *)d_cmp, cmp_size, dims, qb, p,
                                     (cudaStream_t)stream);
    return (int)cudaGetLastError();
}

int ref_decompress_u32(void *d_out, void *d_cmp, size_t cmp_size, unsigned x, unsigned y, unsigned z,
                       const unsigned bins[4], float p, void *stream)
{
    uint3 dims = make_uint3(x, y, z);
    uint4 qb = make_uint4(bins[0], bins[1], bins[2], bins[3]);
    cuLSZ_decompression_uint32_bsize64((uint32_t *)d_out, (unsigned char *)d_cmp, cmp_size, dims, qb, p,
                                       (cudaStream_t)stream);
    return (int)cudaGetLastError();
}

}  // extern "C"
