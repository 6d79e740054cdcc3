// lscomp_cli.cpp -- the lsCOMP command-line tools on the B200 codec:
//   lsCOMP_xpcs   uint16 stacks (built with LSC_CLI_WIDE=0)
//   lsCOMP_cssi   uint32 stacks (built with LSC_CLI_WIDE=1)
//
// Same arguments, checks, messages, exit codes and report lines as the
// reference tools (lsCOMP/example/lsCOMP_xpcs.cpp, lsCOMP_cssi.cpp), so scripts
// that drive or parse them keep working:
//   -i input file, -d x y z (z fastest), -b four bins x <= y <= z <= w,
//   -p pooling threshold in [0, 1], optional -o decoded output file.
// The tool reads the file, runs 3 warm-up compressions, times one
// compression and one decompression (CUDA events on the default stream around
// the whole host call, like the reference), moves the stream to the host and
// back in between, and prints throughput in MiB/ms ("GB/s") and the ratio.
//
// One deliberate difference: the stream copied through the host is the whole
// stream (reported size + the header pad), where the reference copies only
// the reported size and can drop the last 1-3 payload bytes when the block
// count is not a multiple of 4.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "cuLSZ_entry.h"
#include "cuLSZ_timer.h"
#include "cuLSZ_utility.h"
#include "lscomp.h"

#ifndef LSC_CLI_WIDE
#define LSC_CLI_WIDE 0
#endif

#if LSC_CLI_WIDE
typedef uint32_t elem_t;
static elem_t *read_input(char *path, size_t *n, int *st) { return readUInt32Data_Yafan(path, n, st); }
static void write_output(elem_t *d, size_t n, char *path, int *st) { writeUIntData_inBytes_Yafan(d, n, path, st); }
static void compress(elem_t *i, unsigned char *o, size_t *s, uint3 d, uint4 b, float p, cudaStream_t st)
{
    cuLSZ_compression_uint32_bsize64(i, o, s, d, b, p, st);
}
static void decompress(elem_t *o, unsigned char *i, size_t s, uint3 d, uint4 b, float p, cudaStream_t st)
{
    cuLSZ_decompression_uint32_bsize64(o, i, s, d, b, p, st);
}
static uint64_t worst_stream(uint3 d) { return lscomp_max_stream_bytes_u32(d.x, d.y, d.z); }
#else
typedef uint16_t elem_t;
static elem_t *read_input(char *path, size_t *n, int *st) { return readUInt16Data_Yafan(path, n, st); }
static void write_output(elem_t *d, size_t n, char *path, int *st) { writeUShortData_inBytes_Yafan(d, n, path, st); }
static void compress(elem_t *i, unsigned char *o, size_t *s, uint3 d, uint4 b, float p, cudaStream_t st)
{
    cuLSZ_compression_uint16_bsize64(i, o, s, d, b, p, st);
}
static void decompress(elem_t *o, unsigned char *i, size_t s, uint3 d, uint4 b, float p, cudaStream_t st)
{
    cuLSZ_decompression_uint16_bsize64(o, i, s, d, b, p, st);
}
static uint64_t worst_stream(uint3 d) { return lscomp_max_stream_bytes_u16(d.x, d.y, d.z); }
#endif

static void usage(const char *prog)
{
    fprintf(stderr, "Usage:\n");
    fprintf(stderr, "   %s -i oriFilePath -d dims.x dims.y dims.z -b quantBins.x quantBins.y quantBins.z quantBins.w -p value -o decFilePath\n", prog);
    fprintf(stderr, "Options:\n");
    fprintf(stderr, "   -i oriFilePath: Path to the original data file\n");
    fprintf(stderr, "   -d dims.x dims.y dims.z: Dimensions of the original data, where dim.z is the fastest dimension.\n");
    fprintf(stderr, "   -b quantBins.x quantBins.y quantBins.z quantBins.w: Quantization bins for the 4 levels, where x is the base one and x<=y<=z<=w.\n");
    fprintf(stderr, "   -p value: Pooling threshold for a data block.\n");
    fprintf(stderr, "   -o decFilePath: Path to the decompressed data file (optional).\n");
    fprintf(stderr, "Examples:\n");
#if LSC_CLI_WIDE
    fprintf(stderr, "   %s -i data/cssi.bin -d 600 1813 1558 -b 3 5 10 15 -p 0.5\n", prog);
    fprintf(stderr, "   %s -i data/cssi.bin -d 600 1813 1558 -b 3 5 10 15 -p 0.5 -o data/cssi-dec.bin\n", prog);
#else
    fprintf(stderr, "   %s -i data/xpcs.bin -d 1024 1813 1558 -b 3 5 10 15 -p 0.5\n", prog);
    fprintf(stderr, "   %s -i data/xpcs.bin -d 1024 1813 1558 -b 3 5 10 15 -p 0.5 -o data/xpcs-dec.bin\n", prog);
#endif
}

int main(int argc, char *argv[])
{
    char oriFilePath[640] = {0};
    char decFilePath[640] = {0};
    uint3 dims = {0, 0, 0};
    uint4 quantBins = {0, 0, 0, 0};
    float poolingTH = 0.0f;
    int status = 0;

    if (argc < 13) {
        usage(argv[0]);
        return 1;
    }
    for (int i = 1; i < argc; i++) {
        if (strcmp(argv[i], "-i") == 0) {
            if (i + 1 >= argc) { fprintf(stderr, "Error: Missing value for -i\n"); return 1; }
            strncpy(oriFilePath, argv[++i], sizeof(oriFilePath) - 1);
        } else if (strcmp(argv[i], "-d") == 0) {
            if (i + 3 >= argc) { fprintf(stderr, "Error: Missing values for -d\n"); return 1; }
            int x = atoi(argv[i + 1]), y = atoi(argv[i + 2]), z = atoi(argv[i + 3]);
            if (x <= 0 || y <= 0 || z <= 0) {
                fprintf(stderr, "Error: -d values must be positive integers\n");
                return 1;
            }
            dims = make_uint3((unsigned)x, (unsigned)y, (unsigned)z);
            i += 3;
        } else if (strcmp(argv[i], "-b") == 0) {
            if (i + 4 >= argc) { fprintf(stderr, "Error: Missing values for -b\n"); return 1; }
            int b0 = atoi(argv[i + 1]), b1 = atoi(argv[i + 2]), b2 = atoi(argv[i + 3]), b3 = atoi(argv[i + 4]);
            if (b0 <= 0 || b1 <= 0 || b2 <= 0 || b3 <= 0) {
                fprintf(stderr, "Error: -b values must be positive integers\n");
                return 1;
            }
            if (!(b0 <= b1 && b1 <= b2 && b2 <= b3)) {
                fprintf(stderr, "Error: -b values must satisfy x <= y <= z <= w\n");
                return 1;
            }
            quantBins = make_uint4((unsigned)b0, (unsigned)b1, (unsigned)b2, (unsigned)b3);
            i += 4;
        } else if (strcmp(argv[i], "-p") == 0) {
            if (i + 1 >= argc) { fprintf(stderr, "Error: Missing value for -p\n"); return 1; }
            poolingTH = (float)atof(argv[++i]);
            if (poolingTH < 0.0f || poolingTH > 1.0f) {
                fprintf(stderr, "Error: -p value must be between 0 and 1\n");
                return 1;
            }
        } else if (strcmp(argv[i], "-o") == 0) {
            if (i + 1 >= argc) { fprintf(stderr, "Error: Missing value for -o\n"); return 1; }
            strncpy(decFilePath, argv[++i], sizeof(decFilePath) - 1);
        } else {
            fprintf(stderr, "Error: Unknown argument %s\n", argv[i]);
            return 1;
        }
    }

    size_t nbEle = 0, cmpSize = 0;
    elem_t *oriData = read_input(oriFilePath, &nbEle, &status);
    if (!oriData || nbEle != (size_t)dims.x * (size_t)dims.y * (size_t)dims.z) {
        fprintf(stderr, "Error: The number of elements in the original data does not match the dimensions\n");
        free(oriData);
        return 1;
    }
    const size_t dataBytes = nbEle * sizeof(elem_t);
    // the reference sizes the stream buffer like the input; the worst case
    // (incompressible data plus headers) can exceed that, so take the larger
    size_t cmpCap = (size_t)worst_stream(dims);
    if (cmpCap < dataBytes) cmpCap = dataBytes;
    const uint64_t nb = lscomp_block_count(dims.x, dims.y, dims.z);
    const size_t pad = (size_t)((nb + 3) / 4 * 4 - nb);

    elem_t *decData = (elem_t *)malloc(dataBytes);
    elem_t *d_oriData = nullptr, *d_decData = nullptr;
    unsigned char *d_cmpBytes = nullptr;
    if (cudaMalloc((void **)&d_oriData, dataBytes) != cudaSuccess ||
        cudaMalloc((void **)&d_decData, dataBytes) != cudaSuccess ||
        cudaMalloc((void **)&d_cmpBytes, cmpCap) != cudaSuccess) {
        fprintf(stderr, "Error: device allocation failed\n");
        return 1;
    }
    cudaMemcpy(d_oriData, oriData, dataBytes, cudaMemcpyHostToDevice);
    cudaStream_t stream;
    cudaStreamCreate(&stream);

    TimingGPU timer_GPU;
    for (int i = 0; i < 3; i++) compress(d_oriData, d_cmpBytes, &cmpSize, dims, quantBins, poolingTH, stream);
    printf("GPU warmup finished!\n\n");

    timer_GPU.StartCounter();
    compress(d_oriData, d_cmpBytes, &cmpSize, dims, quantBins, poolingTH, stream);
    float cmpTime = timer_GPU.GetCounter();

    // stream to the host and back (checks that the reported size covers it)
    const size_t streamLen = cmpSize + pad;
    unsigned char *cmpBytes = (unsigned char *)malloc(streamLen);
    cudaMemcpy(cmpBytes, d_cmpBytes, streamLen, cudaMemcpyDeviceToHost);
    cudaMemset(d_cmpBytes, 0, cmpCap);
    cudaMemcpy(d_cmpBytes, cmpBytes, streamLen, cudaMemcpyHostToDevice);

    timer_GPU.StartCounter();
    decompress(d_decData, d_cmpBytes, cmpSize, dims, quantBins, poolingTH, stream);
    float decTime = timer_GPU.GetCounter();

    printf("Dataset information:\n");
    printf("  - dims:   %u x %u x %u\n", dims.x, dims.y, dims.z);
    printf("  - length: %zu\n", nbEle);
    printf("  - size:   %f GB\n", dataBytes / 1024.0 / 1024.0 / 1024.0);
    printf("Input arguments:\n");
    printf("  - quantBins: %u %u %u %u\n", quantBins.x, quantBins.y, quantBins.z, quantBins.w);
    printf("  - poolingTH: %f\n\n", poolingTH);
    printf("cuLSZ compression   end-to-end speed: %f GB/s\n", (dataBytes / 1024.0 / 1024.0) / cmpTime);
    printf("cuLSZ decompression end-to-end speed: %f GB/s\n", (dataBytes / 1024.0 / 1024.0) / decTime);
    printf("cuLSZ compression ratio: %f\n", (dataBytes / 1024.0 / 1024.0) / (cmpSize / 1024.0 / 1024.0));

    if (strlen(decFilePath) > 0) {
        cudaMemcpy(decData, d_decData, dataBytes, cudaMemcpyDeviceToHost);
        write_output(decData, nbEle, decFilePath, &status);
    }

    free(oriData);
    free(decData);
    free(cmpBytes);
    cudaFree(d_oriData);
    cudaFree(d_decData);
    cudaFree(d_cmpBytes);
    cudaStreamDestroy(stream);
    return 0;
}
