/*
 * lscomp.h -- C ABI of the B200-native lsCOMP codec (uint16 detector stacks).
 *
 * Plain C: pointers, sizes, an opaque workspace and a CUDA stream passed as
 * void*.  All data pointers are device pointers unless stated otherwise.
 * Every entry point returns an lscomp_status.
 *
 * Stream format (unchanged from the reference, lsCOMP/src/cuLSZ_kernel.cu):
 *   [nb header bytes][zero pad to a multiple of 4][payload blocks in block order]
 * with nb = X * ceil(Y/8) * ceil(Z/8) blocks of 8x8 values (z fastest).
 * Header byte = pool << 7 | bin_choice << 5 | rate.
 *
 * Entry points and the reference interface each replaces:
 *   lscomp_compress_u16 / _async     cuLSZ_compression_uint16_bsize64
 *                                    (lsCOMP/include/cuLSZ_entry.h:10,
 *                                     lsCOMP/src/cuLSZ_entry.cu:93-131)
 *   lscomp_decompress_u16 / _async   cuLSZ_decompression_uint16_bsize64
 *                                    (lsCOMP/include/cuLSZ_entry.h:11,
 *                                     lsCOMP/src/cuLSZ_entry.cu:133-166)
 *   lscomp_compress_u32 / _async     cuLSZ_compression_uint32_bsize64
 *                                    (lsCOMP/include/cuLSZ_entry.h:8, cuLSZ_entry.cu:18-56)
 *   lscomp_decompress_u32 / _async   cuLSZ_decompression_uint32_bsize64
 *                                    (lsCOMP/include/cuLSZ_entry.h:9, cuLSZ_entry.cu:58-91)
 *   lscomp_workspace_*               the per-call cudaMalloc/cudaMemset/cudaFree
 *                                    of the scan scratch (cuLSZ_entry.cu:105-114,
 *                                    128-130), made reusable
 */
#ifndef LSCOMP_H
#define LSCOMP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    LSCOMP_OK = 0,
    LSCOMP_ERR_ARG = 1,      /* bad dimension, bin, pointer alignment or size */
    LSCOMP_ERR_CAPACITY = 2, /* output (or readable input) too small for the stream */
    LSCOMP_ERR_CUDA = 3,     /* a CUDA runtime call failed */
    LSCOMP_ERR_TIMEOUT = 4,  /* a bounded wait inside a kernel ran out */
    LSCOMP_ERR_CORRUPT = 5,  /* stream inconsistent with the given geometry */
    LSCOMP_ERR_RANGE = 6,    /* values the stream format cannot represent */
    LSCOMP_ERR_NOMEM = 7,    /* device or host allocation failed */
    LSCOMP_ERR_TOO_LARGE = 8 /* stack larger than a fixed-size scratch area allows */
} lscomp_status;

typedef struct lscomp_workspace lscomp_workspace;

/* library version, e.g. 100 for 0.1.0 */
int lscomp_version(void);
const char *lscomp_status_string(int status);

/* number of 8x8 blocks of an X x Y x Z stack */
uint64_t lscomp_block_count(uint32_t x, uint32_t y, uint32_t z);
/* worst-case stream length for uint16 data: roundup4(nb) + 128 * nb */
uint64_t lscomp_max_stream_bytes_u16(uint32_t x, uint32_t y, uint32_t z);

/* A workspace holds the scan state of one stream of calls (about 8 bytes
   per tile) on one device.  Calls that share a workspace must be ordered
   (same CUDA stream, or synchronised).  device < 0 means the current device. */
int lscomp_workspace_create(lscomp_workspace **ws, int device);
int lscomp_workspace_destroy(lscomp_workspace *ws);

/* Compress.  d_in: X*Y*Z uint16 (2-byte aligned).  bins: four bins > 0.
   pooling: the -p threshold (a block pools iff (float)zeros/64 > pooling).
   d_out: cap bytes.  On success *stream_len = bytes of the stream and
   *ref_size = payload + nb, the value the reference's host API reports
   (either pointer may be NULL).  Synchronises the stream. */
int lscomp_compress_u16(lscomp_workspace *ws, const uint16_t *d_in, uint32_t x, uint32_t y, uint32_t z,
                        const uint32_t bins[4], float pooling, uint8_t *d_out, uint64_t cap,
                        uint64_t *stream_len, uint64_t *ref_size, void *stream);

/* Same work without any host synchronisation: {stream_len, payload bytes}
   are written to d_sizes[0..1] (device memory, may be NULL) when the kernel
   finishes; errors are read later with lscomp_workspace_check. */
int lscomp_compress_u16_async(lscomp_workspace *ws, const uint16_t *d_in, uint32_t x, uint32_t y,
                              uint32_t z, const uint32_t bins[4], float pooling, uint8_t *d_out,
                              uint64_t cap, uint64_t *d_sizes, void *stream);

/* Decompress.  d_in: stream, cmp_len readable bytes (the stream length, or
   more).  Writes every element of d_out (X*Y*Z uint16), zero for blocks of
   rate 0.  Synchronises the stream. */
int lscomp_decompress_u16(lscomp_workspace *ws, const uint8_t *d_in, uint64_t cmp_len, uint32_t x,
                          uint32_t y, uint32_t z, const uint32_t bins[4], float pooling, uint16_t *d_out,
                          void *stream);

int lscomp_decompress_u16_async(lscomp_workspace *ws, const uint8_t *d_in, uint64_t cmp_len, uint32_t x,
                                uint32_t y, uint32_t z, const uint32_t bins[4], float pooling,
                                uint16_t *d_out, void *stream);

/* uint32 twins (lsCOMP/include/cuLSZ_entry.h:8-9, lsCOMP/src/cuLSZ_entry.cu:18-91).
   Same stream format; a block whose quantised maximum needs 32 bit planes
   (a quotient >= 2^31) cannot be represented in the 5-bit rate field and
   fails with LSCOMP_ERR_RANGE.  Offsets are 64-bit (the reference's are
   32-bit, so the two agree on streams below 4 GiB). */
uint64_t lscomp_max_stream_bytes_u32(uint32_t x, uint32_t y, uint32_t z);
int lscomp_compress_u32(lscomp_workspace *ws, const uint32_t *d_in, uint32_t x, uint32_t y, uint32_t z,
                        const uint32_t bins[4], float pooling, uint8_t *d_out, uint64_t cap,
                        uint64_t *stream_len, uint64_t *ref_size, void *stream);
int lscomp_compress_u32_async(lscomp_workspace *ws, const uint32_t *d_in, uint32_t x, uint32_t y,
                              uint32_t z, const uint32_t bins[4], float pooling, uint8_t *d_out,
                              uint64_t cap, uint64_t *d_sizes, void *stream);
int lscomp_decompress_u32(lscomp_workspace *ws, const uint8_t *d_in, uint64_t cmp_len, uint32_t x,
                          uint32_t y, uint32_t z, const uint32_t bins[4], float pooling, uint32_t *d_out,
                          void *stream);
int lscomp_decompress_u32_async(lscomp_workspace *ws, const uint8_t *d_in, uint64_t cmp_len, uint32_t x,
                                uint32_t y, uint32_t z, const uint32_t bins[4], float pooling,
                                uint32_t *d_out, void *stream);

/* Compression and decompression from and to HOST memory (the reference's
   CLI does this with one blocking copy each way around the device call).
   The stack moves through the device in chunks of whole frames (about
   128 MB each) on two copy streams, so copies up, kernels and copies down
   of different chunks overlap; the stream (h_out, cap bytes) and the
   decoded stack are exactly those of the device-memory calls.  Pinned host
   buffers (cudaMallocHost / cudaHostRegister) let the copies overlap;
   pageable ones work but copy synchronously.  The workspace keeps the copy
   streams and four chunk buffers (about 0.5 GB for uint16) for later
   calls.  Synchronous: returns when every byte is in place. */
int lscomp_compress_host_u16(lscomp_workspace *ws, const uint16_t *h_in, uint32_t x, uint32_t y, uint32_t z,
                             const uint32_t bins[4], float pooling, uint8_t *h_out, uint64_t cap,
                             uint64_t *stream_len, uint64_t *ref_size, void *stream);
int lscomp_compress_host_u32(lscomp_workspace *ws, const uint32_t *h_in, uint32_t x, uint32_t y, uint32_t z,
                             const uint32_t bins[4], float pooling, uint8_t *h_out, uint64_t cap,
                             uint64_t *stream_len, uint64_t *ref_size, void *stream);
int lscomp_decompress_host_u16(lscomp_workspace *ws, const uint8_t *h_in, uint64_t cmp_len, uint32_t x, uint32_t y,
                               uint32_t z, const uint32_t bins[4], float pooling, uint16_t *h_out, void *stream);
int lscomp_decompress_host_u32(lscomp_workspace *ws, const uint8_t *h_in, uint64_t cmp_len, uint32_t x, uint32_t y,
                               uint32_t z, const uint32_t bins[4], float pooling, uint32_t *h_out, void *stream);
/* Input bytes per chunk of the host-memory calls on this workspace (whole
   frames, at least one; 0 restores the default of 128 MB). */
int lscomp_workspace_set_host_chunk(lscomp_workspace *ws, uint64_t bytes);

/* uint16 compression that allocates nothing (no counterpart in the
   reference).  For callers that cannot allocate device memory when they
   compress -- acquisition loops running inside a fixed, pre-reserved memory
   budget, where a cudaMalloc can fail and synchronises the device, or
   processes whose device memory belongs to another allocator.  The scan
   scratch lives in a 2 MiB device array inside the library (per device,
   held until the process exits), which limits the stack to 262,112 tiles
   (about 67 million 8x8 blocks); larger stacks return LSCOMP_ERR_TOO_LARGE.
   Same stream, sizes and synchronisation as lscomp_compress_u16.  All calls
   on a device share the array: calls that overlap on the GPU race (this
   function serialises its own calls within a process).  The first call on a
   device sets up the array's device address; make it before any stream
   capture. */
int lscomp_compress_u16_noalloc(const uint16_t *d_in, uint32_t x, uint32_t y, uint32_t z,
                                const uint32_t bins[4], float pooling, uint8_t *d_out, uint64_t cap,
                                uint64_t *stream_len, uint64_t *ref_size, void *stream);

/* Batch compression (no counterpart in the reference, whose host API takes
   one stack per call).  n stacks of any shapes, all with the same bins and
   pooling threshold, compressed by one persistent launch: the tiles of all
   stacks share the GPU, so many small stacks (a few frames each) cost about
   what one stack of their total size costs, instead of one launch and one
   host round trip each.  Each stack's stream is exactly the stream
   lscomp_compress_u16 / _u32 writes for that stack alone; stream_len[i] and
   ref_size[i] (host arrays of n entries, either may be NULL) receive its
   length and the reference-reported size.  The stacks' input and output
   buffers must not overlap.  Synchronises the stream.  Allocates (once per
   workspace, when a batch is larger than any before) about 120 bytes per
   stack and 4 bytes per tile of device memory, plus pinned staging. */
typedef struct lscomp_stack {
    const void *d_in; /* X*Y*Z elements of the call's type (uint16 or uint32) */
    uint32_t x, y, z; /* dims, z fastest */
    uint8_t *d_out;   /* stream buffer, 4-byte aligned */
    uint64_t cap;     /* its capacity in bytes (lscomp_max_stream_bytes_* is always enough) */
} lscomp_stack;

int lscomp_compress_batch_u16(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n,
                              const uint32_t bins[4], float pooling, uint64_t *stream_len,
                              uint64_t *ref_size, void *stream);
int lscomp_compress_batch_u32(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n,
                              const uint32_t bins[4], float pooling, uint64_t *stream_len,
                              uint64_t *ref_size, void *stream);

/* Batch compression with bins and pooling threshold per stack: bins[4 i ..
   4 i + 3] and pooling[i] belong to stacks[i].  One launch still serves
   all stacks (instantiated for a bins class that covers every stack's:
   lossless and equal bins are special cases of increasing bins); each
   stream equals the single-stack stream with that stack's settings. */
int lscomp_compress_batch_ex_u16(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n,
                                 const uint32_t *bins, const float *pooling, uint64_t *stream_len,
                                 uint64_t *ref_size, void *stream);
int lscomp_compress_batch_ex_u32(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n,
                                 const uint32_t *bins, const float *pooling, uint64_t *stream_len,
                                 uint64_t *ref_size, void *stream);

/* Batch decompression (no counterpart in the reference): n streams decoded
   by two launches (stream offsets for every stack, then one CTA per tile of
   every stack).  stacks[i].d_in = the stream (4-byte aligned), .cap = its
   readable bytes (at least the header), .d_out = X*Y*Z values of the call's
   type, bins[4 i .. 4 i + 3] and pooling[i] its settings.  Every output
   equals lscomp_decompress_u16 / _u32 of that stream alone.  Synchronises
   the stream. */
int lscomp_decompress_batch_u16(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t *bins,
                                const float *pooling, void *stream);
int lscomp_decompress_batch_u32(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t *bins,
                                const float *pooling, void *stream);

/* Exact stream sizes of a batch (no counterpart in the reference): for each
   stack, the number of bytes lscomp_compress_batch_ex_* (or the single-stack
   call) would write with bins[4 i .. 4 i + 3] and pooling[i] -- the header,
   its pad and the payload -- computed by one pass over the inputs that
   writes no stream, so output buffers can be allocated to size instead of
   at the worst case (lscomp_max_stream_bytes_*, about the input's size).
   Only d_in and x, y, z of each stack are used.  A uint32 quotient that
   needs 32 bit planes fails with LSCOMP_ERR_RANGE as compression would.
   Synchronises the stream. */
int lscomp_stream_sizes_batch_u16(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t *bins,
                                  const float *pooling, uint64_t *stream_len, void *stream);
int lscomp_stream_sizes_batch_u32(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t *bins,
                                  const float *pooling, uint64_t *stream_len, void *stream);

/* Graph plans (no counterpart in the reference).  A plan fixes one
   compression -- n stacks (n = 1: the single-stack kernel, n > 1: the batch
   kernel), their buffers and shapes, bins and pooling threshold -- and
   captures it once as a CUDA graph: clearing the scan state, the encoder
   launch and the copy of the sizes and the status to pinned host memory.
   lscomp_plan_run replays the graph on `stream`, waits for it and returns
   the status and the sizes as lscomp_compress_batch_* does; nothing is
   computed or copied on the host per call beyond that.  For loops that
   compress new contents of the same buffers again and again (acquisition
   frames landing in fixed device buffers).  Create runs one ordinary call
   through `ws` first (argument checks, tuning when on; the streams are
   written), then allocates the plan's own scratch (about 12 bytes per tile
   plus the stack table), so plans and workspace calls never share state.
   Replays of one plan are serialised; different plans may run
   concurrently. */
typedef struct lscomp_plan lscomp_plan;
int lscomp_plan_create_u16(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t bins[4],
                           float pooling, void *stream, lscomp_plan **plan);
int lscomp_plan_create_u32(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t bins[4],
                           float pooling, void *stream, lscomp_plan **plan);
/* ... with bins and pooling threshold per stack, as lscomp_compress_batch_ex_* */
int lscomp_plan_create_ex_u16(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t *bins,
                              const float *pooling, void *stream, lscomp_plan **plan);
int lscomp_plan_create_ex_u32(lscomp_workspace *ws, const lscomp_stack *stacks, uint32_t n, const uint32_t *bins,
                              const float *pooling, void *stream, lscomp_plan **plan);
int lscomp_plan_run(lscomp_plan *plan, void *stream, uint64_t *stream_len, uint64_t *ref_size);
int lscomp_plan_destroy(lscomp_plan *plan);

/* Launch-configuration tuner (no counterpart in the reference, whose launch
   shape is fixed).  A configuration is the encoder CTA shape (2 groups of 8,
   7 or -- single stacks -- 13 compute warps; for lossless uint16 single
   stacks also 2 x 8 with shorter code paths for small values) and the most
   8x8 blocks a tile holds (uint16: 256 or 128; uint32: 128 or 64); the
   decoder only has the tile size.  Every
   configuration writes the same stream.  With tuning on (the default;
   environment LSCOMP_AUTOTUNE=0 or lscomp_tune_mode(0) turns it off) the
   first compress / decompress / batch call of a key -- element type, bins
   layout (lossless, equal, increasing, other), pooling on or off, row
   access width, blocks per block-row (single stacks) -- times every
   candidate on the call's own buffers (one untimed and three timed calls
   each, CUDA events) and keeps the fastest for the process; that first
   call therefore synchronises its stream and takes about 16x as long.
   With tuning off, or while the stream is being captured, keys not in the
   table use built-in rules.  lscomp_compress_u16_noalloc uses the table
   but never tunes.
   lscomp_tune_mode: 0 off, 1 on, other values only query; returns the
   previous mode.  lscomp_tune_report writes the table as text (one line per
   key: "es layout pool kind vec bzb -> shape tile_blocks", then
   " | shape tile_blocks ms" per timed candidate; kind 0 compress, 1 batch,
   2 decompress; shape -1 = rule, 0 = 2x8, 1 = 2x7, 2 = 2x13, 3 = 2x8 with
   the short paths) and returns the bytes
   needed including the terminating NUL.  lscomp_tune_save / _load write and
   read that text (load replaces the keys it names; a malformed file changes
   nothing and returns LSCOMP_ERR_ARG).  Single stacks of fewer than 4
   tiles per SM (about 150,000 8x8 blocks of uint16 on B200) are never
   tuned: they use the table or the rules.  lscomp_tune_hits counts the
   calls that found their key in the table. */
int lscomp_tune_mode(int mode);
uint64_t lscomp_tune_hits(void);
int lscomp_tune_clear(void);
uint64_t lscomp_tune_report(char *buf, uint64_t cap);
int lscomp_tune_save(const char *path);
int lscomp_tune_load(const char *path);

/* Container (no counterpart in the reference, whose streams carry neither
   dimensions, bins, pooling threshold nor element type, and whose size is
   returned out of band).  A container is a 64-byte header -- magic "LSCZ",
   version 1, element bytes, x y z, bins, pooling, stream length, reference
   size, CRC-32 of the header, little-endian -- followed by the stream, byte
   for byte unchanged.  Decompression from a container needs no other
   argument. */
typedef struct lscomp_container_info {
    uint32_t elem_bytes; /* 2 (uint16) or 4 (uint32) */
    uint32_t x, y, z;
    uint32_t bins[4];
    float pooling;
    uint64_t stream_len; /* bytes of the stream after the header */
    uint64_t ref_size;   /* the size the reference's host API reports */
} lscomp_container_info;

uint32_t lscomp_container_header_bytes(void);
/* Host functions: fill / parse and check a 64-byte header.  read_header
   takes the container length (or exactly the header length to parse a
   header alone) and returns LSCOMP_ERR_CORRUPT for a wrong magic, version,
   checksum, geometry or a body shorter than the recorded stream. */
int lscomp_container_write_header(uint8_t *hdr, uint32_t elem_bytes, uint32_t x, uint32_t y, uint32_t z,
                                  const uint32_t bins[4], float pooling, uint64_t stream_len, uint64_t ref_size);
int lscomp_container_read_header(const uint8_t *hdr, uint64_t len, lscomp_container_info *info);
/* Compress d_in (elem_bytes 2 or 4) into a container at d_out (4-byte
   aligned, cap bytes; the stream starts 64 bytes in).  Synchronises. */
int lscomp_compress_container(lscomp_workspace *ws, uint32_t elem_bytes, const void *d_in, uint32_t x, uint32_t y,
                              uint32_t z, const uint32_t bins[4], float pooling, uint8_t *d_out, uint64_t cap,
                              uint64_t *container_len, void *stream);
/* Decompress a container of len bytes at d_in into d_out (out_cap bytes);
   *info (may be NULL) receives the header.  Synchronises. */
int lscomp_decompress_container(lscomp_workspace *ws, const uint8_t *d_in, uint64_t len, void *d_out,
                                uint64_t out_cap, lscomp_container_info *info, void *stream);

/* Serving loop (no counterpart in the reference).  A server owns a device
   arena of arena_bytes, 2 x 128 MB of pinned staging (whatever the arena's
   size), a workspace, three CUDA streams and three pipeline threads.  Any
   thread submits requests with host buffers.  The uploader admits waiting
   requests in arrival order as soon as the arena has room for a request's
   worst-case device footprint (input + largest possible output) and copies
   its input up; the launcher runs every request uploaded so far as batch
   launches (the compress requests of one element type as one launch, each
   stack with its own shape, bins and pooling threshold; the decompress
   requests of one element type as another) and, when a batch fails, runs
   its requests again one at a time so a bad request fails alone; the
   downloader copies each output down and releases its arena space.  So
   requests that arrive while others are on the GPU are admitted as memory
   frees, and their copies overlap the kernels of others.  A compress
   request produces a container (see above) in h_out; a decompress request
   takes a container.  Outputs do not depend on what else is in the batch.
   Submit returns a request id > 0, or minus a status (LSCOMP_ERR_TOO_LARGE:
   the footprint exceeds the arena).  Caller buffers must stay valid until
   lscomp_server_wait returns for the request; one thread waits for a given
   request (a second waiter gets LSCOMP_ERR_ARG), and wait releases it.
   destroy runs what was submitted.  Environment: LSCOMP_SERVER_COPY_THREADS
   (default 8) host threads per direction copy between caller buffers and
   staging.  A caller buffer that is page-locked host memory (one
   cudaHostAlloc / cudaHostRegister allocation, or a pinned tensor) is
   copied to or from the device directly instead, with no staging and no
   host-thread copy. */
typedef struct lscomp_server lscomp_server;
typedef struct lscomp_server_result {
    int status;          /* LSCOMP_OK or the request's error */
    uint64_t out_len;    /* bytes written to h_out */
    uint64_t queued_ns;  /* submit -> admitted */
    uint64_t service_ns; /* admitted -> done (copies, kernels, copies) */
    uint64_t admit_ns;   /* when it was admitted and when it was done, on the */
    uint64_t done_ns;    /* host's monotonic clock (ns): compare requests */
} lscomp_server_result;

int lscomp_server_create(lscomp_server **server, int device, uint64_t arena_bytes);
int lscomp_server_destroy(lscomp_server *server);
int64_t lscomp_server_submit_compress(lscomp_server *server, uint32_t elem_bytes, const void *h_in, uint32_t x,
                                      uint32_t y, uint32_t z, const uint32_t bins[4], float pooling, void *h_out,
                                      uint64_t out_cap);
int64_t lscomp_server_submit_decompress(lscomp_server *server, const void *h_container, uint64_t len, void *h_out,
                                        uint64_t out_cap);
int lscomp_server_wait(lscomp_server *server, int64_t id, lscomp_server_result *result);
int lscomp_server_stats(lscomp_server *server, uint64_t *rounds, uint64_t *batches, uint64_t *batched_requests);

/* Lossy quality report on the GPU (the reference computes these on the host,
   lsCOMP/src/cuLSZ_utility.cu:757-946 computePSNR / computeSSIM, on float
   copies of the data; values are converted to float the same way).
   psnr[6] (may be NULL): MSE, value range of the original, PSNR (dB), L2 norm
   of the error, that norm over the L2 norm of the decoded data, NRMSE.
   *ssim (may be NULL): mean SSIM over 7x7x7 windows placed every 2 elements
   along each axis (NaN when a dimension is below 7).  Results equal the
   host functions' up to the order of the final sums.  SSIM reads each value
   ~170 times (about 1000x the cost of PSNR).  Allocates small partial-sum
   buffers per call; synchronises the stream. */
int lscomp_quality_u16(const uint16_t *d_ori, const uint16_t *d_dec, uint32_t x, uint32_t y, uint32_t z,
                       double psnr[6], double *ssim, void *stream);
int lscomp_quality_u32(const uint32_t *d_ori, const uint32_t *d_dec, uint32_t x, uint32_t y, uint32_t z,
                       double psnr[6], double *ssim, void *stream);

/* allow = 0: calls through this workspace never run the launch-configuration
   tuner (they use its table, else the built-in rules) -- for latency-bound
   loops such as the serving loop, whose requests must not wait for a tuning
   run; allow = 1 (the default) restores tuning. */
int lscomp_workspace_set_tuning(lscomp_workspace *ws, int allow);

/* Failure injection for tests (no counterpart in the reference, whose
   look-back spins without a bound, lsCOMP/src/cuLSZ_kernel.cu:1001-1004).
   The next launch through this workspace starts its tile tickets at 1, so
   tile 0 (decoder: segment 0 of the offsets kernel) is never claimed and
   the look-back of its successor waits for a publication that never comes,
   and every wait of that launch is limited to wait_ns (1 ms .. 2 s) instead
   of 2 s.  The call returns LSCOMP_ERR_TIMEOUT after about that long; the
   launch ends without a fault and the workspace serves the next call
   normally.  Needs a stack of at least 2 tiles (decoder: 33 tiles) and a
   workspace that does not tune (lscomp_workspace_set_tuning(ws, 0)), since
   a tuning run would take the injected launch. */
int lscomp_workspace_stall_next(lscomp_workspace *ws, uint64_t wait_ns);

/* Wait for the workspace's last launch on `stream` and return its status. */
int lscomp_workspace_check(lscomp_workspace *ws, void *stream);

/* Number of kernel launches this library has issued in this process (for
   the benchmark's launch count). */
uint64_t lscomp_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* LSCOMP_H */
