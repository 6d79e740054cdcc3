// codec_host.h -- host-side pieces shared by the single-stack entry points
// (codec.cu) and the batch entry points (codec_batch.cu): the workspace,
// argument and geometry helpers, and the kernel launchers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <atomic>
#include <mutex>
#include <utility>
#include <vector>
#include "lscomp.h"
#include "codec_kernels.cuh"

struct lscomp_workspace {
    int device = 0;
    int sm_count = 0;
    lsc::LaunchCtl *ctl = nullptr;     // device
    lsc::LaunchCtl *h_ctl = nullptr;   // pinned host mirror for status reads
    unsigned long long *state = nullptr;   // look-back words, then per-tile offsets
    uint64_t state_cap = 0;            // entries of each of the two arrays
    uint32_t epoch = 0;
    // batch launches: stack descriptors (device and pinned staging), the
    // stack of every tile, and the per-stack sizes (device and pinned)
    lsc::BatchStack *d_stacks = nullptr;
    lsc::BatchStack *h_stacks = nullptr;
    unsigned long long *d_bsizes = nullptr;
    unsigned long long *h_bsizes = nullptr;
    uint32_t stacks_cap = 0;
    uint32_t *d_tile_stack = nullptr;
    uint64_t tile_stack_cap = 0;
    bool no_tune = false;              // calls through this workspace never tune
    void *pipe = nullptr;              // host-memory calls: copy streams, slot buffers (host_pipe.cu)
    uint64_t host_chunk_bytes = 0;     // host-memory calls: input bytes per chunk (0: the default)
    // lscomp_workspace_stall_next: the next launch starts its tile (or
    // segment) tickets at 1 with this wait limit (ns), so tile 0 is never
    // claimed and the look-back of tile 1 waits until the limit runs out
    uint64_t stall_wait_ns = 0;
    unsigned long long stall_words[2] = {0, 0};  // source of that launch's ticket and wait_ns
    std::mutex mu;
};

namespace lsc_host {
using namespace lsc;

inline std::atomic<uint64_t> g_launches{0};

constexpr uint32_t kEpochMax = (1u << 20) - 1;

inline int cuda_status(cudaError_t e)
{
    if (e == cudaSuccess) return LSCOMP_OK;
    if (e == cudaErrorMemoryAllocation) return LSCOMP_ERR_NOMEM;
    return LSCOMP_ERR_CUDA;
}

inline int dev_status(uint32_t e)
{
    switch (e) {
    case DEV_OK: return LSCOMP_OK;
    case DEV_ERR_TIMEOUT: return LSCOMP_ERR_TIMEOUT;
    case DEV_ERR_CAPACITY: return LSCOMP_ERR_CAPACITY;
    case DEV_ERR_CORRUPT: return LSCOMP_ERR_CORRUPT;
    case DEV_ERR_RANGE: return LSCOMP_ERR_RANGE;
    default: return LSCOMP_ERR_CUDA;
    }
}

// smallest zero count k (0..64) with (float)k/64 > p, 65 if none
// (lsCOMP/src/cuLSZ_kernel.cu:920-921; k/64 is exact in binary32)
inline int pool_min_zeros(float p)
{
    for (int k = 0; k <= 64; k++) {
        float sparsity = (float)k / 64.0f;
        if (sparsity > p) return k;
    }
    return 65;
}

// ceil(2^64 / b) for b >= 2: with 2^64 - 1 = q b + r (0 <= r < b), 2^64 / b
// = q + (r + 1) / b and 0 < r + 1 <= b, so the ceiling is always q + 1
inline unsigned long long magic64(uint32_t b)
{
    if (b < 2) return 0;
    return ~0ull / b + 1;
}

inline bool make_geom(uint32_t X, uint32_t Y, uint32_t Z, uint32_t tile_blocks, Geom &g)
{
    if (!X || !Y || !Z) return false;
    g.X = X; g.Y = Y; g.Z = Z;
    g.byb = (Y + 7) / 8;
    g.bzb = (Z + 7) / 8;
    g.nrows_b = (unsigned long long)X * g.byb;
    g.nb = g.nrows_b * g.bzb;
    g.R = (g.nb + 3) / 4 * 4;
    g.N = (unsigned long long)X * Y * Z;
    if (g.bzb <= tile_blocks) {
        g.chunked = 0;
        g.G = tile_blocks / g.bzb;
        g.ntiles = (g.nrows_b + g.G - 1) / g.G;
        g.nc = 1;
        g.W = g.bzb;
        g.inv_bzb = (65536u + g.bzb - 1) / g.bzb;
    } else {
        g.chunked = 1;
        g.G = 1;
        g.nc = (g.bzb + tile_blocks - 1) / tile_blocks;
        g.W = (g.bzb + g.nc - 1) / g.nc;
        g.ntiles = g.nrows_b * g.nc;
        g.inv_bzb = 0;
    }
    g.byb_magic = magic64(g.byb);
    g.nc_magic = magic64(g.nc);
    return true;
}

inline bool make_codec(const uint32_t bins[4], float p, bool wide, Codec &c, int &layout)
{
    if (!bins) return false;
    for (int k = 0; k < 4; k++) {
        if (bins[k] == 0) return false;
        c.bins[k] = bins[k];
        c.magic[k] = bins[k] == 1 ? 0u : (uint32_t)((0x100000000ull + bins[k] - 1) / bins[k]);
        c.magic64[k] = magic64(bins[k]);
        c.binc[k] = (!wide && bins[k] > 65536u) ? 65536u : bins[k];
        c.qsm[k] = lsc_small_quant_magic(bins[k]);
    }
    c.pool_min = pool_min_zeros(p);
    if (bins[0] == 1 && bins[1] == 1 && bins[2] == 1 && bins[3] == 1)
        layout = BINS_IDENT;
    else if (bins[0] == bins[1] && bins[1] == bins[2] && bins[2] == bins[3])
        layout = BINS_EQUAL;
    else if (bins[0] <= bins[1] && bins[1] <= bins[2] && bins[2] <= bins[3])
        layout = BINS_MONO;
    else
        layout = BINS_GENERAL;
    return true;
}

// widest access every row segment of the stack allows (bytes)
inline int vec_class(const void *p, uint32_t Z, size_t es)
{
    uintptr_t a = reinterpret_cast<uintptr_t>(p);
    if (es == 2) {
        if ((Z % 8u) == 0 && (a % 16u) == 0) return 16;
        if ((Z % 2u) == 0 && (a % 4u) == 0) return 4;
        return 2;
    }
    if ((Z % 4u) == 0 && (a % 16u) == 0) return 16;
    return 4;
}

// Ensure the workspace holds `ntiles` scan slots and hand out a fresh epoch.
inline int ws_prepare(lscomp_workspace *ws, uint64_t ntiles, cudaStream_t st)
{
    if (ntiles > ws->state_cap) {
        uint64_t cap = ntiles + ntiles / 4 + 1024;
        unsigned long long *p = nullptr;
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_status(e);
        if (ws->state) cudaFree(ws->state);
        ws->state = nullptr;
        ws->state_cap = 0;
        e = cudaMalloc(&p, 2 * cap * sizeof(unsigned long long));
        if (e != cudaSuccess) return cuda_status(e);
        e = cudaMemsetAsync(p, 0, 2 * cap * sizeof(unsigned long long), st);
        if (e != cudaSuccess) { cudaFree(p); return cuda_status(e); }
        ws->state = p;
        ws->state_cap = cap;
        ws->epoch = 0;
    }
    if (ws->epoch >= kEpochMax) {
        cudaError_t e = cudaMemsetAsync(ws->state, 0, ws->state_cap * sizeof(unsigned long long), st);
        if (e != cudaSuccess) return cuda_status(e);
        ws->epoch = 0;
    }
    ws->epoch++;
    cudaError_t e = cudaMemsetAsync(ws->ctl, 0, sizeof(LaunchCtl), st);
    if (e == cudaSuccess && ws->stall_wait_ns) {
        // one launch with tile 0 left unclaimed and a short wait limit
        ws->stall_words[0] = 1;
        ws->stall_words[1] = ws->stall_wait_ns;
        ws->stall_wait_ns = 0;
        e = cudaMemcpyAsync(&ws->ctl->ticket, &ws->stall_words[0], sizeof(unsigned long long),
                            cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&ws->ctl->wait_ns, &ws->stall_words[1], sizeof(unsigned long long),
                                cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // the pageable source words are reused
    }
    return cuda_status(e);
}

template <typename K>
inline int ctas_per_sm(K kernel, size_t smem)
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, kThreads, smem) != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}

template <typename T, int VEC, int BINS, bool POOL, int GRP, int WPG, bool BATCH, bool NARROW = false>
inline int launch_enc_w(const EncArgs<T> &a, int sm_count, cudaStream_t st)
{
    auto k = enc_kernel<T, VEC, BINS, POOL, GRP, WPG, BATCH, NARROW>;
    const size_t smem = sizeof(EncSmem);
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    // persistent: one CTA per SM (the CTA holds ~200 KB of rings)
    unsigned long long grid = (unsigned long long)sm_count;
    const unsigned long long ntiles = BATCH ? a.ntiles_all : a.g.ntiles;
    if (grid > ntiles) grid = ntiles;
    k<<<(unsigned)grid, EncShape<GRP, WPG>::kThreads, smem, st>>>(a);
    g_launches.fetch_add(1);
    return cuda_status(cudaGetLastError());
}

// Compute warps per encoder CTA: LSC_ENC_GROUPS groups of LSC_ENC_WPG warps.
// Share of the compute warps' unit slots a tile fills when a group of wpg
// warps takes its units round by round (8-block units, ceil(nblk / 8) of them).
inline double unit_fill(const Geom &g, uint32_t wpg)
{
    const uint32_t nblk = g.chunked ? g.W : g.G * g.bzb;
    const uint32_t units = (nblk + 7) / 8;
    return (double)units / (double)(wpg * ((units + wpg - 1) / wpg));
}

// Shape of the encoder CTA when no tuned choice is known (shape < 0): the
// lossless uint16 kernel is bound by its producer and writer warps and keeps
// LSC_ENC_GROUPS x LSC_ENC_WPG; the lossy one is bound by its compute warps
// and takes, of groups of 8, 7 or 13 warps (a group's warps take a tile's
// 8-block units round by round), the one that fills the unit slots best,
// preferring 8 unless another is clearly better (a block-row of 195 blocks:
// 25 units, 78% / 89% / 96%; measured on B200, CSSI-like lossy compress
// 2.71 -> 2.59 ms with 7, 2.51 -> 2.37 ms with 13; XPCS-like tiles of 32
// units keep 8).  Groups of 13 keep only the header bytes between the two
// passes and read the rows again from the input slot (72 registers a
// thread, 28 compute warps on the SM).  shape 0 / 1 / 2 force 2 x 8 / 2 x 7
// / 2 x 13 (uint16; 2 x 13 for single stacks only; uint32 always runs 2 x 8);
// shape 3 is 2 x 8 with block_pack's short paths for small values, for
// lossless uint16 single stacks only (a tuner candidate, never a rule: it
// gains where nearly every unit takes a short path, XPCS-like data, and
// loses a little elsewhere, where its four unrolled copies of the longer
// unit code crowd the instruction cache).
constexpr int kWideWpg = 13;

template <typename T, int VEC, int BINS, bool POOL, bool BATCH>
inline int launch_enc_t(const EncArgs<T> &a, int shape, int sm_count, cudaStream_t st)
{
    if constexpr (sizeof(T) == 2 && LSC_ENC_GROUPS == 2 && LSC_ENC_WPG == 8) {
        if (shape < 0 && BINS != BINS_IDENT && !BATCH) {
            const double f8 = unit_fill(a.g, 8), f7 = unit_fill(a.g, 7), f13 = unit_fill(a.g, kWideWpg);
            if (f13 > f8 + 0.05 && f13 >= f7) shape = 2;
            else if (f7 > f8 + 0.05) shape = 1;
        }
        if constexpr (!BATCH)
            if (shape == 2) return launch_enc_w<T, VEC, BINS, POOL, 2, kWideWpg, BATCH>(a, sm_count, st);
        if constexpr (!BATCH && BINS == BINS_IDENT)
            if (shape == 3) return launch_enc_w<T, VEC, BINS, POOL, 2, 8, BATCH, true>(a, sm_count, st);
        if (shape == 1) return launch_enc_w<T, VEC, BINS, POOL, 2, 7, BATCH>(a, sm_count, st);
    }
    return launch_enc_w<T, VEC, BINS, POOL, LSC_ENC_GROUPS, LSC_ENC_WPG, BATCH>(a, sm_count, st);
}

template <typename T, int VEC, bool BATCH>
inline int launch_enc_v(const EncArgs<T> &a, int layout, bool pool, int shape, int sm, cudaStream_t st)
{
    if (layout == BINS_IDENT)
        return pool ? launch_enc_t<T, VEC, BINS_IDENT, true, BATCH>(a, shape, sm, st)
                    : launch_enc_t<T, VEC, BINS_IDENT, false, BATCH>(a, shape, sm, st);
    if (layout == BINS_EQUAL)
        return pool ? launch_enc_t<T, VEC, BINS_EQUAL, true, BATCH>(a, shape, sm, st)
                    : launch_enc_t<T, VEC, BINS_EQUAL, false, BATCH>(a, shape, sm, st);
    if (layout == BINS_MONO)
        return pool ? launch_enc_t<T, VEC, BINS_MONO, true, BATCH>(a, shape, sm, st)
                    : launch_enc_t<T, VEC, BINS_MONO, false, BATCH>(a, shape, sm, st);
    return pool ? launch_enc_t<T, VEC, BINS_GENERAL, true, BATCH>(a, shape, sm, st)
                : launch_enc_t<T, VEC, BINS_GENERAL, false, BATCH>(a, shape, sm, st);
}

// Encoder launch with the widest row access `vec` allows.
template <typename T, bool BATCH>
inline int launch_enc_any(const EncArgs<T> &a, int vec, int layout, bool pool, int shape, int sm, cudaStream_t st)
{
    switch (vec) {
    case 16: return launch_enc_v<T, 16, BATCH>(a, layout, pool, shape, sm, st);
    case 4: return launch_enc_v<T, 4, BATCH>(a, layout, pool, shape, sm, st);
    default:
        if constexpr (sizeof(T) == 2) return launch_enc_v<T, 2, BATCH>(a, layout, pool, shape, sm, st);
        return LSCOMP_ERR_ARG;
    }
}

template <typename T, int VEC>
inline int launch_dec_t(const DecArgs<T> &a, int sm_count, cudaStream_t st)
{
    // 1) per-tile stream offsets from the header bytes
    const unsigned long long nseg = (a.g.ntiles + kSegTiles - 1) / kSegTiles;
    unsigned long long grid = (unsigned long long)sm_count * 4;
    if (grid > nseg) grid = nseg;
    dec_offsets_kernel<T><<<(unsigned)grid, kThreads, 0, st>>>(a);
    g_launches.fetch_add(1);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e);
    // 2) every tile independently
    if (a.g.ntiles > 0x7fffffffull) return LSCOMP_ERR_ARG;
    dec_kernel<T, VEC, false><<<(unsigned)a.g.ntiles, kThreads, 0, st>>>(a);
    g_launches.fetch_add(1);
    return cuda_status(cudaGetLastError());
}

inline int read_ctl(lscomp_workspace *ws, cudaStream_t st)
{
    cudaError_t e = cudaMemcpyAsync(ws->h_ctl, ws->ctl, sizeof(LaunchCtl), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return cuda_status(e);
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_status(e);
    return dev_status(ws->h_ctl->error);
}

// Frees the workspace's host-memory pipeline state (host_pipe.cu).
void pipe_destroy(lscomp_workspace *ws);

// ---------------------------------------------------------------- tuner
// Launch configuration of one call: encoder CTA shape (-1: the rule of
// launch_enc_t, 0: 2 x 8 warps, 1: 2 x 7) and the most blocks a tile holds.
struct TuneCfg {
    int shape;
    uint32_t tile_blocks;
};

constexpr uint8_t kTuneCompress = 0, kTuneBatch = 1, kTuneDecompress = 2;

// What a choice is kept for: element size, bins layout, pooling on/off,
// call kind, row access width and blocks per block-row (0 for batches).
struct TuneKey {
    uint8_t es, layout, pool, kind, vec;
    uint32_t bzb;
};

int tune_mode();  // 1: tune keys not in the table on first use
bool tune_lookup(const TuneKey &k, TuneCfg &c);  // counts a hit when found
void tune_store(const TuneKey &k, const TuneCfg &c, const std::vector<std::pair<TuneCfg, float>> &times);
std::vector<TuneCfg> tune_candidates(int es, int kind, int layout);

constexpr int kTuneReps = 3;
// Single stacks of fewer tiles than this many per SM are not tuned (their
// time is launch latency and the scan's tail; the rules serve them)
constexpr int kTuneMinTilesPerSm = 4;

// The configuration for `key`: the table's, else (tuning on, may_tune, stream
// not being captured) the fastest candidate, each timed with CUDA events over
// kTuneReps calls after one untimed call; else `rule`.  run(cfg) enqueues
// one complete call on st (control block cleared, kernel launched) and
// returns its launch status; the caller holds the workspace lock.  A
// candidate whose launch or device status fails ends the tuning with
// `rule` and nothing stored.
template <class Run>
inline TuneCfg tune_choose(lscomp_workspace *ws, const TuneKey &key, const TuneCfg &rule, bool may_tune,
                           cudaStream_t st, Run run)
{
    TuneCfg c;
    if (tune_lookup(key, c)) return c;
    if (!may_tune || ws->no_tune || !tune_mode()) return rule;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return rule;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess) return rule;
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return rule;
    }
    std::vector<std::pair<TuneCfg, float>> times;
    bool ok = true;
    for (const TuneCfg &cand : tune_candidates(key.es, key.kind, key.layout)) {
        ok = run(cand) == LSCOMP_OK && read_ctl(ws, st) == LSCOMP_OK;
        if (ok) ok = cudaEventRecord(e0, st) == cudaSuccess;
        for (int i = 0; ok && i < kTuneReps; i++) ok = run(cand) == LSCOMP_OK;
        if (ok) ok = cudaEventRecord(e1, st) == cudaSuccess && read_ctl(ws, st) == LSCOMP_OK;
        float ms = 0.f;
        if (ok) ok = cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
        if (!ok) break;
        times.push_back({cand, ms / kTuneReps});
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!ok || times.empty()) return rule;
    size_t best = 0;
    for (size_t i = 1; i < times.size(); i++)
        if (times[i].second < times[best].second) best = i;
    tune_store(key, times[best].first, times);
    return times[best].first;
}

}  // namespace lsc_host
