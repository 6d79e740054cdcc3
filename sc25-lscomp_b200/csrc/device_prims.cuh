// device_prims.cuh -- sm_100a primitives used by the codec kernels:
// shared-memory mbarriers, 1-D TMA bulk copies (cp.async.bulk), gpu-scope
// acquire/release accesses for the single-pass scan, and bounded waits.
//
// Every wait in this library is bounded: a wait that runs past its time limit
// (or sees another CTA's abort) records an error in the launch's status word
// and returns, so a broken invariant ends the launch with an error code
// instead of hanging the GPU.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace lsc {

// status codes written to the device status word (first error wins)
enum DevError : uint32_t {
    DEV_OK = 0,
    DEV_ERR_TIMEOUT = 1,   // a bounded wait ran out
    DEV_ERR_CAPACITY = 2,  // output would pass the caller's capacity
    DEV_ERR_CORRUPT = 3,   // stream inconsistent with the geometry
    DEV_ERR_RANGE = 4,     // value range the format cannot represent
};

// Per-launch control block in device memory.  Zeroed by the host (one
// cudaMemsetAsync) before every launch.
struct LaunchCtl {
    unsigned long long ticket;   // next tile to claim (pushed past every tile on abort)
    unsigned int error;          // first DevError seen
    unsigned int abort;          // set with error: every CTA stops waiting
    unsigned long long total;    // payload bytes of the stream (encoder)
    unsigned long long stream_len;
    unsigned long long wait_ns;  // limit of a single wait in ns (0: kWaitLimitNs)
    unsigned long long reserved[3];
};

constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // 2 s for any single wait
constexpr unsigned long long kTicketAbort = 1ull << 48;     // added to the ticket on abort

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void raise_error(LaunchCtl *ctl, uint32_t code)
{
    atomicCAS(&ctl->error, 0u, code);
    atomicExch(&ctl->abort, 1u);
    atomicAdd(&ctl->ticket, kTicketAbort);  // every later claim is past the end
}

__device__ __forceinline__ bool aborted(const LaunchCtl *ctl)
{
    return *((volatile const unsigned int *)&ctl->abort) != 0u;
}

// The launch's limit for one wait (read when a wait starts to take long).
__device__ __forceinline__ unsigned long long wait_limit(const LaunchCtl *ctl)
{
    const unsigned long long w = *((volatile const unsigned long long *)&ctl->wait_ns);
    return w ? w : kWaitLimitNs;
}

// ---------------------------------------------------------------- mbarrier
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_cnt(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// A waiting thread is suspended until the phase completes (or this many
// nanoseconds pass), so waiting warps take no issue slots from working ones.
constexpr uint32_t kSuspendHintNs = 1000000u;

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity), "r"(kSuspendHintNs)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase with the given parity to complete.  Returns
// false if another CTA aborted the launch, or (after recording
// DEV_ERR_TIMEOUT) if the phase does not complete in time.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, LaunchCtl *ctl)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    const unsigned long long limit = wait_limit(ctl);
    uint32_t spins = 0;
    while (!mbar_try_wait(bar, parity)) {
        if ((++spins & 31u) == 0) {
            if (aborted(ctl)) return false;
            if (global_ns() - t0 > limit) {
                raise_error(ctl, DEV_ERR_TIMEOUT);
                return false;
            }
        }
    }
    return true;
}

// Wait, bounded by time only (not by the abort flag), for a phase whose
// completion is a TMA load landing: used before a CTA releases shared
// memory that a load may still be writing.  false if the limit passed.
__device__ __forceinline__ bool mbar_wait_landed(uint64_t *bar, uint32_t parity)
{
    const unsigned long long t0 = global_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_ns() - t0 > kWaitLimitNs) return false;
    return true;
}

// ---------------------------------------------------------------- TMA bulk
// 1-D bulk copy global -> shared, completion counted on an mbarrier.
// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Order this thread's earlier generic-proxy accesses to shared memory before
// later async-proxy (TMA) accesses.
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ---------------------------------------------------------------- gpu scope
// The look-back state words carry their flag and value in one 64-bit word
// and nothing else is read on the strength of them, so relaxed gpu-scope
// accesses suffice (no fence before a publication).
__device__ __forceinline__ void st_relaxed_u64(unsigned long long *p, unsigned long long v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// ---------------------------------------------------------------- look-back
// Tile state word: [epoch:20][flag:2][value:42].  The epoch is a per-call
// counter, so words left over from earlier calls read as "not ready" and the
// state array never needs clearing between calls.
constexpr int kEpochShift = 44;
constexpr int kFlagShift = 42;
constexpr unsigned long long kValueMask = (1ull << kFlagShift) - 1;
constexpr uint32_t kFlagAgg = 1;   // value = this tile's own size
constexpr uint32_t kFlagIncl = 2;  // value = inclusive prefix through this tile

__device__ __forceinline__ unsigned long long make_state(uint32_t epoch, uint32_t flag,
                                                         unsigned long long value)
{
    return ((unsigned long long)epoch << kEpochShift) | ((unsigned long long)flag << kFlagShift) |
           (value & kValueMask);
}

// Decoupled look-back over the tile states, run by one full warp.  Returns
// the exclusive prefix of tile `tile` in every lane; `ok` is false if the
// wait timed out or the launch was aborted.  Lane l inspects tile
// (window_end - l); a window is consumed once every tile up to the nearest
// inclusive one has published.
__device__ __forceinline__ unsigned long long lookback_warp(const unsigned long long *state,
                                                            unsigned long long tile, uint32_t epoch,
                                                            LaunchCtl *ctl, bool &ok)
{
    const uint32_t lane = threadIdx.x & 31;
    unsigned long long excl = 0;
    long long end = (long long)tile - 1;
    unsigned long long t0 = 0;
    uint32_t spins = 0;
    ok = true;
    while (end >= 0) {
        long long idx = end - (long long)lane;
        uint32_t flag;
        unsigned long long val;
        if (idx >= 0) {
            unsigned long long w = ld_relaxed_u64(state + idx);
            bool fresh = (uint32_t)(w >> kEpochShift) == epoch;
            flag = fresh ? (uint32_t)((w >> kFlagShift) & 3u) : 0u;
            val = w & kValueMask;
        } else {
            flag = kFlagIncl;  // before tile 0: inclusive prefix 0
            val = 0;
        }
        uint32_t inv = __ballot_sync(0xffffffffu, flag == 0);
        uint32_t incl = __ballot_sync(0xffffffffu, flag == kFlagIncl);
        uint32_t upto = incl ? ((incl & (0u - incl)) << 1) - 1u : 0xffffffffu;  // lanes up to first incl
        if ((inv & upto) == 0) {
            unsigned long long part = (lane < 32 && ((upto >> lane) & 1u)) ? val : 0ull;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
            excl += part;
            if (incl) break;
            end -= 32;
            continue;
        }
        // some predecessor has not published yet: back off, bounded
        if (spins == 0) t0 = global_ns();
        ++spins;
        if ((spins & 63u) == 0) {
            bool stop = false;
            if (lane == 0) stop = aborted(ctl) || (global_ns() - t0 > wait_limit(ctl));
            stop = __shfl_sync(0xffffffffu, stop, 0);
            if (stop) {
                if (lane == 0) raise_error(ctl, DEV_ERR_TIMEOUT);
                ok = false;
                return 0;
            }
        }
        __nanosleep(32);
    }
    return excl;
}


// Decoupled look-back with a known floor: the exclusive prefix of `tile`
// from the state words of tiles floor+1 .. tile-1 plus the inclusive prefix
// `floor_incl` of tile `floor` (< tile), which the caller already holds
// (floor = -1, floor_incl = 0 to walk from the start).  A walk stops early
// at a nearer inclusive word.  Each round reads 8 consecutive words per lane,
// 256 tiles per round trip.  Flag and value share one 64-bit word, so relaxed
// loads suffice.  Run by one full warp; ok = false on timeout or abort.
constexpr int kLookPerLane = 8;

__device__ __forceinline__ unsigned long long lookback_floor(const unsigned long long *state, long long tile,
                                                             long long floor, unsigned long long floor_incl,
                                                             uint32_t epoch, LaunchCtl *ctl, bool &ok)
{
    const uint32_t lane = threadIdx.x & 31;
    unsigned long long excl = 0;
    long long top = tile - 1;
    unsigned long long t0 = 0;
    uint32_t spins = 0;
    ok = true;
    for (;;) {
        uint32_t fl[kLookPerLane];
        unsigned long long v[kLookPerLane];
#pragma unroll
        for (int q = 0; q < kLookPerLane; q++) {
            const long long idx = top - (long long)(kLookPerLane * lane + q);
            if (idx > floor) {
                const unsigned long long w = ld_relaxed_u64(state + idx);
                const bool fresh = (uint32_t)(w >> kEpochShift) == epoch;
                fl[q] = fresh ? (uint32_t)((w >> kFlagShift) & 3u) : 0u;
                v[q] = w & kValueMask;
            } else {
                fl[q] = kFlagIncl;  // the floor itself (entries past it are never reached)
                v[q] = idx == floor ? floor_incl : 0ull;
            }
        }
        uint32_t qi = kLookPerLane, qv = kLookPerLane;  // first inclusive / first missing entry
#pragma unroll
        for (int q = kLookPerLane - 1; q >= 0; q--) {
            if (fl[q] == kFlagIncl) qi = (uint32_t)q;
            if (fl[q] == 0u) qv = (uint32_t)q;
        }
        const uint32_t inclm = __ballot_sync(0xffffffffu, qi < (uint32_t)kLookPerLane);
        const uint32_t first = inclm ? (uint32_t)(__ffs(inclm) - 1) : 32u;
        const bool missing = (lane < first && qv < (uint32_t)kLookPerLane) || (lane == first && qv < qi);
        if (!__any_sync(0xffffffffu, missing)) {
            unsigned long long part = 0;
#pragma unroll
            for (int q = 0; q < kLookPerLane; q++)
                if (lane < first || (lane == first && (uint32_t)q <= qi)) part += v[q];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
            excl += part;
            if (inclm) break;
            top -= 32 * kLookPerLane;
            continue;
        }
        // a tile in range has not published yet: back off, bounded
        if (spins == 0) t0 = global_ns();
        ++spins;
        if ((spins & 15u) == 0) {
            bool stop = false;
            if (lane == 0) stop = aborted(ctl) || (global_ns() - t0 > wait_limit(ctl));
            stop = __shfl_sync(0xffffffffu, stop, 0);
            if (stop) {
                if (lane == 0) raise_error(ctl, DEV_ERR_TIMEOUT);
                ok = false;
                return 0;
            }
        }
        __nanosleep(64);
    }
    return excl;
}

}  // namespace lsc
