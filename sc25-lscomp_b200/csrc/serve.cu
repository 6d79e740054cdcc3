// serve.cu -- a request-serving loop over the codec (include/lscomp.h,
// lscomp_server_*): host buffers in, host buffers out, continuous batching.
//
// Callers submit compress requests (a stack in host memory -> a container in
// host memory) and decompress requests (a container -> the stack) from any
// thread.  Three threads per server move the requests through a pipeline on
// one device, each on its own CUDA stream:
//
//   * uploader: admits waiting requests in arrival order as soon as the
//     device arena has room for a request's worst-case footprint (its input
//     plus the largest output it can produce; a compress output is bounded
//     by the header and 128 (uint16) or 248 (uint32) bytes per block), so the
//     device never runs out of memory however the load arrives; a request
//     larger than the whole arena is refused at submission
//     (LSCOMP_ERR_TOO_LARGE).  It then streams the request's input onto the
//     device through a ring of pinned staging slots: the host copy of one
//     slot overlaps the host-to-device copy of the previous one.
//   * launcher: takes every request whose upload has been queued -- however
//     many arrived while the previous launches ran -- and runs them as batch
//     launches: the compress requests of one element type as one
//     lscomp_compress_batch_ex_* launch (each stack with its own shape, bins
//     and pooling threshold), the decompress requests of one element type as
//     one lscomp_decompress_batch_* (a group of one request runs the
//     single-stack call instead).  If a batch fails, its requests run again
//     one at a time, so a bad request fails alone.
//   * downloader: streams each finished output back through its own ring of
//     pinned slots, releases the request's arena space (which may admit the
//     next waiting request) and completes the request.
//
// While one batch is on the GPU, later requests upload and earlier ones
// download; the staging rings are a fixed 2 x 128 MB of pinned memory
// whatever the arena's size.  A request whose host buffer is itself
// page-locked (cudaHostAlloc, cudaHostRegister, or a framework's pinned
// tensor) skips the staging ring in that direction: its bytes cross PCIe
// with one direct copy, and no host thread copies them.  A request's output depends only on the
// request: batched or alone, its container is byte-identical to what
// lscomp_compress_container writes.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <utility>
#include <vector>
#include "lscomp.h"

namespace {

constexpr uint64_t kAlign = 256;
constexpr uint32_t kHdr = 64;
constexpr int kSlots = 4;                     // staging slots per direction
constexpr uint64_t kSlotBytes = 32ull << 20;  // bytes per staging slot
constexpr uint64_t kInlineCopy = 1ull << 20;  // host copies below this run on the pipeline thread itself

uint64_t align_up(uint64_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

uint64_t now_ns()
{
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

// True when the first and the last byte of [p, p + n) are page-locked host
// memory, so the device copies the range directly (a buffer is expected to
// be one such allocation).  Pageable memory reports cudaMemoryTypeUnregistered.
bool host_pinned(const void *p, uint64_t n)
{
    const uint8_t *b = static_cast<const uint8_t *>(p);
    for (const uint8_t *q : {b, b + (n ? n - 1 : 0)}) {
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, q) != cudaSuccess) {
            cudaGetLastError();  // clear it: this query's error is not the caller's
            return false;
        }
        if (a.type != cudaMemoryTypeHost) return false;
    }
    return true;
}

struct Request {
    int64_t id = 0;
    int op = 0;  // 0 compress, 1 decompress
    uint32_t eb = 2;
    const void *h_in = nullptr;
    uint64_t in_bytes = 0;
    uint32_t x = 0, y = 0, z = 0;
    uint32_t bins[4] = {0, 0, 0, 0};
    float p = 0.f;
    uint64_t body_len = 0;  // decompress: stream bytes after the container header
    void *h_out = nullptr;
    uint64_t out_cap = 0;
    uint64_t out_dev = 0;   // device bytes reserved for the output
    uint64_t in_off = 0, out_off = 0;  // arena offsets while admitted
    cudaEvent_t uploaded = nullptr;    // recorded after the input's last copy
    uint8_t hdr[kHdr];                 // compress: the container header
    int status = 0;
    uint64_t out_len = 0;
    uint64_t t_submit = 0, t_start = 0, t_done = 0;
    bool done = false, waited = false;
    bool in_pinned = false, out_pinned = false;  // host buffers the device can copy directly
    uint64_t footprint() const { return align_up(in_bytes) + align_up(out_dev); }
};

// First-fit allocator over the device arena (offsets only; host bookkeeping).
class Arena {
  public:
    explicit Arena(uint64_t bytes) { free_[0] = bytes; }
    bool alloc(uint64_t n, uint64_t &off)
    {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            off = it->first;
            const uint64_t left = it->second - n;
            free_.erase(it);
            if (left) free_[off + n] = left;
            return true;
        }
        return false;
    }
    void release(uint64_t off, uint64_t n)
    {
        auto next = free_.lower_bound(off);
        if (next != free_.end() && off + n == next->first) {
            n += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                prev->second += n;
                return;
            }
        }
        free_[off] = n;
    }

  private:
    std::map<uint64_t, uint64_t> free_;  // offset -> bytes
};

// A fixed pool of host threads that copies one list of byte ranges at a
// time, split into pieces of at most kPiece bytes (one caller per pool).
class CopyPool {
  public:
    explicit CopyPool(unsigned n)
    {
        for (unsigned i = 0; i < n; i++) th_.emplace_back([this] { run(); });
    }
    ~CopyPool()
    {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto &t : th_) t.join();
    }
    void copy(void *dst, const void *src, uint64_t n)
    {
        if (n <= kInlineCopy || th_.empty()) {
            memcpy(dst, src, n);
            return;
        }
        std::unique_lock<std::mutex> lk(mu_);
        uint8_t *d = static_cast<uint8_t *>(dst);
        const uint8_t *s = static_cast<const uint8_t *>(src);
        for (uint64_t o = 0; o < n; o += kPiece) work_.push_back({d + o, s + o, n - o < kPiece ? n - o : kPiece});
        pending_ += (n + kPiece - 1) / kPiece;
        cv_.notify_all();
        done_cv_.wait(lk, [&] { return pending_ == 0; });
    }

  private:
    static constexpr uint64_t kPiece = 4ull << 20;
    struct Job {
        uint8_t *d;
        const uint8_t *s;
        uint64_t n;
    };
    void run()
    {
        std::unique_lock<std::mutex> lk(mu_);
        for (;;) {
            cv_.wait(lk, [&] { return stop_ || !work_.empty(); });
            if (work_.empty()) return;
            Job j = work_.front();
            work_.pop_front();
            lk.unlock();
            memcpy(j.d, j.s, j.n);
            lk.lock();
            if (--pending_ == 0) done_cv_.notify_all();
        }
    }
    std::vector<std::thread> th_;
    std::deque<Job> work_;
    uint64_t pending_ = 0;
    bool stop_ = false;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
};

unsigned copy_threads()
{
    const char *e = getenv("LSCOMP_SERVER_COPY_THREADS");
    const int n = e ? atoi(e) : 8;
    return n < 0 ? 0u : (n > 32 ? 32u : (unsigned)n);
}

// A ring of pinned staging slots with one event each (the copy that last
// used the slot).
struct Ring {
    uint8_t *buf = nullptr;
    cudaEvent_t ev[kSlots] = {};
    bool busy[kSlots] = {};
    uint8_t *slot(int k) { return buf + (uint64_t)k * kSlotBytes; }
};

}  // namespace

struct lscomp_server {
    int device = 0;
    cudaStream_t up = nullptr, comp = nullptr, down = nullptr;
    lscomp_workspace *ws = nullptr;  // used by the launcher only
    uint8_t *arena = nullptr;        // device
    uint64_t arena_bytes = 0;
    Arena *alloc = nullptr;          // guarded by mu
    Ring rin, rout;
    CopyPool *copy_in = nullptr, *copy_out = nullptr;
    std::mutex mu;
    std::condition_variable cv_admit, cv_launch, cv_down, cv_done;
    std::deque<Request *> waiting, ready, finished;
    std::unordered_map<int64_t, Request *> reqs;
    std::vector<cudaEvent_t> events;  // spare upload events
    std::thread uploader, launcher, downloader;
    bool stop = false, uploads_over = false, launches_over = false;
    int64_t next_id = 1;
    uint64_t rounds = 0, batches = 0, batched_requests = 0;
};

namespace {

// ---------------------------------------------------------------- uploader
void upload(lscomp_server *s, Request *r)
{
    const uint8_t *src = static_cast<const uint8_t *>(r->h_in);
    uint8_t *dst = s->arena + r->in_off;
    static thread_local int next = 0;
    int st = LSCOMP_OK;
    // checked here, on the server's device, so that submitting makes no
    // CUDA call on the client's thread
    r->in_pinned = host_pinned(r->h_in, r->in_bytes);
    if (r->in_pinned) {  // one direct copy, no staging
        if (cudaMemcpyAsync(dst, src, r->in_bytes, cudaMemcpyHostToDevice, s->up) != cudaSuccess)
            st = LSCOMP_ERR_CUDA;
        if (!st && cudaEventRecord(r->uploaded, s->up) != cudaSuccess) st = LSCOMP_ERR_CUDA;
        r->status = st;
        return;
    }
    for (uint64_t o = 0; o < r->in_bytes; o += kSlotBytes) {
        const int k = next;
        next = (next + 1) % kSlots;
        // the slot's previous host-to-device copy must be done before it is refilled
        if (s->rin.busy[k] && cudaEventSynchronize(s->rin.ev[k]) != cudaSuccess) {
            st = LSCOMP_ERR_CUDA;
            break;
        }
        const uint64_t n = r->in_bytes - o < kSlotBytes ? r->in_bytes - o : kSlotBytes;
        s->copy_in->copy(s->rin.slot(k), src + o, n);
        if (cudaMemcpyAsync(dst + o, s->rin.slot(k), n, cudaMemcpyHostToDevice, s->up) != cudaSuccess ||
            cudaEventRecord(s->rin.ev[k], s->up) != cudaSuccess) {
            st = LSCOMP_ERR_CUDA;
            break;
        }
        s->rin.busy[k] = true;
    }
    if (!st && cudaEventRecord(r->uploaded, s->up) != cudaSuccess) st = LSCOMP_ERR_CUDA;
    r->status = st;
}

void uploader_main(lscomp_server *s)
{
    cudaSetDevice(s->device);
    for (;;) {
        Request *r = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            for (;;) {
                if (!s->waiting.empty()) {
                    Request *h = s->waiting.front();
                    uint64_t off = 0;
                    if (s->alloc->alloc(h->footprint(), off)) {  // admitted in arrival order
                        s->waiting.pop_front();
                        h->in_off = off;
                        h->out_off = off + align_up(h->in_bytes);
                        h->t_start = now_ns();
                        if (!s->events.empty()) {
                            h->uploaded = s->events.back();
                            s->events.pop_back();
                        }
                        r = h;
                        break;
                    }
                } else if (s->stop) {
                    s->uploads_over = true;
                    s->cv_launch.notify_all();
                    return;
                }
                s->cv_admit.wait(lk);
            }
        }
        if (!r->uploaded && cudaEventCreateWithFlags(&r->uploaded, cudaEventDisableTiming) != cudaSuccess) {
            r->uploaded = nullptr;
            r->status = LSCOMP_ERR_CUDA;
        } else {
            upload(s, r);
        }
        std::lock_guard<std::mutex> lk(s->mu);
        s->ready.push_back(r);
        s->cv_launch.notify_all();
    }
}

// ---------------------------------------------------------------- launcher
void compress_group(lscomp_server *s, const std::vector<Request *> &v, uint32_t eb)
{
    const size_t n = v.size();
    std::vector<lscomp_stack> stacks(n);
    std::vector<uint32_t> bins(4 * n);
    std::vector<float> pool(n);
    std::vector<uint64_t> len(n), ref(n);
    for (size_t i = 0; i < n; i++) {
        Request *r = v[i];
        stacks[i].d_in = s->arena + r->in_off;
        stacks[i].x = r->x;
        stacks[i].y = r->y;
        stacks[i].z = r->z;
        stacks[i].d_out = s->arena + r->out_off;
        stacks[i].cap = r->out_dev;
        memcpy(&bins[4 * i], r->bins, sizeof(r->bins));
        pool[i] = r->p;
    }
    auto batch = [&](size_t i0, size_t cnt) {
        if (cnt == 1) {
            // one request: the single-stack kernel, which spares the batch
            // launch's per-tile stack lookup (the same stream either way)
            const lscomp_stack &q = stacks[i0];
            return eb == 2 ? lscomp_compress_u16(s->ws, static_cast<const uint16_t *>(q.d_in), q.x, q.y, q.z,
                                                 &bins[4 * i0], pool[i0], q.d_out, q.cap, &len[i0], &ref[i0], s->comp)
                           : lscomp_compress_u32(s->ws, static_cast<const uint32_t *>(q.d_in), q.x, q.y, q.z,
                                                 &bins[4 * i0], pool[i0], q.d_out, q.cap, &len[i0], &ref[i0], s->comp);
        }
        return eb == 2 ? lscomp_compress_batch_ex_u16(s->ws, &stacks[i0], (uint32_t)cnt, &bins[4 * i0], &pool[i0],
                                                      &len[i0], &ref[i0], s->comp)
                       : lscomp_compress_batch_ex_u32(s->ws, &stacks[i0], (uint32_t)cnt, &bins[4 * i0], &pool[i0],
                                                      &len[i0], &ref[i0], s->comp);
    };
    std::vector<int> st(n, batch(0, n));
    if (st[0] && n > 1)
        for (size_t i = 0; i < n; i++) st[i] = batch(i, 1);  // one at a time: a bad request fails alone
    {
        std::lock_guard<std::mutex> lk(s->mu);  // lscomp_server_stats reads these under the lock
        s->batches++;
        s->batched_requests += n;
    }
    for (size_t i = 0; i < n; i++) {
        Request *r = v[i];
        if (!st[i] && kHdr + len[i] > r->out_cap) st[i] = LSCOMP_ERR_CAPACITY;
        if (!st[i]) {
            lscomp_container_write_header(r->hdr, eb, r->x, r->y, r->z, r->bins, r->p, len[i], ref[i]);
            r->out_len = kHdr + len[i];
        }
        r->status = st[i];
    }
}

void decompress_group(lscomp_server *s, const std::vector<Request *> &v, uint32_t eb)
{
    const size_t n = v.size();
    std::vector<lscomp_stack> stacks(n);
    std::vector<uint32_t> bins(4 * n);
    std::vector<float> pool(n);
    for (size_t i = 0; i < n; i++) {
        Request *r = v[i];
        stacks[i].d_in = s->arena + r->in_off + kHdr;
        stacks[i].x = r->x;
        stacks[i].y = r->y;
        stacks[i].z = r->z;
        stacks[i].d_out = s->arena + r->out_off;
        stacks[i].cap = r->body_len;
        memcpy(&bins[4 * i], r->bins, sizeof(r->bins));
        pool[i] = r->p;
    }
    auto batch = [&](size_t i0, size_t cnt) {
        if (cnt == 1) {  // one request: the single-stack decoder
            const lscomp_stack &q = stacks[i0];
            const uint8_t *in = static_cast<const uint8_t *>(q.d_in);
            return eb == 2 ? lscomp_decompress_u16(s->ws, in, q.cap, q.x, q.y, q.z, &bins[4 * i0], pool[i0],
                                                   reinterpret_cast<uint16_t *>(q.d_out), s->comp)
                           : lscomp_decompress_u32(s->ws, in, q.cap, q.x, q.y, q.z, &bins[4 * i0], pool[i0],
                                                   reinterpret_cast<uint32_t *>(q.d_out), s->comp);
        }
        return eb == 2 ? lscomp_decompress_batch_u16(s->ws, &stacks[i0], (uint32_t)cnt, &bins[4 * i0], &pool[i0],
                                                     s->comp)
                       : lscomp_decompress_batch_u32(s->ws, &stacks[i0], (uint32_t)cnt, &bins[4 * i0], &pool[i0],
                                                     s->comp);
    };
    std::vector<int> st(n, batch(0, n));
    if (st[0] && n > 1)
        for (size_t i = 0; i < n; i++) st[i] = batch(i, 1);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->batches++;
        s->batched_requests += n;
    }
    for (size_t i = 0; i < n; i++) {
        v[i]->status = st[i];
        if (!st[i]) v[i]->out_len = v[i]->out_dev;
    }
}

void launcher_main(lscomp_server *s)
{
    cudaSetDevice(s->device);
    for (;;) {
        std::vector<Request *> round;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_launch.wait(lk, [&] { return !s->ready.empty() || s->uploads_over; });
            if (s->ready.empty()) {
                s->launches_over = true;
                s->cv_down.notify_all();
                return;
            }
            round.assign(s->ready.begin(), s->ready.end());  // everything uploaded so far
            s->ready.clear();
            s->rounds++;
        }
        // the kernels wait for the uploads on the device, not on the host
        for (Request *r : round) {
            if (r->status) continue;
            if (cudaStreamWaitEvent(s->comp, r->uploaded, 0) != cudaSuccess) r->status = LSCOMP_ERR_CUDA;
        }
        for (int op = 0; op < 2; op++)
            for (uint32_t eb : {2u, 4u}) {
                std::vector<Request *> g;
                for (Request *r : round)
                    if (!r->status && r->op == op && r->eb == eb) g.push_back(r);
                if (g.empty()) continue;
                if (op == 0) compress_group(s, g, eb);
                else decompress_group(s, g, eb);
            }
        std::lock_guard<std::mutex> lk(s->mu);
        for (Request *r : round) {
            if (r->uploaded) s->events.push_back(r->uploaded);  // waits already queued keep their state
            r->uploaded = nullptr;
            s->finished.push_back(r);
        }
        s->cv_down.notify_all();
    }
}

// ---------------------------------------------------------------- downloader
// Device [src, src + n) to host dst through the ring: each slot's copy out
// of staging runs while the following slots' device-to-host copies fly.
// A page-locked dst takes one direct copy instead.
int download(lscomp_server *s, uint8_t *dst, const uint8_t *src, uint64_t n, bool pinned)
{
    if (pinned) {
        if (n && cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, s->down) != cudaSuccess) return LSCOMP_ERR_CUDA;
        return cudaStreamSynchronize(s->down) == cudaSuccess ? LSCOMP_OK : LSCOMP_ERR_CUDA;
    }
    struct Piece {
        int k;
        uint64_t off, n;
    };
    std::deque<Piece> fly;
    int st = LSCOMP_OK;
    int k = 0;
    auto drain_one = [&]() {
        Piece p = fly.front();
        fly.pop_front();
        if (cudaEventSynchronize(s->rout.ev[p.k]) != cudaSuccess) st = LSCOMP_ERR_CUDA;
        if (!st) s->copy_out->copy(dst + p.off, s->rout.slot(p.k), p.n);
    };
    for (uint64_t o = 0; o < n && !st; o += kSlotBytes) {
        if ((int)fly.size() == kSlots) drain_one();  // frees slot k (its previous piece)
        const uint64_t m = n - o < kSlotBytes ? n - o : kSlotBytes;
        if (cudaMemcpyAsync(s->rout.slot(k), src + o, m, cudaMemcpyDeviceToHost, s->down) != cudaSuccess ||
            cudaEventRecord(s->rout.ev[k], s->down) != cudaSuccess) {
            st = LSCOMP_ERR_CUDA;
            break;
        }
        fly.push_back({k, o, m});
        k = (k + 1) % kSlots;
    }
    while (!fly.empty()) drain_one();
    return st;
}

void downloader_main(lscomp_server *s)
{
    cudaSetDevice(s->device);
    for (;;) {
        Request *r = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_down.wait(lk, [&] { return !s->finished.empty() || s->launches_over; });
            if (s->finished.empty()) return;
            r = s->finished.front();
            s->finished.pop_front();
        }
        if (!r->status) {
            uint8_t *out = static_cast<uint8_t *>(r->h_out);
            r->out_pinned = host_pinned(out, r->out_cap);
            if (r->op == 0) {
                memcpy(out, r->hdr, kHdr);
                r->status = download(s, out + kHdr, s->arena + r->out_off, r->out_len - kHdr, r->out_pinned);
            } else {
                r->status = download(s, out, s->arena + r->out_off, r->out_len, r->out_pinned);
            }
        }
        std::lock_guard<std::mutex> lk(s->mu);
        s->alloc->release(r->in_off, r->footprint());
        r->t_done = now_ns();
        if (r->status) r->out_len = 0;
        r->done = true;
        s->cv_admit.notify_all();
        s->cv_done.notify_all();
    }
}

int64_t enqueue(lscomp_server *s, Request *r)
{
    if (r->footprint() > s->arena_bytes) {
        delete r;
        return -(int64_t)LSCOMP_ERR_TOO_LARGE;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) {
        delete r;
        return -(int64_t)LSCOMP_ERR_ARG;
    }
    r->id = s->next_id++;
    r->t_submit = now_ns();
    s->reqs[r->id] = r;
    s->waiting.push_back(r);
    s->cv_admit.notify_all();
    return r->id;
}

}  // namespace

extern "C" {

int lscomp_server_create(lscomp_server **out, int device, uint64_t arena_bytes)
{
    if (!out || arena_bytes < 1024) return LSCOMP_ERR_ARG;
    *out = nullptr;
    int prev = 0;
    cudaGetDevice(&prev);
    int dev = device;
    if (dev < 0) dev = prev;
    if (cudaSetDevice(dev) != cudaSuccess) return LSCOMP_ERR_CUDA;
    lscomp_server *s = new lscomp_server();
    s->device = dev;
    s->arena_bytes = arena_bytes;
    int st = lscomp_workspace_create(&s->ws, dev);
    // no request waits for a tuning run: the server's calls use the tuner's
    // table when it has the key (lscomp_tune_load at start-up) and the
    // built-in rules otherwise
    if (!st) st = lscomp_workspace_set_tuning(s->ws, 0);
    for (cudaStream_t *p : {&s->up, &s->comp, &s->down})
        if (!st && cudaStreamCreateWithFlags(p, cudaStreamNonBlocking) != cudaSuccess) st = LSCOMP_ERR_CUDA;
    if (!st && cudaMalloc(&s->arena, arena_bytes) != cudaSuccess) st = LSCOMP_ERR_NOMEM;
    for (Ring *g : {&s->rin, &s->rout}) {
        if (!st && cudaMallocHost(&g->buf, kSlots * kSlotBytes) != cudaSuccess) st = LSCOMP_ERR_NOMEM;
        for (int k = 0; k < kSlots && !st; k++)
            if (cudaEventCreateWithFlags(&g->ev[k], cudaEventDisableTiming) != cudaSuccess) st = LSCOMP_ERR_CUDA;
    }
    cudaSetDevice(prev);
    if (st) {
        lscomp_server_destroy(s);
        return st;
    }
    s->alloc = new Arena(arena_bytes);
    s->copy_in = new CopyPool(copy_threads());
    s->copy_out = new CopyPool(copy_threads());
    s->uploader = std::thread(uploader_main, s);
    s->launcher = std::thread(launcher_main, s);
    s->downloader = std::thread(downloader_main, s);
    *out = s;
    return LSCOMP_OK;
}

int lscomp_server_destroy(lscomp_server *s)
{
    if (!s) return LSCOMP_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv_admit.notify_all();
    }
    // each stage ends once the stage before it has ended and its queue is
    // empty: everything submitted runs to completion
    if (s->uploader.joinable()) s->uploader.join();
    if (s->launcher.joinable()) s->launcher.join();
    if (s->downloader.joinable()) s->downloader.join();
    delete s->copy_in;
    delete s->copy_out;
    delete s->alloc;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(s->device);
    for (Ring *g : {&s->rin, &s->rout}) {
        for (int k = 0; k < kSlots; k++)
            if (g->ev[k]) cudaEventDestroy(g->ev[k]);
        if (g->buf) cudaFreeHost(g->buf);
    }
    for (cudaEvent_t e : s->events) cudaEventDestroy(e);
    if (s->arena) cudaFree(s->arena);
    for (cudaStream_t p : {s->up, s->comp, s->down})
        if (p) cudaStreamDestroy(p);
    if (s->ws) lscomp_workspace_destroy(s->ws);
    cudaSetDevice(prev);
    for (auto &kv : s->reqs) delete kv.second;
    delete s;
    return LSCOMP_OK;
}

int64_t lscomp_server_submit_compress(lscomp_server *s, uint32_t elem_bytes, const void *h_in, uint32_t x,
                                      uint32_t y, uint32_t z, const uint32_t bins[4], float pooling, void *h_out,
                                      uint64_t out_cap)
{
    if (!s || !h_in || !h_out || !bins || (elem_bytes != 2 && elem_bytes != 4) || !x || !y || !z)
        return -(int64_t)LSCOMP_ERR_ARG;
    for (int k = 0; k < 4; k++)
        if (!bins[k]) return -(int64_t)LSCOMP_ERR_ARG;
    Request *r = new Request();
    r->op = 0;
    r->eb = elem_bytes;
    r->h_in = h_in;
    r->in_bytes = (uint64_t)x * y * z * elem_bytes;
    r->x = x;
    r->y = y;
    r->z = z;
    memcpy(r->bins, bins, sizeof(r->bins));
    r->p = pooling;
    r->h_out = h_out;
    r->out_cap = out_cap;
    r->out_dev = elem_bytes == 2 ? lscomp_max_stream_bytes_u16(x, y, z) : lscomp_max_stream_bytes_u32(x, y, z);
    return enqueue(s, r);
}

int64_t lscomp_server_submit_decompress(lscomp_server *s, const void *h_container, uint64_t len, void *h_out,
                                        uint64_t out_cap)
{
    if (!s || !h_container || !h_out) return -(int64_t)LSCOMP_ERR_ARG;
    lscomp_container_info info;
    const int st = lscomp_container_read_header((const uint8_t *)h_container, len, &info);
    if (st) return -(int64_t)st;
    const uint64_t out_bytes = (uint64_t)info.x * info.y * info.z * info.elem_bytes;
    if (out_cap < out_bytes) return -(int64_t)LSCOMP_ERR_CAPACITY;
    Request *r = new Request();
    r->op = 1;
    r->eb = info.elem_bytes;
    r->h_in = h_container;
    r->in_bytes = kHdr + info.stream_len;  // the header and the stream; anything after is not needed
    r->body_len = info.stream_len;
    r->x = info.x;
    r->y = info.y;
    r->z = info.z;
    memcpy(r->bins, info.bins, sizeof(r->bins));
    r->p = info.pooling;
    r->h_out = h_out;
    r->out_cap = out_cap;
    r->out_dev = out_bytes;
    return enqueue(s, r);
}

int lscomp_server_wait(lscomp_server *s, int64_t id, lscomp_server_result *res)
{
    if (!s) return LSCOMP_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return LSCOMP_ERR_ARG;
    Request *r = it->second;
    if (r->waited) return LSCOMP_ERR_ARG;  // another thread is waiting for this request
    r->waited = true;
    s->cv_done.wait(lk, [&] { return r->done; });
    if (res) {
        res->status = r->status;
        res->out_len = r->out_len;
        res->queued_ns = r->t_start - r->t_submit;
        res->service_ns = r->t_done - r->t_start;
        res->admit_ns = r->t_start;
        res->done_ns = r->t_done;
    }
    s->reqs.erase(id);
    delete r;
    return LSCOMP_OK;
}

int lscomp_server_stats(lscomp_server *s, uint64_t *rounds, uint64_t *batches, uint64_t *batched_requests)
{
    if (!s) return LSCOMP_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    if (rounds) *rounds = s->rounds;
    if (batches) *batches = s->batches;
    if (batched_requests) *batched_requests = s->batched_requests;
    return LSCOMP_OK;
}

}  // extern "C"
