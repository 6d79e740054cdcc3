// serve.cu -- a request-serving loop over the codec (include/lscomp.h,
// lscomp_server_*): host buffers in, host buffers out.
//
// Callers submit compress requests (a stack in host memory -> a container in
// host memory) and decompress requests (a container -> the stack) from any
// thread; one worker thread per server runs them on one device:
//
//   * admission: every request has a device footprint -- its input plus the
//     worst case of its output (a compress output is bounded by the header,
//     the 64-byte container header and 128 (uint16) or 248 (uint32) bytes
//     per block); a round admits waiting requests in arrival order while
//     their footprints fit the arena, so the device never runs out of memory
//     however the load arrives, and a request larger than the whole arena is
//     refused (LSCOMP_ERR_TOO_LARGE);
//   * continuous batching: the compress requests of a round of one element
//     type go to the GPU as one batch launch (lscomp_compress_batch_ex_*),
//     whatever their shapes, bins and pooling thresholds; decompress
//     requests of the round run one after the other;
//   * staging: inputs and outputs pass through pinned host memory of the
//     arena's size, so the device copies run at full link speed from
//     pageable caller buffers; the host-side copies of a round are split
//     over a pool of copy threads;
//   * every request records its time in the queue and in service.
//
// A request's output depends only on the request: batched or alone, its
// container is byte-identical to what lscomp_compress_container writes.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>
#include "lscomp.h"

namespace {

constexpr uint64_t kAlign = 256;
constexpr uint32_t kHdr = 64;

uint64_t align_up(uint64_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

uint64_t now_ns()
{
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
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
    void *h_out = nullptr;
    uint64_t out_cap = 0;
    uint64_t out_dev = 0;  // device bytes reserved for the output
    int status = 0;
    uint64_t out_len = 0;
    uint64_t t_submit = 0, t_start = 0, t_done = 0;
    bool done = false;
    uint64_t footprint() const { return align_up(in_bytes) + align_up(out_dev); }
};

// A fixed pool of host threads that runs lists of memcpy jobs, split into
// chunks of at most kChunk bytes.
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
    // copy every (dst, src, n) of the list; returns when all are done
    void copy(const std::vector<std::tuple<void *, const void *, uint64_t>> &jobs)
    {
        std::unique_lock<std::mutex> lk(mu_);
        for (const auto &j : jobs) {
            uint8_t *d = static_cast<uint8_t *>(std::get<0>(j));
            const uint8_t *s = static_cast<const uint8_t *>(std::get<1>(j));
            for (uint64_t o = 0, n = std::get<2>(j); o < n; o += kChunk)
                work_.push_back({d + o, s + o, n - o < kChunk ? n - o : kChunk});
        }
        pending_ += work_.size();
        cv_.notify_all();
        done_cv_.wait(lk, [&] { return pending_ == 0; });
    }

  private:
    static constexpr uint64_t kChunk = 4ull << 20;
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

constexpr unsigned kCopyThreads = 8;

}  // namespace

struct lscomp_server {
    int device = 0;
    cudaStream_t st = nullptr;
    lscomp_workspace *ws = nullptr;
    uint8_t *arena = nullptr;    // device
    uint8_t *staging = nullptr;  // pinned host, same size
    uint64_t arena_bytes = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> queue;
    std::unordered_map<int64_t, Request *> reqs;
    std::thread worker;
    bool stop = false;
    int64_t next_id = 1;
    uint64_t rounds = 0, batches = 0, batched_requests = 0;
    CopyPool *copies = nullptr;
};

namespace {

void finish(lscomp_server *s, Request *r, int status, uint64_t len)
{
    r->status = status;
    r->out_len = len;
    r->t_done = now_ns();
    r->done = true;
}

// One round: run the admitted requests, in place in the arena/staging.
void run_round(lscomp_server *s, std::vector<Request *> &round)
{
    // layout: each request's input then its output, 256-byte aligned
    std::vector<uint64_t> in_off(round.size()), out_off(round.size());
    uint64_t off = 0;
    for (size_t i = 0; i < round.size(); i++) {
        in_off[i] = off;
        off += align_up(round[i]->in_bytes);
        out_off[i] = off;
        off += align_up(round[i]->out_dev);
    }
    // inputs: caller -> pinned staging (copy threads) -> device
    std::vector<int> st(round.size(), LSCOMP_OK);
    {
        std::vector<std::tuple<void *, const void *, uint64_t>> jobs;
        for (size_t i = 0; i < round.size(); i++) jobs.emplace_back(s->staging + in_off[i], round[i]->h_in, round[i]->in_bytes);
        s->copies->copy(jobs);
    }
    for (size_t i = 0; i < round.size(); i++) {
        if (cudaMemcpyAsync(s->arena + in_off[i], s->staging + in_off[i], round[i]->in_bytes, cudaMemcpyHostToDevice,
                            s->st) != cudaSuccess)
            st[i] = LSCOMP_ERR_CUDA;
    }
    // compress requests of one element type: one batch launch, each stack
    // with its own bins and pooling threshold
    std::vector<bool> taken(round.size(), false);
    for (size_t i = 0; i < round.size(); i++) {
        Request *r = round[i];
        if (taken[i] || r->op != 0 || st[i]) continue;
        std::vector<size_t> grp;
        for (size_t j = i; j < round.size(); j++) {
            Request *q = round[j];
            if (!taken[j] && q->op == 0 && !st[j] && q->eb == r->eb) {
                grp.push_back(j);
                taken[j] = true;
            }
        }
        std::vector<lscomp_stack> stacks(grp.size());
        std::vector<uint32_t> bins(4 * grp.size());
        std::vector<float> pool(grp.size());
        std::vector<uint64_t> len(grp.size()), ref(grp.size());
        for (size_t g = 0; g < grp.size(); g++) {
            const size_t j = grp[g];
            stacks[g].d_in = s->arena + in_off[j];
            stacks[g].x = round[j]->x;
            stacks[g].y = round[j]->y;
            stacks[g].z = round[j]->z;
            stacks[g].d_out = s->arena + out_off[j] + kHdr;
            stacks[g].cap = round[j]->out_dev - kHdr;
            memcpy(&bins[4 * g], round[j]->bins, sizeof(round[j]->bins));
            pool[g] = round[j]->p;
        }
        const int b = r->eb == 2 ? lscomp_compress_batch_ex_u16(s->ws, stacks.data(), (uint32_t)grp.size(),
                                                                bins.data(), pool.data(), len.data(), ref.data(), s->st)
                                 : lscomp_compress_batch_ex_u32(s->ws, stacks.data(), (uint32_t)grp.size(),
                                                                bins.data(), pool.data(), len.data(), ref.data(), s->st);
        {
            std::lock_guard<std::mutex> lk(s->mu);  // lscomp_server_stats reads these under the lock
            s->batches++;
            s->batched_requests += grp.size();
        }
        for (size_t g = 0; g < grp.size(); g++) {
            const size_t j = grp[g];
            Request *q = round[j];
            if (b) {
                st[j] = b;
                continue;
            }
            if (kHdr + len[g] > q->out_cap) {
                st[j] = LSCOMP_ERR_CAPACITY;
                continue;
            }
            lscomp_container_write_header(s->staging + out_off[j], q->eb, q->x, q->y, q->z, q->bins, q->p, len[g],
                                          ref[g]);
            q->out_len = kHdr + len[g];
            if (cudaMemcpyAsync(s->staging + out_off[j] + kHdr, s->arena + out_off[j] + kHdr, len[g],
                                cudaMemcpyDeviceToHost, s->st) != cudaSuccess)
                st[j] = LSCOMP_ERR_CUDA;
        }
    }
    // decompress requests, one call each
    for (size_t i = 0; i < round.size(); i++) {
        Request *r = round[i];
        if (r->op != 1 || st[i]) continue;
        lscomp_container_info info;
        st[i] = lscomp_decompress_container(s->ws, s->arena + in_off[i], r->in_bytes, s->arena + out_off[i],
                                            r->out_dev, &info, s->st);
        if (st[i]) continue;
        r->out_len = (uint64_t)info.x * info.y * info.z * info.elem_bytes;
        if (cudaMemcpyAsync(s->staging + out_off[i], s->arena + out_off[i], r->out_len, cudaMemcpyDeviceToHost,
                            s->st) != cudaSuccess)
            st[i] = LSCOMP_ERR_CUDA;
    }
    const int sync = cudaStreamSynchronize(s->st) == cudaSuccess ? LSCOMP_OK : LSCOMP_ERR_CUDA;
    // outputs: pinned staging -> caller (copy threads)
    {
        std::vector<std::tuple<void *, const void *, uint64_t>> jobs;
        for (size_t i = 0; i < round.size(); i++)
            if (!(st[i] ? st[i] : sync)) jobs.emplace_back(round[i]->h_out, s->staging + out_off[i], round[i]->out_len);
        s->copies->copy(jobs);
    }
    std::lock_guard<std::mutex> lk(s->mu);
    for (size_t i = 0; i < round.size(); i++) {
        Request *r = round[i];
        int status = st[i] ? st[i] : sync;
        finish(s, r, status, status ? 0 : r->out_len);
    }
    s->rounds++;
    s->cv_done.notify_all();
}

void worker_main(lscomp_server *s)
{
    cudaSetDevice(s->device);
    for (;;) {
        std::vector<Request *> round;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] { return s->stop || !s->queue.empty(); });
            if (s->queue.empty()) return;  // stopping and drained
            // admit in arrival order while the footprints fit the arena
            uint64_t used = 0;
            while (!s->queue.empty()) {
                Request *r = s->queue.front();
                const uint64_t fp = r->footprint();
                if (used + fp > s->arena_bytes) break;
                used += fp;
                r->t_start = now_ns();
                round.push_back(r);
                s->queue.pop_front();
            }
        }
        run_round(s, round);
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
    s->queue.push_back(r);
    s->cv_work.notify_one();
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
    if (!st && cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess) st = LSCOMP_ERR_CUDA;
    if (!st && cudaMalloc(&s->arena, arena_bytes) != cudaSuccess) st = LSCOMP_ERR_NOMEM;
    if (!st && cudaMallocHost(&s->staging, arena_bytes) != cudaSuccess) st = LSCOMP_ERR_NOMEM;
    cudaSetDevice(prev);
    if (st) {
        lscomp_server_destroy(s);
        return st;
    }
    s->copies = new CopyPool(kCopyThreads);
    s->worker = std::thread(worker_main, s);
    *out = s;
    return LSCOMP_OK;
}

int lscomp_server_destroy(lscomp_server *s)
{
    if (!s) return LSCOMP_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv_work.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();  // runs what was submitted
    delete s->copies;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(s->device);
    if (s->arena) cudaFree(s->arena);
    if (s->staging) cudaFreeHost(s->staging);
    if (s->st) cudaStreamDestroy(s->st);
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
    r->out_dev = kHdr + (elem_bytes == 2 ? lscomp_max_stream_bytes_u16(x, y, z) : lscomp_max_stream_bytes_u32(x, y, z));
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
    r->h_in = h_container;
    r->in_bytes = len;
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
    s->cv_done.wait(lk, [&] { return r->done; });
    if (res) {
        res->status = r->status;
        res->out_len = r->out_len;
        res->queued_ns = r->t_start - r->t_submit;
        res->service_ns = r->t_done - r->t_start;
    }
    s->reqs.erase(it);
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
