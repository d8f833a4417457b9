// server.cpp -- continuous-batching request server over device-resident stripes.
//
// No counterpart in the reference (one synchronous call per stripe there).
// Requests (Encode / Reconstruct / ReconstructData / Verify of classic or
// Leopard stripes already in HBM) are queued by any host thread.  A server
// thread admits queued requests in arrival order while
//   * the bytes of work in flight stay under `inflight_budget`, and
//   * reconstruct outputs the caller did not provide fit in the server's HBM
//     arena (`arena_bytes`, carved at creation; released with
//     rsgpu_server_release),
// and launches each admitted group as one micro-batch on a free stream:
// classic stripes go into one persistent batched launch (batch.cu), Leopard
// stripes into their fused FFT kernels.  Classic and Leopard requests queue
// in separate lanes with their own streams, so microsecond-scale classic
// stripes never wait behind millisecond-scale Leopard stripes: the classic
// lane runs on high-priority streams and may use the whole byte budget
// except what Leopard work holds, while the Leopard lane is held to three
// quarters of it.  Requests that arrive while earlier micro-batches run are
// admitted as soon as a stream and budget free up, so their work overlaps
// on the device.  Host callbacks queued behind every micro-batch (and behind
// every Leopard stripe) timestamp completion.  No device code waits on the
// host, so nothing on the GPU can spin.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <thread>

#include "leo_host.h"
#include "rsgpu_internal.h"
#include "trace.h"

using Clock = std::chrono::steady_clock;

namespace rsgpu {
namespace {

constexpr int kLanes = 2;          // 0: classic stripes, 1: Leopard stripes
constexpr int kLeoPerSlot = 2;     // Leopard stripes per micro-batch (each is a full-GPU launch)

struct Req {
    uint64_t ticket = 0;
    int lane = 0;
    rsgpu_request *user = nullptr;  // output pointers are written back here
    rsgpu_request r{};
    std::vector<uint8_t *> shards;
    std::vector<uint8_t> present;
    std::vector<size_t> arena_off;  // arena blocks owned by this request
    size_t footprint = 0;           // algorithmic bytes (reads + writes)
    int status = RS_OK;
    int verify_slot = -1;
    Clock::time_point t_submit, t_launch, t_done;
    std::atomic<int64_t> t_kernel_done{0};  // set by a host callback (Leopard stripes)
};

struct Slot {
    rsgpu_server *sv = nullptr;
    int lane = 0;
    cudaStream_t stream = nullptr;
    rsgpu_batch *batch = nullptr;
    std::vector<Req *> reqs;
    bool busy = false;
    std::atomic<bool> finished{false};
    Clock::time_point t_done;
};

// First-fit allocator over [0, size) in 256-byte units.
struct Arena {
    size_t size = 0;
    std::map<size_t, size_t> free_blocks;  // offset -> length
    std::map<size_t, size_t> used;         // offset -> length
    void init(size_t n) {
        size = n;
        free_blocks.clear();
        used.clear();
        if (n) free_blocks[0] = n;
    }
    bool alloc(size_t n, size_t *off) {
        n = (n + 255) & ~(size_t)255;
        for (auto it = free_blocks.begin(); it != free_blocks.end(); ++it)
            if (it->second >= n) {
                *off = it->first;
                const size_t rest = it->second - n;
                const size_t start = it->first + n;
                free_blocks.erase(it);
                if (rest) free_blocks[start] = rest;
                used[*off] = n;
                return true;
            }
        return false;
    }
    void release(size_t off) {
        auto u = used.find(off);
        if (u == used.end()) return;
        size_t start = off, len = u->second;
        used.erase(u);
        auto nx = free_blocks.lower_bound(start);
        if (nx != free_blocks.end() && start + len == nx->first) {
            len += nx->second;
            nx = free_blocks.erase(nx);
        }
        if (nx != free_blocks.begin()) {
            auto pv = std::prev(nx);
            if (pv->first + pv->second == start) {
                start = pv->first;
                len += pv->second;
                free_blocks.erase(pv);
            }
        }
        free_blocks[start] = len;
    }
};

}  // namespace
}  // namespace rsgpu

using namespace rsgpu;

struct rsgpu_server {
    rsgpu_ctx *ctx = nullptr;
    size_t inflight_budget = 0;
    int max_batch = 0;
    uint8_t *arena_ptr = nullptr;
    Arena arena;
    std::vector<Slot *> slots;
    std::map<std::tuple<int, int, int>, rsgpu_encoder *> encoders;

    std::mutex mu;  // guards everything below
    std::condition_variable cv;
    std::deque<Req *> queue[kLanes]; // submitted, not admitted
    std::map<uint64_t, Req *> live;  // admitted or done, not yet polled/released
    std::deque<Req *> done;          // completed, not yet polled
    uint64_t next_ticket = 1;
    size_t inflight[kLanes] = {0, 0};
    bool stop = false;
    std::thread worker;

    // statistics
    uint64_t n_submitted = 0, n_completed = 0, n_failed = 0;
    double bytes_done = 0;
    size_t max_inflight = 0;
    std::vector<double> latencies_us;
    Clock::time_point t_first, t_last;
    bool any = false;
    std::atomic<int> verify_count{0};
    int *d_verify = nullptr;
    int verify_cap = 0;
};

namespace {

void CUDART_CB on_slot_done(void *arg) {
    auto *s = static_cast<Slot *>(arg);
    s->t_done = Clock::now();
    s->finished.store(true, std::memory_order_release);
    s->sv->cv.notify_all();
}

void CUDART_CB on_req_done(void *arg) {
    auto *q = static_cast<Req *>(arg);
    q->t_kernel_done.store(Clock::now().time_since_epoch().count(), std::memory_order_release);
}

bool queues_empty(const rsgpu_server *sv) {
    for (int l = 0; l < kLanes; l++)
        if (!sv->queue[l].empty()) return false;
    return true;
}

size_t total_inflight(const rsgpu_server *sv) {
    size_t t = 0;
    for (int l = 0; l < kLanes; l++) t += sv->inflight[l];
    return t;
}

int encoder_for(rsgpu_server *sv, const rsgpu_request &r, rsgpu_encoder **out) {
    auto key = std::make_tuple(r.data_shards, r.parity_shards, r.leopard);
    auto it = sv->encoders.find(key);
    if (it != sv->encoders.end()) {
        *out = it->second;
        return RS_OK;
    }
    rsgpu_options o;
    rsgpu_options_init(&o);
    o.leopard = r.leopard;
    rsgpu_encoder *e = nullptr;
    int rc = rsgpu_encoder_new(sv->ctx, r.data_shards, r.parity_shards, &o, &e);
    if (rc) return rc;
    sv->encoders[key] = e;
    *out = e;
    return RS_OK;
}

// Outputs a reconstruct request will write (classic: the decode plan's
// outputs; Leopard: every missing data shard, parity too unless data-only).
int outputs_of(rsgpu_server *sv, Req *q, rsgpu_encoder *e, std::vector<int> &outs) {
    outs.clear();
    const bool data_only = q->r.op == RS_JOB_RECONSTRUCT_DATA;
    if (e->codec == RS_CODEC_CLASSIC) {
        std::vector<uint8_t> rows;
        std::vector<int> in_idx;
        return classic_decode_plan(e, q->present.data(), data_only, nullptr, 0, rows, outs, in_idx);
    }
    (void)sv;
    int np = 0, dp = 0;
    for (int i = 0; i < e->total; i++)
        if (q->present[i]) {
            np++;
            if (i < e->k) dp++;
        }
    if (np == 0) return RS_ERR_SHARD_NO_DATA;
    if (np == e->total || (data_only && dp == e->k)) return RS_OK;
    if (np < e->k) return RS_ERR_TOO_FEW_SHARDS;
    for (int i = 0; i < e->total; i++)
        if (!q->present[i] && (i < e->k || !data_only)) outs.push_back(i);
    return RS_OK;
}

void finish(rsgpu_server *sv, Req *q, Clock::time_point t) {
    q->t_done = t;
    if (q->status == RS_OK) {
        sv->n_completed++;
        sv->bytes_done += (double)q->footprint;
    } else {
        sv->n_failed++;
    }
    sv->latencies_us.push_back(std::chrono::duration<double, std::micro>(t - q->t_submit).count());
    if (!sv->any || t > sv->t_last) sv->t_last = t;
    sv->done.push_back(q);
}

// Admits queued requests into slot s (caller holds sv->mu).  Returns the
// number admitted.
int admit(rsgpu_server *sv, Slot *s) {
    int n = 0;
    auto &queue = sv->queue[s->lane];
    const int max_n = s->lane == 1 ? std::min(sv->max_batch, kLeoPerSlot) : sv->max_batch;
    const size_t cap = s->lane == 1 ? sv->inflight_budget - sv->inflight_budget / 4
                                    : sv->inflight_budget - std::min(sv->inflight_budget, sv->inflight[1]);
    size_t &inflight = sv->inflight[s->lane];
    while (!queue.empty() && n < max_n) {
        Req *q = queue.front();
        rsgpu_encoder *e = nullptr;
        int rc = encoder_for(sv, q->r, &e);
        std::vector<int> outs;
        if (rc == RS_OK && (q->r.op == RS_JOB_RECONSTRUCT || q->r.op == RS_JOB_RECONSTRUCT_DATA))
            rc = outputs_of(sv, q, e, outs);
        if (rc != RS_OK) {  // fails immediately, no device work
            queue.pop_front();
            q->status = rc;
            finish(sv, q, Clock::now());
            continue;
        }
        // footprint: every shard read plus every shard written
        const size_t sz = q->r.shard_size;
        size_t fp = 0;
        if (q->r.op == RS_JOB_ENCODE) fp = (size_t)e->total * sz;
        else if (q->r.op == RS_JOB_VERIFY) fp = (size_t)e->total * sz;
        else {
            size_t reads = (size_t)e->k;  // classic reads the first k present shards
            if (e->codec != RS_CODEC_CLASSIC) {
                reads = 0;  // Leopard reads every present shard
                for (uint8_t pr : q->present) reads += pr ? 1 : 0;
            }
            fp = (reads + outs.size()) * sz;
        }
        if (inflight > 0 && inflight + fp > cap) break;
        // reconstruct outputs without a caller buffer come from the arena
        std::vector<size_t> offs;
        bool ok = true;
        for (int o : outs)
            if (!q->shards[o]) {
                size_t off;
                if (!sv->arena.alloc(sz, &off)) {
                    ok = false;
                    break;
                }
                offs.push_back(off);
                q->shards[o] = sv->arena_ptr + off;
            }
        if (!ok) {
            for (size_t off : offs) sv->arena.release(off);
            for (int o : outs)
                if (q->user && !q->user->shards[o]) q->shards[o] = nullptr;
            if (n == 0 && total_inflight(sv) == 0 && sv->arena.used.empty()) {
                queue.pop_front();  // can never fit
                q->status = RS_ERR_NOMEM;
                finish(sv, q, Clock::now());
                continue;
            }
            break;
        }
        q->arena_off = offs;
        q->footprint = fp;
        queue.pop_front();
        inflight += fp;
        sv->max_inflight = std::max(sv->max_inflight, total_inflight(sv));
        s->reqs.push_back(q);
        n++;
    }
    return n;
}

// Plans and launches slot s's requests (caller holds sv->mu).
void launch(rsgpu_server *sv, Slot *s) {
    RS_TRACE(s->lane ? "rsgpu_server micro-batch (leopard)" : "rsgpu_server micro-batch (classic)");
    const Clock::time_point now = Clock::now();
    for (Req *q : s->reqs) q->t_launch = now;
    rsgpu_batch_clear(s->batch);
    bool has_classic = false;
    std::vector<Req *> leo;
    for (Req *q : s->reqs) {
        rsgpu_encoder *e = nullptr;
        encoder_for(sv, q->r, &e);
        if (e->codec != RS_CODEC_CLASSIC) {
            leo.push_back(q);
            continue;
        }
        rsgpu_stripe st{};
        st.op = q->r.op;
        st.data_shards = q->r.data_shards;
        st.parity_shards = q->r.parity_shards;
        st.shard_size = q->r.shard_size;
        st.shards = q->shards.data();
        st.present = q->present.data();
        q->verify_slot = -1;
        const int before = batch_stripe_count(s->batch);
        int rc = rsgpu_batch_add(s->batch, &st, 1);
        if (rc) q->status = rc;
        else {
            q->verify_slot = before;
            has_classic = true;
        }
    }
    cudaStream_t st = s->stream;
    if (has_classic) {
        int rc = batch_run_on(s->batch, RS_BATCH_PERSISTENT, st);
        if (rc)
            for (Req *q : s->reqs) q->status = q->status ? q->status : rc;
    }
    for (Req *q : leo) {
        rsgpu_encoder *e = nullptr;
        encoder_for(sv, q->r, &e);
        int rc = RS_OK;
        if (q->r.op == RS_JOB_ENCODE) rc = leo_encode_enqueue(e, q->shards.data(), q->r.shard_size, st);
        else if (q->r.op == RS_JOB_VERIFY) rc = RS_ERR_NOT_SUPPORTED;
        else
            rc = leo_reconstruct_enqueue(e, q->shards.data(), q->present.data(), q->r.shard_size,
                                         q->r.op == RS_JOB_RECONSTRUCT, st);
        if (rc) q->status = rc;
        else if (cudaLaunchHostFunc(st, on_req_done, q) != cudaSuccess) q->t_kernel_done.store(0);
    }
    s->finished.store(false);
    s->busy = true;
    cudaError_t ce = cudaLaunchHostFunc(st, on_slot_done, s);
    if (ce != cudaSuccess) {
        cuda_status(ce, "cudaLaunchHostFunc");
        cudaStreamSynchronize(st);
        on_slot_done(s);
    }
}

void reap(rsgpu_server *sv, Slot *s) {
    std::vector<int> ok;
    const int nb = batch_stripe_count(s->batch);
    bool any_verify = false;
    for (Req *q : s->reqs) any_verify |= q->r.op == RS_JOB_VERIFY;
    if (any_verify && nb > 0) {
        ok.resize(nb);
        if (batch_read_flags(s->batch, ok.data(), nb, s->stream) != RS_OK) ok.assign(nb, 0);
    }
    for (Req *q : s->reqs) {
        if (q->status == RS_OK && q->r.op == RS_JOB_VERIFY && q->user)
            q->user->result = (q->verify_slot >= 0 && q->verify_slot < (int)ok.size()) ? ok[q->verify_slot] : 0;
        if (q->user)
            for (size_t i = 0; i < q->shards.size(); i++) q->user->shards[i] = q->shards[i];
        sv->inflight[q->lane] -= q->footprint;
        const int64_t t = q->t_kernel_done.load(std::memory_order_acquire);
        finish(sv, q, t ? Clock::time_point(Clock::duration(t)) : s->t_done);
    }
    s->reqs.clear();
    s->busy = false;
}

void worker_loop(rsgpu_server *sv) {
    cudaSetDevice(sv->ctx->device);
    std::unique_lock<std::mutex> lk(sv->mu);
    while (true) {
        bool progress = false;
        for (Slot *s : sv->slots)
            if (s->busy && s->finished.load(std::memory_order_acquire)) {
                reap(sv, s);
                progress = true;
            }
        if (sv->stop && queues_empty(sv)) {
            bool busy = false;
            for (Slot *s : sv->slots) busy |= s->busy;
            if (!busy) break;
        }
        for (Slot *s : sv->slots) {
            if (s->busy || sv->queue[s->lane].empty()) continue;
            if (admit(sv, s) > 0) {
                launch(sv, s);
                progress = true;
            }
        }
        if (!progress) {
            bool busy = false;
            for (Slot *s : sv->slots) busy |= s->busy;
            // Idle: sleep until a submit or shutdown (both change the state
            // under the lock before notifying, so no wakeup is lost).  With work on the device, poll
            // every 20 us as well: completion callbacks notify without the
            // lock and may race with this check.
            if (!busy && queues_empty(sv) && !sv->stop) sv->cv.wait(lk);
            else sv->cv.wait_for(lk, std::chrono::microseconds(20));
        } else {
            sv->cv.notify_all();
        }
    }
    sv->cv.notify_all();
}

}  // namespace

extern "C" {

int rsgpu_server_create(rsgpu_ctx *ctx, size_t arena_bytes, size_t inflight_budget, int max_batch, int streams,
                        rsgpu_server **out) {
    if (!ctx || !out || streams < 1 || streams > 16 || max_batch < 1 || inflight_budget == 0)
        return RS_ERR_INVALID_INPUT;
    auto *sv = new rsgpu_server();
    sv->ctx = ctx;
    sv->inflight_budget = inflight_budget;
    sv->max_batch = max_batch;
    RS_CUDA(cudaSetDevice(ctx->device));
    if (arena_bytes) {
        cudaError_t e = cudaMalloc(&sv->arena_ptr, arena_bytes);
        if (e != cudaSuccess) {
            delete sv;
            return cuda_status(e, "server arena");
        }
    }
    sv->arena.init(arena_bytes);
    int prio_low = 0, prio_high = 0;
    cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
    for (int lane = 0; lane < kLanes; lane++)
        for (int i = 0; i < streams; i++) {
            auto *s = new Slot();
            s->sv = sv;
            s->lane = lane;
            cudaStreamCreateWithPriority(&s->stream, cudaStreamNonBlocking, lane == 0 ? prio_high : prio_low);
            rsgpu_batch_create(ctx, nullptr, &s->batch);
            sv->slots.push_back(s);
        }
    sv->worker = std::thread(worker_loop, sv);
    *out = sv;
    return RS_OK;
}

int rsgpu_server_submit(rsgpu_server *sv, rsgpu_request *r, uint64_t *ticket) {
    if (!sv || !r || !r->shards) return RS_ERR_INVALID_INPUT;
    const int n = r->data_shards + r->parity_shards;
    if (n <= 0 || r->shard_size == 0) return RS_ERR_INVALID_INPUT;
    if (r->op < RS_JOB_ENCODE || r->op > RS_JOB_VERIFY) return RS_ERR_INVALID_INPUT;
    auto *q = new Req();
    q->user = r;
    q->r = *r;
    q->lane = r->leopard ? 1 : 0;
    q->shards.assign(r->shards, r->shards + n);
    if (r->present) q->present.assign(r->present, r->present + n);
    else q->present.assign(n, 1);
    q->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        if (sv->stop) {
            delete q;
            return RS_ERR_INVALID_INPUT;
        }
        q->ticket = sv->next_ticket++;
        sv->live[q->ticket] = q;
        sv->queue[q->lane].push_back(q);
        sv->n_submitted++;
        if (!sv->any) {
            sv->any = true;
            sv->t_first = q->t_submit;
            sv->t_last = q->t_submit;
        }
    }
    sv->cv.notify_all();
    if (ticket) *ticket = q->ticket;
    return RS_OK;
}

int rsgpu_server_poll(rsgpu_server *sv, rsgpu_completion *out, int max) {
    if (!sv || (!out && max > 0)) return RS_ERR_INVALID_INPUT;
    std::lock_guard<std::mutex> lk(sv->mu);
    int n = 0;
    while (n < max && !sv->done.empty()) {
        Req *q = sv->done.front();
        sv->done.pop_front();
        out[n].ticket = q->ticket;
        out[n].tag = q->r.tag;
        out[n].status = q->status;
        out[n].latency_us = std::chrono::duration<double, std::micro>(q->t_done - q->t_submit).count();
        out[n].queue_us = q->t_launch == Clock::time_point()
                              ? out[n].latency_us
                              : std::chrono::duration<double, std::micro>(q->t_launch - q->t_submit).count();
        n++;
    }
    return n;
}

int rsgpu_server_release(rsgpu_server *sv, uint64_t ticket) {
    if (!sv) return RS_ERR_INVALID_INPUT;
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->live.find(ticket);
    if (it == sv->live.end()) return RS_ERR_INVALID_INPUT;
    Req *q = it->second;
    if (q->t_done == Clock::time_point()) return RS_ERR_INVALID_INPUT;  // still running
    for (size_t off : q->arena_off) sv->arena.release(off);
    sv->live.erase(it);
    delete q;
    sv->cv.notify_all();
    return RS_OK;
}

int rsgpu_server_wait_idle(rsgpu_server *sv, int timeout_ms) {
    if (!sv) return RS_ERR_INVALID_INPUT;
    std::unique_lock<std::mutex> lk(sv->mu);
    const auto deadline = Clock::now() + std::chrono::milliseconds(timeout_ms);
    while (true) {
        bool busy = !queues_empty(sv);
        for (Slot *s : sv->slots) busy |= s->busy;
        if (!busy) return RS_OK;
        if (sv->cv.wait_until(lk, deadline) == std::cv_status::timeout) {
            busy = !queues_empty(sv);
            for (Slot *s : sv->slots) busy |= s->busy;
            return busy ? RS_ERR_TIMEOUT : RS_OK;
        }
    }
}

int rsgpu_server_get_stats(rsgpu_server *sv, rsgpu_server_stats *st) {
    if (!sv || !st) return RS_ERR_INVALID_INPUT;
    std::lock_guard<std::mutex> lk(sv->mu);
    memset(st, 0, sizeof *st);
    st->submitted = sv->n_submitted;
    st->completed = sv->n_completed;
    st->failed = sv->n_failed;
    st->bytes = sv->bytes_done;
    st->max_inflight_bytes = (double)sv->max_inflight;
    st->elapsed_s = sv->any ? std::chrono::duration<double>(sv->t_last - sv->t_first).count() : 0;
    std::vector<double> l = sv->latencies_us;
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        auto pct = [&](double q) { return l[std::min(l.size() - 1, (size_t)(q * (l.size() - 1) + 0.5))]; };
        st->p50_us = pct(0.50);
        st->p99_us = pct(0.99);
        st->max_us = l.back();
        double s = 0;
        for (double x : l) s += x;
        st->mean_us = s / l.size();
    }
    return RS_OK;
}

int rsgpu_server_reset_stats(rsgpu_server *sv) {
    if (!sv) return RS_ERR_INVALID_INPUT;
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->n_submitted = sv->n_completed = sv->n_failed = 0;
    sv->bytes_done = 0;
    sv->max_inflight = total_inflight(sv);
    sv->latencies_us.clear();
    sv->any = false;
    return RS_OK;
}

// Open-loop load generator: submits reqs[i] at arrival_us[i] (microseconds
// after the call) from a dedicated thread; returns once all are submitted.
int rsgpu_server_replay(rsgpu_server *sv, rsgpu_request *reqs, const double *arrival_us, int n,
                        uint64_t *tickets) {
    if (!sv || (n > 0 && (!reqs || !arrival_us))) return RS_ERR_INVALID_INPUT;
    int rc = RS_OK;
    std::thread t([&]() {
        const auto t0 = Clock::now();
        for (int i = 0; i < n; i++) {
            const auto at = t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double, std::micro>(arrival_us[i]));
            while (Clock::now() < at) {
                const auto left = at - Clock::now();
                if (left > std::chrono::microseconds(200)) std::this_thread::sleep_for(left - std::chrono::microseconds(100));
                else std::this_thread::yield();
            }
            int r = rsgpu_server_submit(sv, &reqs[i], tickets ? &tickets[i] : nullptr);
            if (r && rc == RS_OK) rc = r;
        }
    });
    t.join();
    return rc;
}

int rsgpu_server_destroy(rsgpu_server *sv) {
    if (!sv) return RS_OK;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;
    }
    sv->cv.notify_all();
    if (sv->worker.joinable()) sv->worker.join();
    for (Slot *s : sv->slots) {
        cudaStreamSynchronize(s->stream);
        rsgpu_batch_destroy(s->batch);
        cudaStreamDestroy(s->stream);
        delete s;
    }
    for (auto &kv : sv->encoders) rsgpu_encoder_free(kv.second);
    for (auto &kv : sv->live) delete kv.second;
    if (sv->arena_ptr) cudaFree(sv->arena_ptr);
    delete sv;
    return RS_OK;
}

}  // extern "C"
