// serve.cpp — continuous-batching product server (nbg_server_*).
//
// Requests (one product each) are submitted from any thread and return a
// ticket at once.  A worker thread owned by the server turns whatever is
// pending into a batch as soon as a batch slot and device memory are free,
// launches it asynchronously, and keeps forming the next batch while earlier
// ones run: up to MAX_FLIGHT batches are in flight on their own streams, so
// requests that arrive while others are on the GPU overlap with them.
// Admission is by HBM footprint: every batch's descriptors, job lists,
// workspace and (for host requests) staged operands and results are carved
// from one arena of `hbm_budget` bytes; a batch is cut where the arena is
// full, and requests wait until retired batches free their space.
// Completion is detected with CUDA events; each request records its submit
// and completion times for the p50/p99 latency report.
//
// Requests are either device-resident (operands and result in device
// memory: no copies) or host (operands gathered into pinned staging, copied
// in and out with the batch).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/nbgpu.h"
#include "engine.h"

using namespace nbg;

namespace {

constexpr int MAX_FLIGHT = 3;

double now_us() {
    return std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

inline size_t up256(size_t x) { return (x + 255) / 256 * 256; }

// First-fit allocator over [0, size).
class Arena {
   public:
    void reset(size_t size) {
        free_.clear();
        free_[0] = size;
        size_ = size;
    }
    bool alloc(size_t n, size_t& off) {
        n = up256(n);
        for (auto it = free_.begin(); it != free_.end(); ++it)
            if (it->second >= n) {
                off = it->first;
                const size_t rest = it->second - n;
                const size_t at = it->first + n;
                free_.erase(it);
                if (rest) free_[at] = rest;
                return true;
            }
        return false;
    }
    void release(size_t off, size_t n) {
        n = up256(n);
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    size_t size() const { return size_; }

   private:
    std::map<size_t, size_t> free_;
    size_t size_ = 0;
};

struct Request {
    ProdIn in;
    bool host = false;
    double t_submit = 0, t_done = 0;
    int state = 0;  // 0 pending, 1 in flight, 2 done, 3 failed
    int rc = 0;
};

struct Flight {
    std::vector<int64_t> ids;
    BatchBuild bb;
    size_t off = 0, bytes = 0;
    int slot = -1;
    cudaEvent_t done = nullptr;
    cudaStream_t st = nullptr;
    // host requests: operands and results staged in the slot's pinned buffer
    char* hstage = nullptr;
    std::vector<std::pair<size_t, int64_t>> host_results;  // staging offset, request id
};

}  // namespace

struct nbg_server {
    nbg_server_opts opts;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<int64_t> pending;
    std::unordered_map<int64_t, Request> reqs;
    std::atomic<bool> stop{false};
    int64_t next_id = 1;
    char* dmem = nullptr;
    Arena arena;
    std::deque<Flight> flights;
    // one stream and one pinned staging buffer per flight slot
    cudaStream_t streams[MAX_FLIGHT] = {};
    char* pinned[MAX_FLIGHT] = {};
    size_t pinned_bytes[MAX_FLIGHT] = {};
    bool slot_busy[MAX_FLIGHT] = {};
    std::vector<double> latencies_us;
    int64_t completed = 0, failed = 0;
    double limbs_done = 0, t_first = 0, t_last = 0;

    void run();
    bool launch_batch(std::unique_lock<std::mutex>& lk);
    void retire(std::unique_lock<std::mutex>& lk, bool wait_one);
};

// Forms one batch from the front of the queue, within the arena.  Called with
// the server lock held; the engine lock is taken inside.
bool nbg_server::launch_batch(std::unique_lock<std::mutex>& lk) {
    if (pending.empty() || (int)flights.size() >= MAX_FLIGHT) return false;
    std::vector<int64_t> ids;
    std::vector<ProdIn> in;
    size_t host_in = 0, host_out = 0;
    const int64_t maxb = opts.max_batch > 0 ? opts.max_batch : 100000;
    for (int64_t id : pending) {
        if ((int64_t)ids.size() >= maxb) break;
        const Request& q = reqs[id];
        ids.push_back(id);
        in.push_back(q.in);
        if (q.host) {  // each operand padded on its own, as laid out below
            host_in += up256(8 * (size_t)q.in.m) + (q.in.sqr ? 0 : up256(8 * (size_t)q.in.n));
            host_out += up256(8 * (size_t)(q.in.m + q.in.n));
        }
    }
    Engine& E = g_eng;
    std::lock_guard<std::recursive_mutex> elk(E.mu);
    // shrink the batch until it fits in the free arena
    Flight f;
    size_t off = 0;
    for (;;) {
        int rc = build_batch(E, in.data(), (int64_t)in.size(), f.bb);
        if (rc) {  // a request the engine refuses (size): fail it alone
            if (in.size() == 1) {
                Request& q = reqs[ids[0]];
                q.state = 3;
                q.rc = rc;
                q.t_done = now_us();
                failed++;
                pending.pop_front();
                cv_done.notify_all();
                return true;
            }
            in.resize(in.size() / 2);
            ids.resize(in.size());
            continue;
        }
        host_in = host_out = 0;
        for (int64_t id : ids)
            if (reqs[id].host) {
                const ProdIn& q = reqs[id].in;
                host_in += up256(8 * (size_t)q.m) + (q.sqr ? 0 : up256(8 * (size_t)q.n));
                host_out += up256(8 * (size_t)(q.m + q.n));
            }
        f.bytes = up256(f.bb.dev_bytes) + host_in + host_out;
        if (arena.alloc(f.bytes, off)) break;
        if (f.bytes > arena.size() && in.size() == 1) {  // can never fit
            Request& q = reqs[ids[0]];
            q.state = 3;
            q.rc = fail(NBG_ENOMEM, "request needs %zu bytes, over the server's HBM budget", f.bytes);
            q.t_done = now_us();
            failed++;
            pending.pop_front();
            cv_done.notify_all();
            return true;
        }
        if (in.size() == 1) return false;  // wait for memory to free up
        in.resize(in.size() / 2);
        ids.resize(in.size());
    }
    f.off = off;
    char* base = dmem + off;
    int slot = 0;
    while (slot_busy[slot]) slot++;  // flights.size() < MAX_FLIGHT: a slot is free
    f.slot = slot;
    f.st = streams[slot];
    // host requests: gather operands into the slot's pinned staging, one copy in
    const size_t dev_in = up256(f.bb.dev_bytes), dev_out = dev_in + host_in;
    if (host_in) {
        if (pinned_bytes[slot] < host_in + host_out) {
            if (pinned[slot]) cudaFreeHost(pinned[slot]);
            pinned[slot] = nullptr;
            pinned_bytes[slot] = 0;
            const size_t want = std::max(host_in + host_out, (size_t)(8 << 20));
            if (cudaMallocHost(&pinned[slot], want) != cudaSuccess) {
                cudaGetLastError();
                arena.release(off, f.bytes);
                return false;
            }
            pinned_bytes[slot] = want;
        }
        f.hstage = pinned[slot];
    }
    slot_busy[slot] = true;
    size_t ho = 0, ro = 0;
    for (size_t k = 0; k < ids.size(); k++) {
        Request& q = reqs[ids[k]];
        DProd& P = f.bb.prods[k];
        if (q.host) {
            const size_t na = 8 * (size_t)q.in.m;
            memcpy(f.hstage + ho, q.in.a, na);
            P.a = (const uint64_t*)(base + dev_in + ho);
            ho += up256(na);
            if (q.in.sqr) {
                P.b = P.a;
            } else {
                const size_t nb = 8 * (size_t)q.in.n;
                memcpy(f.hstage + ho, q.in.b, nb);
                P.b = (const uint64_t*)(base + dev_in + ho);
                ho += up256(nb);
            }
            P.r = (uint64_t*)(base + dev_out + ro);
            f.host_results.push_back({host_in + ro, ids[k]});
            ro += up256(8 * (size_t)(q.in.m + q.in.n));
        }
        q.state = 1;
    }
    bool ok = true;
    if (host_in) ok = cudaMemcpyAsync(base + dev_in, f.hstage, host_in, cudaMemcpyHostToDevice, f.st) == cudaSuccess;
    ok = ok && upload_batch(E, f.bb, base, f.st) == NBG_OK;
    ok = ok && run_launches(E, f.bb, base, f.st) == NBG_OK;
    if (ok && host_out)
        ok = cudaMemcpyAsync(f.hstage + host_in, base + dev_out, host_out, cudaMemcpyDeviceToHost, f.st) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&f.done, cudaEventDisableTiming) == cudaSuccess;
    ok = ok && cudaEventRecord(f.done, f.st) == cudaSuccess;
    for (size_t k = 0; k < ids.size(); k++) pending.pop_front();
    f.ids = std::move(ids);
    if (!ok) {
        // the stream's work is abandoned: fail the batch's requests
        cudaStreamSynchronize(f.st);
        for (int64_t id : f.ids) {
            Request& q = reqs[id];
            q.state = 3;
            q.rc = NBG_ECUDA;
            q.t_done = now_us();
            failed++;
        }
        if (f.done) cudaEventDestroy(f.done);
        arena.release(f.off, f.bytes);
        slot_busy[f.slot] = false;
        cv_done.notify_all();
        return true;
    }
    flights.push_back(std::move(f));
    (void)lk;
    return true;
}

// Marks finished batches done.  wait_one: block on the oldest if nothing finished.
void nbg_server::retire(std::unique_lock<std::mutex>& lk, bool wait_one) {
    bool any = false;
    for (auto it = flights.begin(); it != flights.end();) {
        cudaError_t q = cudaEventQuery(it->done);
        if (q == cudaErrorNotReady) {
            ++it;
            continue;
        }
        const double t = now_us();
        for (const auto& hr : it->host_results) {
            Request& rq = reqs[hr.second];
            memcpy(rq.in.r, it->hstage + hr.first, 8 * (size_t)(rq.in.m + rq.in.n));
        }
        for (int64_t id : it->ids) {
            Request& rq = reqs[id];
            rq.state = q == cudaSuccess ? 2 : 3;
            rq.rc = q == cudaSuccess ? NBG_OK : NBG_ECUDA;
            rq.t_done = t;
            if (q == cudaSuccess) {
                completed++;
                latencies_us.push_back(t - rq.t_submit);
                limbs_done += (double)(rq.in.m + rq.in.n);
                t_last = t;
            } else {
                failed++;
            }
        }
        cudaEventDestroy(it->done);
        arena.release(it->off, it->bytes);
        slot_busy[it->slot] = false;
        it = flights.erase(it);
        any = true;
    }
    if (any) {
        cv_done.notify_all();
        return;
    }
    if (wait_one && !flights.empty()) {
        cudaEvent_t ev = flights.front().done;
        lk.unlock();
        cudaEventSynchronize(ev);
        lk.lock();
    }
}

void nbg_server::run() {
    std::unique_lock<std::mutex> lk(mu);
    while (!stop.load() || !pending.empty() || !flights.empty()) {
        retire(lk, false);
        bool launched = false;
        while (launch_batch(lk)) launched = true;
        if (launched) continue;
        if (!flights.empty()) {
            // a batch slot or memory will free up when the oldest batch ends;
            // new arrivals also wake us
            if (pending.empty()) cv_work.wait_for(lk, std::chrono::microseconds(50));
            else retire(lk, true);
        } else if (!stop.load()) {
            cv_work.wait_for(lk, std::chrono::milliseconds(5));
        }
    }
}

extern "C" {

int nbg_server_create(const nbg_server_opts* opts, nbg_server** out) {
    if (!opts || !out || opts->hbm_budget_bytes < (int64_t)(16 << 20)) return fail(NBG_EINVAL, "bad server options");
    *out = nullptr;
    {
        std::lock_guard<std::recursive_mutex> lk(g_eng.mu);
        int rc = g_eng.ensure();
        if (rc) return rc;
    }
    nbg_server* s = new nbg_server();
    s->opts = *opts;
    if (cudaMalloc(&s->dmem, (size_t)opts->hbm_budget_bytes) != cudaSuccess) {
        cudaGetLastError();
        delete s;
        return fail(NBG_ENOMEM, "server arena of %lld bytes unavailable", (long long)opts->hbm_budget_bytes);
    }
    s->arena.reset((size_t)opts->hbm_budget_bytes);
    for (int i = 0; i < MAX_FLIGHT; i++) cudaStreamCreateWithFlags(&s->streams[i], cudaStreamNonBlocking);
    s->worker = std::thread([s] { s->run(); });
    *out = s;
    return NBG_OK;
}

static int submit(nbg_server* s, const nbg_desc* d, bool host, int64_t* ticket) {
    if (!s || !d || !ticket) return fail(NBG_EINVAL, "null argument");
    ProdIn q;
    if (!d->r || !d->a || d->m < 1) return fail(NBG_EINVAL, "bad request");
    const bool sqr = d->b == nullptr || (d->b == d->a && d->n == d->m);
    if (!sqr && d->n < 1) return fail(NBG_EINVAL, "bad request");
    q.a = d->a;
    q.b = sqr ? d->a : d->b;
    q.r = d->r;
    q.m = d->m;
    q.n = sqr ? d->m : d->n;
    q.sqr = sqr;
    if (host) {
        q.bits_a = magnitude_bits(d->a, d->m);
        q.bits_b = sqr ? q.bits_a : magnitude_bits(d->b, q.n);
    } else {
        if (d->bits_a < 1 || (!sqr && d->bits_b < 1))
            return fail(NBG_EINVAL, "device requests carry their magnitude bits");
        q.bits_a = d->bits_a;
        q.bits_b = sqr ? d->bits_a : d->bits_b;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop.load()) return fail(NBG_EINVAL, "server is stopping");
    if (s->opts.max_queue > 0 && (int64_t)s->pending.size() >= s->opts.max_queue)
        return fail(NBG_EBUSY, "queue full");
    const int64_t id = s->next_id++;
    Request& r = s->reqs[id];
    r.in = q;
    r.host = host;
    r.t_submit = now_us();
    if (s->t_first == 0) s->t_first = r.t_submit;
    s->pending.push_back(id);
    *ticket = id;
    s->cv_work.notify_one();
    return NBG_OK;
}

int nbg_submit(nbg_server* s, const nbg_desc* d, int64_t* ticket) { return submit(s, d, true, ticket); }
int nbg_submit_dev(nbg_server* s, const nbg_desc* d, int64_t* ticket) { return submit(s, d, false, ticket); }

int nbg_poll(nbg_server* s, int64_t ticket, int32_t* done) {
    if (!s || !done) return fail(NBG_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return fail(NBG_EINVAL, "unknown ticket");
    *done = it->second.state >= 2;
    return it->second.state == 3 ? it->second.rc : NBG_OK;
}

int nbg_wait(nbg_server* s, int64_t ticket, int64_t timeout_us) {
    if (!s) return fail(NBG_EINVAL, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return fail(NBG_EINVAL, "unknown ticket");
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::microseconds(timeout_us);
    while (s->reqs[ticket].state < 2) {
        if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && s->reqs[ticket].state < 2)
            return fail(NBG_ETIMEOUT, "request %lld not done within %lld us", (long long)ticket, (long long)timeout_us);
    }
    const Request& r = s->reqs[ticket];
    return r.state == 3 ? r.rc : NBG_OK;
}

int nbg_release(nbg_server* s, int64_t ticket) {
    if (!s) return fail(NBG_EINVAL, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return fail(NBG_EINVAL, "unknown ticket");
    if (it->second.state < 2) return fail(NBG_EBUSY, "request still running");
    s->reqs.erase(it);
    return NBG_OK;
}

int nbg_server_stats(nbg_server* s, nbg_server_stats_t* st) {
    if (!s || !st) return fail(NBG_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    std::vector<double> l = s->latencies_us;
    std::sort(l.begin(), l.end());
    auto pct = [&](double p) { return l.empty() ? 0.0 : l[std::min(l.size() - 1, (size_t)(p * (double)l.size()))]; };
    st->completed = s->completed;
    st->failed = s->failed;
    st->pending = (int64_t)s->pending.size();
    st->in_flight_batches = (int32_t)s->flights.size();
    st->p50_ms = pct(0.50) / 1e3;
    st->p99_ms = pct(0.99) / 1e3;
    const double span = s->t_last - s->t_first;
    st->output_limbs_per_s = span > 0 ? s->limbs_done / (span * 1e-6) : 0.0;
    return NBG_OK;
}

int nbg_server_destroy(nbg_server* s) {
    if (!s) return NBG_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop.store(true);
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    for (int i = 0; i < MAX_FLIGHT; i++) {
        cudaStreamDestroy(s->streams[i]);
        if (s->pinned[i]) cudaFreeHost(s->pinned[i]);
    }
    cudaFree(s->dmem);
    delete s;
    return NBG_OK;
}

}  // extern "C"
