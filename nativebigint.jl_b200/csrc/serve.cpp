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
constexpr int NSIDE = 3;                     // side streams per slot: a step's launches run side by side
constexpr int64_t DEFAULT_BATCH_POINTS = int64_t(1) << 23;
constexpr int64_t DEFAULT_MAX_HOLD_US = 2000;

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
    double points = 0;  // transform length (what the request costs the GPU, roughly)
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
    // host requests: results staged in the slot's pinned buffer, copied to
    // the caller's buffer on retirement
    struct HostResult {
        size_t stage_off;
        uint64_t* dst;
        size_t bytes;
    };
    std::vector<HostResult> host_results;
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
    cudaStream_t side[MAX_FLIGHT][NSIDE] = {};
    char* pinned[MAX_FLIGHT] = {};
    size_t pinned_bytes[MAX_FLIGHT] = {};
    bool slot_busy[MAX_FLIGHT] = {};
    std::vector<double> latencies_us;
    int64_t completed = 0, failed = 0, batches = 0, batched_requests = 0;
    double pending_points = 0;
    bool wake = false;  // a submission or a batch completion since the worker last looked
    double limbs_done = 0, t_first = 0, t_last = 0;

    double hold_us() const { return (double)(opts.max_hold_us > 0 ? opts.max_hold_us : DEFAULT_MAX_HOLD_US); }
    void run();
    bool launch_batch(std::unique_lock<std::mutex>& lk);
    void retire(std::unique_lock<std::mutex>& lk);
    void fail_front(int rc);
    static void CUDART_CB on_batch_done(void* self);
};

// Fails the request at the front of the queue (server lock held).
void nbg_server::fail_front(int rc) {
    Request& q = reqs[pending.front()];
    pending_points -= q.points;
    q.state = 3;
    q.rc = rc;
    q.t_done = now_us();
    failed++;
    pending.pop_front();
    cv_done.notify_all();
}

// Forms one batch from the front of the queue, within the free arena, and
// launches it.  Entered and left with the server lock held, but the lock is
// dropped while the batch is built, staged and launched so that submitters
// never wait for that host work.  Only the worker thread pops the queue and
// touches the arena, the slots and the flight list's contents, so the
// requests at the front stay where they are meanwhile.
bool nbg_server::launch_batch(std::unique_lock<std::mutex>& lk) {
    if (pending.empty() || (int)flights.size() >= MAX_FLIGHT) return false;
    const double target = (double)(opts.batch_points > 0 ? opts.batch_points : DEFAULT_BATCH_POINTS);
    // let the next batch grow, unless its oldest request has waited max_hold_us
    if (flights.size() >= 2 && pending_points < target && now_us() - reqs[pending.front()].t_submit < hold_us())
        return false;
    std::vector<int64_t> ids;
    std::vector<ProdIn> in;
    std::vector<char> host;
    const int64_t maxb = opts.max_batch > 0 ? opts.max_batch : 100000;
    for (int64_t id : pending) {
        if ((int64_t)ids.size() >= maxb) break;
        const Request& q = reqs[id];
        ids.push_back(id);
        in.push_back(q.in);
        host.push_back(q.host);
    }
    lk.unlock();
    Engine& E = g_eng;
    Flight f;
    size_t off = 0, host_in = 0, host_out = 0;
    int refuse = 0;
    {
        std::lock_guard<std::recursive_mutex> elk(E.mu);
        // shrink the batch until it fits in the free arena
        for (;;) {
            int rc = build_batch(E, in.data(), (int64_t)in.size(), f.bb);
            if (rc) {  // a request the engine refuses (size): fail it alone
                if (in.size() == 1) {
                    refuse = rc;
                    break;
                }
                in.resize(in.size() / 2);
                continue;
            }
            host_in = host_out = 0;
            for (size_t k = 0; k < in.size(); k++)
                if (host[k]) {  // each operand padded on its own, as laid out below
                    host_in += up256(8 * (size_t)in[k].m) + (in[k].sqr ? 0 : up256(8 * (size_t)in[k].n));
                    host_out += up256(8 * (size_t)(in[k].m + in[k].n));
                }
            f.bytes = up256(f.bb.dev_bytes) + host_in + host_out;
            if (arena.alloc(f.bytes, off)) break;
            if (in.size() == 1) {
                if (f.bytes > arena.size())  // can never fit
                    refuse = fail(NBG_ENOMEM, "request needs %zu bytes, over the server's HBM budget", f.bytes);
                else
                    refuse = -1;  // wait for memory to free up
                break;
            }
            in.resize(in.size() / 2);
        }
    }
    if (refuse) {
        lk.lock();
        if (refuse < 0) return false;
        fail_front(refuse);
        return true;
    }
    ids.resize(in.size());
    f.off = off;
    char* base = dmem + off;
    int slot = 0;
    while (slot_busy[slot]) slot++;  // flights.size() < MAX_FLIGHT: a slot is free
    f.slot = slot;
    f.st = streams[slot];
    // The slot's pinned buffer holds [descriptors and jobs | host operands |
    // host results]; descriptors and operands go over in one copy each.
    const size_t head = f.bb.head_bytes;
    const size_t dev_in = up256(f.bb.dev_bytes), dev_out = dev_in + host_in;
    const size_t need = up256(head) + host_in + host_out;
    if (pinned_bytes[slot] < need) {
        if (pinned[slot]) cudaFreeHost(pinned[slot]);
        pinned[slot] = nullptr;
        pinned_bytes[slot] = 0;
        const size_t want = std::max(need + need / 4, (size_t)(8 << 20));
        if (cudaMallocHost(&pinned[slot], want) != cudaSuccess) {
            cudaGetLastError();
            arena.release(off, f.bytes);
            lk.lock();
            fail_front(fail(NBG_ENOMEM, "pinned staging of %zu bytes unavailable", want));
            return true;
        }
        pinned_bytes[slot] = want;
    }
    char* stage = pinned[slot];
    const size_t st_in = up256(head), st_out = st_in + host_in;
    slot_busy[slot] = true;
    size_t ho = 0, ro = 0;
    for (size_t k = 0; k < in.size(); k++) {
        if (!host[k]) continue;
        const ProdIn& q = in[k];
        DProd& P = f.bb.prods[k];
        const size_t na = 8 * (size_t)q.m;
        memcpy(stage + st_in + ho, q.a, na);
        P.a = (const uint64_t*)(base + dev_in + ho);
        ho += up256(na);
        if (q.sqr) {
            P.b = P.a;
        } else {
            const size_t nb = 8 * (size_t)q.n;
            memcpy(stage + st_in + ho, q.b, nb);
            P.b = (const uint64_t*)(base + dev_in + ho);
            ho += up256(nb);
        }
        P.r = (uint64_t*)(base + dev_out + ro);
        f.host_results.push_back({st_out + ro, q.r, 8 * (size_t)(q.m + q.n)});
        ro += up256(8 * (size_t)(q.m + q.n));
    }
    bool ok = bind_batch(f.bb, base) == NBG_OK;
    stage_batch(f.bb, stage);
    ok = ok && cudaMemcpyAsync(base, stage, head, cudaMemcpyHostToDevice, f.st) == cudaSuccess;
    if (ok && host_in)
        ok = cudaMemcpyAsync(base + dev_in, stage + st_in, host_in, cudaMemcpyHostToDevice, f.st) == cudaSuccess;
    {
        std::lock_guard<std::recursive_mutex> elk(E.mu);
        ok = ok && run_launches_branched(E, f.bb, base, f.st, side[slot], NSIDE) == NBG_OK;
    }
    if (ok && host_out)
        ok = cudaMemcpyAsync(stage + st_out, base + dev_out, host_out, cudaMemcpyDeviceToHost, f.st) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&f.done, cudaEventDisableTiming) == cudaSuccess;
    ok = ok && cudaEventRecord(f.done, f.st) == cudaSuccess;
    ok = ok && cudaLaunchHostFunc(f.st, on_batch_done, this) == cudaSuccess;
    if (!ok) {
        // the stream's work is abandoned: fail the batch's requests
        cudaStreamSynchronize(f.st);
        if (f.done) cudaEventDestroy(f.done);
        arena.release(f.off, f.bytes);
        slot_busy[f.slot] = false;
        lk.lock();
        for (size_t k = 0; k < ids.size(); k++) fail_front(NBG_ECUDA);
        return true;
    }
    lk.lock();
    for (size_t k = 0; k < ids.size(); k++) {
        Request& q = reqs[ids[k]];
        q.state = 1;
        pending_points -= q.points;
        pending.pop_front();
    }
    batches++;
    batched_requests += (int64_t)ids.size();
    f.ids = std::move(ids);
    flights.push_back(std::move(f));
    return true;
}

// Marks finished batches done.  Entered and left with the server lock held; host results are
// copied out to the callers' buffers with the lock dropped.
void nbg_server::retire(std::unique_lock<std::mutex>& lk) {
    std::vector<std::pair<Flight, cudaError_t>> fin;
    for (auto it = flights.begin(); it != flights.end();) {
        cudaError_t q = cudaEventQuery(it->done);
        if (q == cudaErrorNotReady) {
            ++it;
            continue;
        }
        fin.emplace_back(std::move(*it), q);
        it = flights.erase(it);
    }
    if (fin.empty()) return;
    lk.unlock();
    const double t = now_us();
    for (auto& fe : fin) {
        Flight& fl = fe.first;
        if (fe.second == cudaSuccess)
            for (const auto& hr : fl.host_results) memcpy(hr.dst, pinned[fl.slot] + hr.stage_off, hr.bytes);
        cudaEventDestroy(fl.done);
        arena.release(fl.off, fl.bytes);
        slot_busy[fl.slot] = false;
    }
    lk.lock();
    for (auto& fe : fin) {
        for (int64_t id : fe.first.ids) {
            Request& rq = reqs[id];
            const bool ok = fe.second == cudaSuccess;
            rq.state = ok ? 2 : 3;
            rq.rc = ok ? NBG_OK : NBG_ECUDA;
            rq.t_done = t;
            if (ok) {
                completed++;
                latencies_us.push_back(t - rq.t_submit);
                limbs_done += (double)(rq.in.m + rq.in.n);
                t_last = t;
            } else {
                failed++;
            }
        }
    }
    cv_done.notify_all();
}

// Host callback queued behind each batch: wakes the worker to retire it.
// It takes only the server lock and calls no CUDA function.
void CUDART_CB nbg_server::on_batch_done(void* self) {
    nbg_server* s = (nbg_server*)self;
    std::lock_guard<std::mutex> lk(s->mu);
    s->wake = true;
    s->cv_work.notify_all();
}

void nbg_server::run() {
    std::unique_lock<std::mutex> lk(mu);
    while (!stop.load() || !pending.empty() || !flights.empty()) {
        wake = false;
        retire(lk);
        bool launched = false;
        while (launch_batch(lk)) launched = true;
        if (launched || wake) continue;  // wake: something happened while the lock was dropped
        // woken by a submission or a batch's completion callback; the timeout
        // is a backstop, and the moment the oldest held request's hold ends
        double wait_us = flights.empty() ? 5000.0 : 2000.0;
        if (!pending.empty()) {
            const double left = reqs[pending.front()].t_submit + hold_us() - now_us();
            wait_us = std::max(50.0, std::min(wait_us, left));
        }
        cv_work.wait_for(lk, std::chrono::microseconds((int64_t)wait_us));
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
    for (int i = 0; i < MAX_FLIGHT; i++) {
        cudaStreamCreateWithFlags(&s->streams[i], cudaStreamNonBlocking);
        for (int j = 0; j < NSIDE; j++) cudaStreamCreateWithFlags(&s->side[i][j], cudaStreamNonBlocking);
    }
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
    {  // the result must not overlap an operand (src/fpntt.jl:979-981)
        const char* rp = (const char*)d->r;
        const char* ap = (const char*)d->a;
        const char* bp = (const char*)d->b;
        const int64_t n = sqr ? d->m : d->n;
        const size_t rb = 8 * (size_t)(d->m + n);
        if ((rp < ap + 8 * (size_t)d->m && ap < rp + rb) || (!sqr && rp < bp + 8 * (size_t)n && bp < rp + rb))
            return fail(NBG_EINVAL, "r must not alias a or b");
    }
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
    double points = 0;
    {
        int bw = 0;
        int64_t N = 0;
        if (ntt_params(q.bits_a, q.bits_b, &bw, &N) == NBG_OK) points = (double)N;
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
    r.points = points;
    s->pending_points += points;
    s->wake = true;
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
    st->batches = s->batches;
    st->mean_batch_requests = s->batches ? (double)s->batched_requests / (double)s->batches : 0.0;
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
        cudaStreamSynchronize(s->streams[i]);  // its completion callbacks included
        cudaStreamDestroy(s->streams[i]);
        for (int j = 0; j < NSIDE; j++) cudaStreamDestroy(s->side[i][j]);
        if (s->pinned[i]) cudaFreeHost(s->pinned[i]);
    }
    cudaFree(s->dmem);
    delete s;
    return NBG_OK;
}

}  // extern "C"
