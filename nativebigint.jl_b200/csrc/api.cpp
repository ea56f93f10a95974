// api.cpp — the extern "C" entry points of include/nbgpu.h.
#include <cuda_runtime.h>

#include <dlfcn.h>

#include <algorithm>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/nbgpu.h"
#include "engine.h"
#include "kernels.h"

using namespace nbg;

namespace {

#define CUDA_TRY(x)                                                                         \
    do {                                                                                    \
        cudaError_t e_ = (x);                                                               \
        if (e_ != cudaSuccess) return fail(NBG_ECUDA, "%s: %s", #x, cudaGetErrorString(e_)); \
    } while (0)

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

bool overlaps(const void* p, size_t pn, const void* q, size_t qn) {
    const char* a = (const char*)p;
    const char* b = (const char*)q;
    return a < b + qn && b < a + pn;
}

// Validates one descriptor; fills a ProdIn (pointers left as given).
int check_desc(const nbg_desc& d, ProdIn& q, bool host) {
    if (!d.r || !d.a) return fail(NBG_EINVAL, "null pointer");
    if (d.m < 1) return fail(NBG_EINVAL, "operand length %lld < 1", (long long)d.m);
    const bool sqr = (d.b == nullptr) || (d.b == d.a && d.n == d.m);
    if (!sqr && d.n < 1) return fail(NBG_EINVAL, "operand length %lld < 1", (long long)d.n);
    const int64_t n = sqr ? d.m : d.n;
    const size_t rb = sizeof(uint64_t) * (size_t)(d.m + n);
    if (overlaps(d.r, rb, d.a, sizeof(uint64_t) * (size_t)d.m) ||
        (!sqr && overlaps(d.r, rb, d.b, sizeof(uint64_t) * (size_t)n)))
        return fail(NBG_EINVAL, "r must not alias a or b");
    q.a = d.a;
    q.b = sqr ? d.a : d.b;
    q.r = d.r;
    q.m = d.m;
    q.n = n;
    q.sqr = sqr ? 1 : 0;
    q.bits_a = d.bits_a;
    q.bits_b = sqr ? d.bits_a : d.bits_b;
    if (host) {
        q.bits_a = magnitude_bits(d.a, d.m);
        q.bits_b = sqr ? q.bits_a : magnitude_bits(d.b, n);
    }
    return NBG_OK;
}

namespace {

constexpr size_t CHUNK_BYTES = size_t(128) << 20;
constexpr int NBUF = 3;
// chunks with fewer operand and result bytes copy pageable spans directly
constexpr size_t STAGE_MIN_BYTES = size_t(8) << 20;

struct Span {
    const char* h;  // host start
    size_t n;       // bytes
    size_t d;       // offset in the chunk's span area
};

// Merges [p, p + n) ranges into spans; `gap` bytes of slack may be bridged.
// Returns for each range its device offset; spans[] gets the copies.
size_t layout_spans(const std::vector<std::pair<const char*, size_t>>& rg, size_t gap, std::vector<Span>& spans,
                    std::vector<size_t>& dev_off) {
    std::vector<size_t> ord(rg.size());
    for (size_t i = 0; i < ord.size(); i++) ord[i] = i;
    std::sort(ord.begin(), ord.end(), [&](size_t x, size_t y) { return rg[x].first < rg[y].first; });
    dev_off.assign(rg.size(), 0);
    spans.clear();
    size_t total = 0;
    for (size_t k = 0; k < ord.size(); k++) {
        const char* p = rg[ord[k]].first;
        const size_t n = rg[ord[k]].second;
        if (!spans.empty()) {
            Span& sp = spans.back();
            const char* end = sp.h + sp.n;
            if (p >= sp.h && p <= end + gap) {  // extend the span
                const char* ne = std::max(end, p + n);
                total += (size_t)(ne - end);
                sp.n = (size_t)(ne - sp.h);
                dev_off[ord[k]] = sp.d + (size_t)(p - sp.h);
                continue;
            }
        }
        total = align_up(total, 256);
        spans.push_back(Span{p, n, total});
        dev_off[ord[k]] = total;
        total += n;
    }
    return align_up(total, 256);
}

struct Chunk {
    int64_t start, count;
    BatchBuild bb;
    std::vector<Span> in_spans, out_spans;
    size_t in_bytes = 0, out_bytes = 0, region = 0;
    // spans in pageable host memory go through the slot's pinned staging
    // buffers (in: gathered before the copy; out: scattered after it)
    std::vector<char> in_pg, out_pg;
    bool any_out_pg = false;
};

// True when [p, p + n) lies in memory the GPU can copy to or from directly
// (pinned or registered host memory, device or managed memory).
bool dma_ok(const void* p, size_t n) {
    for (const char* q : {(const char*)p, (const char*)p + (n ? n - 1 : 0)}) {
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, q) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        if (a.type == cudaMemoryTypeUnregistered) return false;
    }
    return true;
}

// Host threads for the copies between pageable buffers and pinned staging
// (one thread reaches a fraction of the host's memory bandwidth).  The pieces
// of one run() are split over the workers; run() returns when all are done.
class CopyPool {
public:
    struct Piece {
        char* dst;
        const char* src;
        size_t n;
    };
    static CopyPool& get() {
        static CopyPool pool;
        return pool;
    }
    void run(std::vector<Piece>& pieces) {
        std::vector<Piece> split;
        constexpr size_t PIECE = size_t(4) << 20;
        for (const Piece& p : pieces)
            for (size_t o = 0; o < p.n; o += PIECE) split.push_back({p.dst + o, p.src + o, std::min(PIECE, p.n - o)});
        if (split.empty()) return;
        if (split.size() == 1) {  // small: no hand-off
            std::memcpy(split[0].dst, split[0].src, split[0].n);
            return;
        }
        std::unique_lock<std::mutex> lk(mu_);
        work_ = &split;
        next_ = 0;
        left_ = split.size();
        gen_++;
        cv_.notify_all();
        done_cv_.wait(lk, [&] { return left_ == 0; });
        work_ = nullptr;
    }
    ~CopyPool() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
            gen_++;
        }
        cv_.notify_all();
        for (std::thread& th : threads_) th.join();
    }

private:
    CopyPool() {
        const unsigned hc = std::thread::hardware_concurrency();
        const int n = (int)std::max(2u, std::min(hc ? hc : 4u, 16u));
        for (int i = 0; i < n; i++) threads_.emplace_back([this] { loop(); });
    }
    void loop() {
        uint64_t seen = 0;
        std::unique_lock<std::mutex> lk(mu_);
        for (;;) {
            cv_.wait(lk, [&] { return stop_ || (gen_ != seen && work_ && next_ < work_->size()); });
            if (stop_) return;
            seen = gen_;
            while (work_ && next_ < work_->size()) {
                const Piece p = (*work_)[next_++];
                lk.unlock();
                std::memcpy(p.dst, p.src, p.n);
                lk.lock();
                if (--left_ == 0) done_cv_.notify_all();
            }
        }
    }
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    std::vector<std::thread> threads_;
    std::vector<Piece>* work_ = nullptr;
    size_t next_ = 0, left_ = 0;
    uint64_t gen_ = 0;
    bool stop_ = false;
};

}  // namespace

// Grows a pinned staging buffer to at least `bytes` (its old contents are dropped).
int ensure_pinned(char*& buf, size_t& cap, size_t bytes) {
    if (bytes <= cap) return NBG_OK;
    if (buf) cudaFreeHost(buf);
    buf = nullptr;
    cap = 0;
    const size_t want = std::max(bytes + bytes / 8, (size_t)1 << 20);
    if (cudaMallocHost((void**)&buf, want) != cudaSuccess) {
        cudaGetLastError();
        return fail(NBG_ENOMEM, "pinned staging of %zu bytes unavailable", want);
    }
    cap = want;
    return NBG_OK;
}

// Results of a chunk that land in pinned staging and go on to pageable memory.
struct PendingOut {
    std::vector<Span> spans;
    std::vector<char> pg;
    bool any = false;
};

void scatter_out(PendingOut& po, const char* staged) {
    if (!po.any) return;
    std::vector<CopyPool::Piece> pieces;
    for (size_t i = 0; i < po.spans.size(); i++)
        if (po.pg[i]) pieces.push_back({(char*)po.spans[i].h, staged + po.spans[i].d, po.spans[i].n});
    CopyPool::get().run(pieces);
    po.any = false;
}

int host_batch(const nbg_desc* descs, int64_t count) {
    if (!descs || count <= 0) return fail(NBG_EINVAL, "empty batch");
    Engine& E = g_eng;
    std::vector<ProdIn> in((size_t)count);
    for (int64_t k = 0; k < count; k++) {
        int rc = check_desc(descs[k], in[(size_t)k], true);
        if (rc) return rc;
    }
    {
        int rc = E.ensure();
        if (rc) return rc;
    }
    // chunks of ~CHUNK_BYTES operands, in input order
    std::vector<std::pair<int64_t, int64_t>> bounds;  // (start, count)
    {
        size_t acc = 0;
        int64_t st = 0;
        for (int64_t k = 0; k < count; k++) {
            const ProdIn& q = in[(size_t)k];
            acc += 8 * (size_t)(q.m + (q.sqr ? 0 : q.n));
            if (acc >= CHUNK_BYTES || k == count - 1) {
                bounds.push_back({st, k + 1 - st});
                st = k + 1;
                acc = 0;
            }
        }
    }
    // Each chunk is built on the host while the chunks before it copy and
    // compute; its device region comes from the stream-ordered allocator and
    // goes back after its results are copied out.  At most NBUF chunks are in
    // flight (the host waits for the oldest before starting another).  A
    // chunk's launches of one pipeline step run on parallel streams (a chunk
    // holds a tenth of a large batch, so one step's launches are small and
    // their tails overlap): 10,000 mixed products 45.6 -> 40.9 ms.  The
    // per-slot events are the engine's (host calls are serialized by the API
    // lock).
    static_assert(NBUF <= 4, "the engine keeps 4 event slots");
    cudaEvent_t* ev_in = E.hb_ev[0];
    cudaEvent_t* ev_comp = E.hb_ev[1];
    cudaEvent_t* ev_out = E.hb_ev[2];
    PendingOut pend[NBUF];  // per slot: the last chunk's results staged for pageable memory
    {
        // keep freed chunk regions in the device's memory pool for the next call
        // instead of returning them to the driver at each synchronization
        static int tuned_dev = -1;
        if (tuned_dev != E.dev) {
            cudaMemPool_t mp;
            if (cudaDeviceGetDefaultMemPool(&mp, E.dev) == cudaSuccess) {
                uint64_t thr = UINT64_MAX;
                cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &thr);
            }
            cudaGetLastError();
            tuned_dev = E.dev;
        }
    }
    int rc = NBG_OK;
    for (size_t ci = 0; ci < bounds.size() && rc == NBG_OK; ci++) {
        const int buf = (int)(ci % (size_t)NBUF);
        Chunk c;
        c.start = bounds[ci].first;
        c.count = bounds[ci].second;
        if ((rc = build_batch(E, in.data() + c.start, c.count, c.bb))) break;
        std::vector<std::pair<const char*, size_t>> ir, orr;
        for (int64_t k = 0; k < c.count; k++) {
            const ProdIn& q = in[(size_t)(c.start + k)];
            ir.push_back({(const char*)q.a, 8 * (size_t)q.m});
            if (!q.sqr) ir.push_back({(const char*)q.b, 8 * (size_t)q.n});
            orr.push_back({(const char*)q.r, 8 * (size_t)(q.m + q.n)});
        }
        std::vector<size_t> ioff, ooff;
        c.in_bytes = layout_spans(ir, 0, c.in_spans, ioff);
        c.out_bytes = layout_spans(orr, 0, c.out_spans, ooff);
        // small chunks (single products) leave pageable spans to the driver's
        // own staged copies: checking and staging cost more there (4864-limb
        // product per call 103 us against 126 us)
        bool any_in_pg = false;
        c.in_pg.assign(c.in_spans.size(), 0);
        c.out_pg.assign(c.out_spans.size(), 0);
        if (c.in_bytes + c.out_bytes >= STAGE_MIN_BYTES) {
            for (size_t i = 0; i < c.in_spans.size(); i++)
                if (!dma_ok(c.in_spans[i].h, c.in_spans[i].n)) c.in_pg[i] = 1, any_in_pg = true;
            for (size_t i = 0; i < c.out_spans.size(); i++)
                if (!dma_ok(c.out_spans[i].h, c.out_spans[i].n)) c.out_pg[i] = 1, c.any_out_pg = true;
        }
        const size_t base_in = align_up(c.bb.dev_bytes, 256), base_out = base_in + c.in_bytes;
        c.region = align_up(base_out + c.out_bytes, 256);
        // the slot's previous chunk: its staging buffer and its events are reused
        if (ci >= (size_t)NBUF && cudaEventSynchronize(ev_out[buf]) != cudaSuccess) {
            rc = fail(NBG_ECUDA, "pipeline wait");
            break;
        }
        // that chunk's results staged for pageable memory go out now; this
        // chunk's pageable operands come in (the host threads do both at once)
        {
            std::vector<CopyPool::Piece> pieces;
            if (pend[buf].any)
                for (size_t i = 0; i < pend[buf].spans.size(); i++)
                    if (pend[buf].pg[i])
                        pieces.push_back({(char*)pend[buf].spans[i].h, E.pg_out[buf] + pend[buf].spans[i].d,
                                          pend[buf].spans[i].n});
            pend[buf].any = false;
            if (any_in_pg) {
                if ((rc = ensure_pinned(E.pg_in[buf], E.pg_in_bytes[buf], c.in_bytes))) break;
                for (size_t i = 0; i < c.in_spans.size(); i++)
                    if (c.in_pg[i]) pieces.push_back({E.pg_in[buf] + c.in_spans[i].d, c.in_spans[i].h, c.in_spans[i].n});
            }
            CopyPool::get().run(pieces);
            if (c.any_out_pg && (rc = ensure_pinned(E.pg_out[buf], E.pg_out_bytes[buf], c.out_bytes))) break;
        }
        char* base = nullptr;
        if (cudaMallocAsync((void**)&base, c.region, E.copy_in) != cudaSuccess) {
            cudaGetLastError();
            rc = fail(NBG_ENOMEM, "device region of %zu bytes unavailable", c.region);
            break;
        }
        // everything after the allocation: on an error the region is freed
        // once the streams are idle
        int crc = NBG_OK;
        do {
            size_t ii = 0;
            for (int64_t k = 0; k < c.count; k++) {
                const ProdIn& q = in[(size_t)(c.start + k)];
                DProd& P = c.bb.prods[(size_t)k];
                P.a = (const uint64_t*)(base + base_in + ioff[ii++]);
                P.b = q.sqr ? P.a : (const uint64_t*)(base + base_in + ioff[ii++]);
                P.r = (uint64_t*)(base + base_out + ooff[(size_t)k]);
            }
            // descriptors and job table through the slot's pinned staging buffer
            if ((crc = E.ensure_stage(buf, c.bb.head_bytes))) break;
            if ((crc = bind_batch(c.bb, base))) break;
            stage_batch(c.bb, E.stage[buf]);
            if (cudaMemcpyAsync(base, E.stage[buf], c.bb.head_bytes, cudaMemcpyHostToDevice, E.copy_in) != cudaSuccess) {
                crc = fail(NBG_ECUDA, "descriptor copy failed");
                break;
            }
            for (size_t i = 0; i < c.in_spans.size(); i++) {
                const Span& sp = c.in_spans[i];
                const char* src = c.in_pg[i] ? E.pg_in[buf] + sp.d : sp.h;
                if (cudaMemcpyAsync(base + base_in + sp.d, src, sp.n, cudaMemcpyHostToDevice, E.copy_in) != cudaSuccess) {
                    crc = fail(NBG_ECUDA, "operand copy failed");
                    break;
                }
            }
            if (crc) break;
            cudaEventRecord(ev_in[buf], E.copy_in);
            cudaStreamWaitEvent(E.stream, ev_in[buf], 0);
            if ((crc = run_launches_branched(E, c.bb, base, E.stream, E.side, 4))) break;
            cudaEventRecord(ev_comp[buf], E.stream);
            cudaStreamWaitEvent(E.copy_out, ev_comp[buf], 0);
            for (size_t i = 0; i < c.out_spans.size(); i++) {
                const Span& sp = c.out_spans[i];
                void* dst = c.out_pg[i] ? (void*)(E.pg_out[buf] + sp.d) : (void*)sp.h;
                if (cudaMemcpyAsync(dst, base + base_out + sp.d, sp.n, cudaMemcpyDeviceToHost, E.copy_out) !=
                    cudaSuccess) {
                    crc = fail(NBG_ECUDA, "result copy failed");
                    break;
                }
            }
            if (crc) break;
        } while (0);
        if (crc) {
            cudaStreamSynchronize(E.copy_in);
            cudaStreamSynchronize(E.stream);
            cudaStreamSynchronize(E.copy_out);
            cudaFreeAsync(base, E.copy_out);
            rc = crc;
            break;
        }
        cudaFreeAsync(base, E.copy_out);
        cudaEventRecord(ev_out[buf], E.copy_out);
        pend[buf].spans = std::move(c.out_spans);
        pend[buf].pg = std::move(c.out_pg);
        pend[buf].any = c.any_out_pg;
    }
    cudaError_t e1 = cudaStreamSynchronize(E.copy_in);
    cudaError_t e2 = cudaStreamSynchronize(E.stream);
    cudaError_t e3 = cudaStreamSynchronize(E.copy_out);
    if (rc == NBG_OK && e1 == cudaSuccess && e2 == cudaSuccess && e3 == cudaSuccess)
        for (int i = 0; i < NBUF; i++) scatter_out(pend[i], E.pg_out[i]);
    if (rc) return rc;
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess)
        return fail(NBG_ECUDA, "host batch: %s", cudaGetErrorString(e1 != cudaSuccess ? e1 : e2 != cudaSuccess ? e2 : e3));
    return NBG_OK;
}

// Reads the operands' top limbs on the device (magnitude_bits) for
// descriptors that leave bits_a / bits_b at 0.
int fill_bits_dev(std::vector<ProdIn>& in, cudaStream_t st) {
    std::vector<int64_t> need;
    for (size_t k = 0; k < in.size(); k++)
        if (in[k].bits_a <= 0 || (!in[k].sqr && in[k].bits_b <= 0)) need.push_back((int64_t)k);
    if (need.empty()) return NBG_OK;
    Engine& E = g_eng;
    std::vector<DProd> tmp(need.size());
    for (size_t i = 0; i < need.size(); i++) {
        memset(&tmp[i], 0, sizeof(DProd));
        const ProdIn& q = in[(size_t)need[i]];
        tmp[i].a = q.a;
        tmp[i].b = q.b;
        tmp[i].m = q.m;
        tmp[i].n = q.n;
    }
    const size_t pb = align_up(sizeof(DProd) * tmp.size(), 256);
    const size_t bb = sizeof(int64_t) * 2 * tmp.size();
    int rc = E.ensure_pool(pb + bb);
    if (rc) return rc;
    char* d = (char*)E.pool;
    CUDA_TRY(cudaMemcpyAsync(d, tmp.data(), sizeof(DProd) * tmp.size(), cudaMemcpyHostToDevice, st));
    CUDA_TRY(launch_topbits((const DProd*)d, (int64_t)tmp.size(), (int64_t*)(d + pb), st));
    g_launches++;
    std::vector<int64_t> bits(2 * tmp.size());
    CUDA_TRY(cudaMemcpyAsync(bits.data(), d + pb, bb, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    for (size_t i = 0; i < need.size(); i++) {
        ProdIn& q = in[(size_t)need[i]];
        q.bits_a = bits[2 * i];
        q.bits_b = q.sqr ? q.bits_a : bits[2 * i + 1];
    }
    return NBG_OK;
}

int dev_batch(const nbg_desc* descs, int64_t count, cudaStream_t st) {
    if (!descs || count <= 0) return fail(NBG_EINVAL, "empty batch");
    Engine& E = g_eng;
    std::vector<ProdIn> in((size_t)count);
    for (int64_t k = 0; k < count; k++) {
        int rc = check_desc(descs[k], in[(size_t)k], false);
        if (rc) return rc;
    }
    int rc = E.ensure();
    if (rc) return rc;
    rc = fill_bits_dev(in, st);
    if (rc) return rc;
    BatchBuild bb;
    rc = build_batch(E, in.data(), count, bb);
    if (rc) return rc;
    // the pool is reused by the next call: order it after earlier work on E.stream
    rc = E.ensure_pool(bb.dev_bytes);
    if (rc) return rc;
    char* dbase = (char*)E.pool;
    rc = upload_batch(E, bb, dbase, st);
    if (rc) return rc;
    rc = run_launches(E, bb, dbase, st);
    if (rc) return rc;
    // descriptors/jobs live in pageable host memory copied asynchronously;
    // keep them valid until the copies ran.
    CUDA_TRY(cudaStreamSynchronize(st));
    return NBG_OK;
}

// NULL is the legacy default stream, as everywhere in CUDA
cudaStream_t as_stream(void* s) { return (cudaStream_t)s; }

const char* NBG_VERSION = "0.4.0";

std::string json_str(const std::string& js, const char* key) {
    std::string k = std::string("\"") + key + "\"";
    size_t p = js.find(k);
    if (p == std::string::npos) return "";
    p = js.find(':', p + k.size());
    if (p == std::string::npos) return "";
    p = js.find('"', p);
    if (p == std::string::npos) return "";
    size_t e = js.find('"', p + 1);
    if (e == std::string::npos) return "";
    return js.substr(p + 1, e - p - 1);
}

// Applies a tuning file written by the autotuner if it was made for this GPU
// model and library version; anything else keeps the defaults.
int load_tuning_file(const char* path) {
    FILE* f = fopen(path, "rb");
    if (!f) return fail(NBG_EINVAL, "tuning file %s not readable", path);
    std::string js;
    char buf[4096];
    size_t n;
    while ((n = fread(buf, 1, sizeof buf, f)) > 0) js.append(buf, n);
    fclose(f);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, g_eng.dev) != cudaSuccess) return fail(NBG_ECUDA, "device properties");
    const std::string gpu = json_str(js, "gpu"), ver = json_str(js, "version");
    if (gpu != prop.name || ver != NBG_VERSION)
        return fail(NBG_EINVAL, "stale tuning file %s (gpu '%s', version '%s'; this is '%s', %s)", path, gpu.c_str(),
                    ver.c_str(), prop.name, NBG_VERSION);
    const size_t t = js.find("\"tuning\"");
    if (t == std::string::npos) return fail(NBG_EINVAL, "tuning file %s has no tuning object", path);
    const size_t ob = js.find('{', t);
    if (ob == std::string::npos) return fail(NBG_EINVAL, "tuning file %s malformed", path);
    int rc = g_eng.tun.from_json(js.c_str() + ob);
    if (rc) return rc;
    g_eng.drop_plans();
    return NBG_OK;
}

// NBGPU_TUNING, else <library dir>/../tuning/<gpu name with spaces as _>.json
void autoload_tuning() {
    std::string path;
    if (const char* env = getenv("NBGPU_TUNING")) {
        path = env;
    } else {
        Dl_info info;
        cudaDeviceProp prop;
        if (!dladdr((void*)&autoload_tuning, &info) || !info.dli_fname) return;
        if (cudaGetDeviceProperties(&prop, g_eng.dev) != cudaSuccess) return;
        std::string lib = info.dli_fname;
        size_t sl = lib.rfind('/');
        std::string dir = sl == std::string::npos ? "." : lib.substr(0, sl);
        std::string name = prop.name;
        for (char& ch : name)
            if (ch == ' ') ch = '_';
        path = dir + "/../tuning/" + name + ".json";
    }
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) return;
    fclose(f);
    std::string keep = last_error();
    (void)load_tuning_file(path.c_str());  // a stale or foreign file leaves the defaults
}

// One product descriptor wrapping a preloaded transform or an unpack.
int transform_passes(double* x, int64_t N, int prime, bool fwd, cudaStream_t st) {
    if (!x || prime < 0 || prime > 1) return fail(NBG_EINVAL, "bad argument");
    Engine& E = g_eng;
    PlanRec* pr;
    int rc = E.get_plan(N, 0, &pr);
    if (rc) return rc;
    // the pass kernels transform both primes' tiles together: the other prime
    // works on a scratch copy in the pool that is discarded
    DProd P;
    memset(&P, 0, sizeof P);
    P.plan = pr->slot;
    P.npass = pr->d.npass;
    P.flags = PF_PRELOADED;
    std::vector<Job> jobs;
    std::vector<Launch> ls;
    const int np = pr->d.npass;
    for (int i = 0; i < np; i++) {
        const int p = fwd ? i : np - 1 - i;
        const DPass& ps = pr->d.pass[p];
        Launch L{fwd ? (int)JK_FWD : (int)JK_REV, (int64_t)jobs.size(), ps.ntiles,
                 sizeof(double) * 2 * (size_t)tile_stride_doubles(ps.G * ps.C)};
        for (int64_t t = 0; t < ps.ntiles; t++) jobs.push_back(Job{0, p << 8, t});
        ls.push_back(L);
    }
    const size_t jo = 256;
    const size_t so = align_up(jo + sizeof(Job) * jobs.size(), 256);
    rc = E.ensure_pool(so + sizeof(double) * (size_t)N);
    if (rc) return rc;
    char* d = (char*)E.pool;
    P.xa[prime] = x;
    P.xa[1 - prime] = (double*)(d + so);
    CUDA_TRY(cudaMemcpyAsync(d, &P, sizeof P, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(d + jo, jobs.data(), sizeof(Job) * jobs.size(), cudaMemcpyHostToDevice, st));
    for (const Launch& L : ls) {
        CUDA_TRY(launch_jobs(L.kind, (const DProd*)d, E.d_plans, job_list((const Job*)(d + jo) + L.off), L.n, L.smem, 0, st));
        g_launches++;
    }
    CUDA_TRY(cudaStreamSynchronize(st));
    return NBG_OK;
}

}  // namespace

namespace nbg {
void autoload_tuning_hook() { autoload_tuning(); }
}  // namespace nbg

// ---------------------------------------------------------------------------

#define API_LOCK() std::lock_guard<std::recursive_mutex> lk_(g_eng.mu)
#define API_LOCK_DEV()                                   \
    std::lock_guard<std::recursive_mutex> lk_(g_eng.mu); \
    {                                                    \
        int rc_ = g_eng.ensure();                        \
        if (rc_) return rc_;                             \
    }

extern "C" {

int nbg_init(int32_t device) {
    std::lock_guard<std::recursive_mutex> lk(g_eng.mu);
    const bool was = g_eng.ready;
    int rc = g_eng.init(device);
    if (!rc && !was) autoload_tuning();
    return rc;
}

const char* nbg_version(void) { return NBG_VERSION; }

int nbg_trim_plans(void) {
    std::lock_guard<std::recursive_mutex> lk(g_eng.mu);
    if (g_eng.ready) g_eng.trim_plans();
    return NBG_OK;
}

int nbg_load_tuning(const char* path) {
    if (!path) return fail(NBG_EINVAL, "null path");
    std::lock_guard<std::recursive_mutex> lk(g_eng.mu);
    int rc = g_eng.ensure();
    if (rc) return rc;
    return load_tuning_file(path);
}

const char* nbg_last_error(void) { return last_error(); }

void* nbg_default_stream(void) {
    std::lock_guard<std::recursive_mutex> lk(g_eng.mu);
    if (g_eng.ensure()) return nullptr;
    return (void*)g_eng.stream;
}

int64_t nbg_launch_count(void) { return g_launches.load(); }

int nbg_device_faults(int64_t* count) {
    if (!count) return fail(NBG_EINVAL, "null pointer");
    std::lock_guard<std::recursive_mutex> lk(g_eng.mu);
    unsigned int n = 0;
    cudaError_t e = kernels_take_faults(&n);
    if (e != cudaSuccess) return fail(NBG_ECUDA, "reading the fault count: %s", cudaGetErrorString(e));
    *count = (int64_t)n;
    return NBG_OK;
}

int nbg_kernel_arch(int32_t* version) {
    if (!version) return fail(NBG_EINVAL, "null pointer");
    int v = 0;
    cudaError_t e = kernels_binary_version(&v);
    if (e != cudaSuccess) return fail(NBG_ECUDA, "cudaFuncGetAttributes: %s", cudaGetErrorString(e));
    *version = v;
    return NBG_OK;
}

int nbg_mul(uint64_t* r, const uint64_t* a, int64_t m, const uint64_t* b, int64_t n) {
    if (!b) return fail(NBG_EINVAL, "null pointer");
    API_LOCK();
    nbg_desc d{r, a, b, m, n, 0, 0};
    return host_batch(&d, 1);
}

int nbg_sqr(uint64_t* r, const uint64_t* a, int64_t n) {
    API_LOCK();
    nbg_desc d{r, a, nullptr, n, n, 0, 0};
    return host_batch(&d, 1);
}

// Low halves: operand limbs at or above k cannot reach the low k limbs, so
// the operands are cut to k limbs, the full product runs on the GPU, and its
// low k limbs are kept (the reference's full-product branches of mullo! and
// sqrlo!, src/mul.jl:316-319 and :361-364, at every size).
static int low_product(uint64_t* r, const uint64_t* a, int64_t la, const uint64_t* b, int64_t lb, int64_t k) {
    if (!r || !a || la < 1 || k < 1 || (b && lb < 1)) return fail(NBG_EINVAL, "bad argument");
    la = std::min(la, k);
    lb = b ? std::min(lb, k) : la;
    std::vector<uint64_t> full((size_t)(la + lb));
    nbg_desc d{full.data(), a, b, la, lb, 0, 0};
    int rc = host_batch(&d, 1);
    if (rc) return rc;
    const int64_t keep = std::min(k, la + lb);
    memcpy(r, full.data(), sizeof(uint64_t) * (size_t)keep);
    if (keep < k) memset(r + keep, 0, sizeof(uint64_t) * (size_t)(k - keep));
    return NBG_OK;
}

int nbg_mullo(uint64_t* r, const uint64_t* a, int64_t la, const uint64_t* b, int64_t lb, int64_t k) {
    if (!b) return fail(NBG_EINVAL, "null pointer");
    API_LOCK();
    return low_product(r, a, la, b, lb, k);
}

int nbg_sqrlo(uint64_t* r, const uint64_t* a, int64_t la, int64_t k) {
    API_LOCK();
    return low_product(r, a, la, nullptr, 0, k);
}

int nbg_mul_dev(uint64_t* r, const uint64_t* a, int64_t m, const uint64_t* b, int64_t n, void* stream) {
    if (!b) return fail(NBG_EINVAL, "null pointer");
    API_LOCK();
    nbg_desc d{r, a, b, m, n, 0, 0};
    return dev_batch(&d, 1, as_stream(stream));
}

int nbg_sqr_dev(uint64_t* r, const uint64_t* a, int64_t n, void* stream) {
    API_LOCK();
    nbg_desc d{r, a, nullptr, n, n, 0, 0};
    return dev_batch(&d, 1, as_stream(stream));
}

int nbg_mul_batch(const nbg_desc* descs, int64_t count) {
    API_LOCK();
    return host_batch(descs, count);
}

int nbg_mul_batch_dev(const nbg_desc* descs, int64_t count, void* stream) {
    API_LOCK();
    return dev_batch(descs, count, as_stream(stream));
}

// ---- reusable batches (CUDA graph) ----------------------------------------

struct nbg_batch {
    BatchBuild bb;
    char* dmem = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    QueueRun q;  // tuning "queue" > 0: the graph is one persistent work-queue launch
};

int nbg_batch_create(const nbg_desc* descs, int64_t count, nbg_batch** out) {
    if (!out) return fail(NBG_EINVAL, "null out");
    API_LOCK();
    *out = nullptr;
    if (!descs || count <= 0) return fail(NBG_EINVAL, "empty batch");
    Engine& E = g_eng;
    std::vector<ProdIn> in((size_t)count);
    for (int64_t k = 0; k < count; k++) {
        int rc = check_desc(descs[k], in[(size_t)k], false);
        if (rc) return rc;
    }
    int rc = E.ensure();
    if (rc) return rc;
    rc = fill_bits_dev(in, E.stream);
    if (rc) return rc;
    nbg_batch* bt = new nbg_batch();
    rc = build_batch(E, in.data(), count, bt->bb);
    if (rc) {
        delete bt;
        return rc;
    }
    if (cudaMalloc(&bt->dmem, bt->bb.dev_bytes) != cudaSuccess) {
        cudaGetLastError();
        const size_t want = bt->bb.dev_bytes;
        delete bt;
        return fail(NBG_ENOMEM, "batch workspace of %zu bytes unavailable", want);
    }
    rc = upload_batch(E, bt->bb, bt->dmem, E.stream);
    const bool queue = E.tun.queue > 0;
    if (!rc && queue) rc = queue_prepare(E, bt->bb, bt->dmem, bt->q, E.stream);
    if (!rc && cudaStreamSynchronize(E.stream) != cudaSuccess) rc = fail(NBG_ECUDA, "batch upload failed");
    if (!rc) {
        cudaStream_t cs;
        if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) {
            rc = fail(NBG_ECUDA, "stream create failed");
        } else {
            constexpr int NSIDE = 4;
            cudaStream_t side[NSIDE];
            for (int i = 0; i < NSIDE; i++) cudaStreamCreateWithFlags(&side[i], cudaStreamNonBlocking);
            if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
                rc = fail(NBG_ECUDA, "begin capture failed");
            } else {
                int64_t before = g_launches.load();
                // a step's launches (one per shared-memory size) become parallel
                // graph branches, or the whole batch is one work-queue launch
                int rl = queue ? queue_run(E, bt->bb, bt->dmem, bt->q, cs)
                               : run_launches_branched(E, bt->bb, bt->dmem, cs, side, NSIDE);
                g_launches.store(before);  // captured, not issued
                cudaError_t ec = cudaStreamEndCapture(cs, &bt->graph);
                if (rl) rc = rl;
                else if (ec != cudaSuccess) rc = fail(NBG_ECUDA, "end capture: %s", cudaGetErrorString(ec));
                else if (cudaGraphInstantiate(&bt->exec, bt->graph, 0) != cudaSuccess)
                    rc = fail(NBG_ECUDA, "graph instantiate failed");
            }
            for (int i = 0; i < NSIDE; i++) cudaStreamDestroy(side[i]);
            cudaStreamDestroy(cs);
        }
    }
    if (rc) {
        if (bt->exec) cudaGraphExecDestroy(bt->exec);
        if (bt->graph) cudaGraphDestroy(bt->graph);
        cudaFree(bt->dmem);
        queue_free(bt->q);
        delete bt;
        return rc;
    }
    *out = bt;
    return NBG_OK;
}

int nbg_batch_run(nbg_batch* bt, void* stream) {
    if (!bt) return fail(NBG_EINVAL, "null batch");
    API_LOCK_DEV();
    CUDA_TRY(cudaGraphLaunch(bt->exec, as_stream(stream)));
    g_launches += bt->q.d ? 2 : (int64_t)bt->bb.launches.size();
    return NBG_OK;
}

int nbg_batch_launches(const nbg_batch* bt) { return bt ? (int)bt->bb.launches.size() : 0; }

int nbg_batch_stats(const nbg_batch* bt, int32_t* kinds, int64_t* njobs, double* alg_ops, double* alg_bytes,
                    int32_t cap) {
    if (!bt || cap < 0) return fail(NBG_EINVAL, "bad argument");
    const auto& ls = bt->bb.launches;
    for (size_t i = 0; i < ls.size() && (int32_t)i < cap; i++) {
        if (kinds) kinds[i] = ls[i].kind;
        if (njobs) njobs[i] = ls[i].n;
        if (alg_ops) alg_ops[i] = ls[i].alg_ops;
        if (alg_bytes) alg_bytes[i] = ls[i].alg_bytes;
    }
    return NBG_OK;
}

int nbg_batch_profile(nbg_batch* bt, void* stream, float* ms, int32_t cap) {
    if (!bt || !ms) return fail(NBG_EINVAL, "bad argument");
    API_LOCK_DEV();
    cudaStream_t st = as_stream(stream);
    const auto& ls = bt->bb.launches;
    std::vector<cudaEvent_t> ev(ls.size() + 1);
    for (auto& e : ev) CUDA_TRY(cudaEventCreate(&e));
    const DProd* prods = (const DProd*)(bt->dmem + bt->bb.off_prods);
    const Job* jobs = (const Job*)(bt->dmem + bt->bb.off_joblist);
    CUDA_TRY(expand_jobs(bt->bb, bt->dmem, st));
    int rc = NBG_OK;
    CUDA_TRY(cudaEventRecord(ev[0], st));
    for (size_t i = 0; i < ls.size(); i++) {
        const Launch& L = ls[i];
        cudaError_t e = launch_jobs(L.kind, prods, g_eng.d_plans, job_list(jobs + L.off), L.n, L.smem, 0, st, L.odd);
        if (e != cudaSuccess) { rc = fail(NBG_ECUDA, "profile launch: %s", cudaGetErrorString(e)); break; }
        g_launches++;
        CUDA_TRY(cudaEventRecord(ev[i + 1], st));
    }
    if (!rc && cudaEventSynchronize(ev[ls.size()]) != cudaSuccess) rc = fail(NBG_ECUDA, "profile sync failed");
    for (size_t i = 0; !rc && i < ls.size() && (int32_t)i < cap; i++) cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]);
    for (auto& e : ev) cudaEventDestroy(e);
    return rc;
}

int nbg_batch_destroy(nbg_batch* bt) {
    if (!bt) return NBG_OK;
    std::lock_guard<std::recursive_mutex> lk(g_eng.mu);
    if (bt->exec) cudaGraphExecDestroy(bt->exec);
    if (bt->graph) cudaGraphDestroy(bt->graph);
    if (bt->dmem) cudaFree(bt->dmem);
    queue_free(bt->q);
    delete bt;
    return NBG_OK;
}

// ---- admission -------------------------------------------------------------

int nbg_ntt_params(int64_t bits_a, int64_t bits_b, int32_t* b, int64_t* N) {
    if (!b || !N || bits_a < 1 || bits_b < 1) return fail(NBG_EINVAL, "bad argument");
    int bb;
    int rc = ntt_params(bits_a, bits_b, &bb, N);
    if (rc) return rc;
    *b = bb;
    return NBG_OK;
}

int nbg_ntt_len(int64_t T, int64_t* N) {
    if (!N || T < 1) return fail(NBG_EINVAL, "bad argument");
    int64_t v = ntt_len(T);
    if (v < 0) return fail(NBG_ERANGE, "fp NTT length %lld exceeds the 315*2^34 the primes support", (long long)T);
    *N = v;
    return NBG_OK;
}

int64_t nbg_magnitude_bits(const uint64_t* a, int64_t n) {
    if (!a || n < 1) return -1;
    return magnitude_bits(a, n);
}

// ---- transform level --------------------------------------------------------

int nbg_pack_dev(double* x, int64_t N, const uint64_t* limbs, int64_t n, int32_t b, int64_t nch, void* stream) {
    if (!x || !limbs || n < 1 || b < 1 || b > 52 || nch < 0 || nch > N) return fail(NBG_EINVAL, "bad argument");
    if ((nch - 1) * (int64_t)b >= 64 * n) return fail(NBG_EINVAL, "nch exceeds the operand");
    API_LOCK_DEV();
    CUDA_TRY(launch_pack(x, N, limbs, n, b, nch, as_stream(stream)));
    g_launches++;
    return NBG_OK;
}

int nbg_ntt_fwd_dev(double* x, int64_t N, int32_t prime, void* stream) {
    API_LOCK_DEV();
    return transform_passes(x, N, prime, true, as_stream(stream));
}

int nbg_ntt_rev_dev(double* x, int64_t N, int32_t prime, void* stream) {
    API_LOCK_DEV();
    return transform_passes(x, N, prime, false, as_stream(stream));
}

int nbg_pointwise_dev(double* xa, const double* xb, int64_t N, int32_t prime, void* stream) {
    if (!xa || !xb || N < 1 || prime < 0 || prime > 1) return fail(NBG_EINVAL, "bad argument");
    API_LOCK_DEV();
    CUDA_TRY(launch_pointwise(xa, xb, N, prime, as_stream(stream)));
    g_launches++;
    return NBG_OK;
}

int nbg_unpack_dev(uint64_t* r, int64_t rn, const double* x1, const double* x2, int64_t N, int64_t nconv, int32_t b,
                   void* stream) {
    if (!r || !x1 || !x2 || rn < 1 || nconv < 1 || nconv > N || b < 1 || b > 52) return fail(NBG_EINVAL, "bad argument");
    API_LOCK_DEV();
    Engine& E = g_eng;
    cudaStream_t st = as_stream(stream);
    PlanRec* pr;
    int rc = E.get_plan(N, 0, &pr);
    if (rc) return rc;
    DProd P;
    memset(&P, 0, sizeof P);
    P.plan = pr->slot;
    P.r = r;
    P.rn = rn;
    P.nconv = nconv;
    P.bch = b;
    P.xa[0] = (double*)x1;
    P.xa[1] = (double*)x2;
    P.ntl = (rn + UNPACK_TL - 1) / UNPACK_TL;
    std::vector<Job> jobs;
    for (int64_t t = 0; t < P.ntl; t++) jobs.push_back(Job{0, 0, t});
    jobs.push_back(Job{0, 0, 0});
    const size_t jo = 256, ao = align_up(jo + sizeof(Job) * jobs.size(), 256);
    rc = E.ensure_pool(ao + sizeof(uint32_t) * (size_t)P.ntl);
    if (rc) return rc;
    char* d = (char*)E.pool;
    P.agg = (uint32_t*)(d + ao);
    CUDA_TRY(cudaMemcpyAsync(d, &P, sizeof P, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(d + jo, jobs.data(), sizeof(Job) * jobs.size(), cudaMemcpyHostToDevice, st));
    CUDA_TRY(launch_jobs(JK_UNPACK, (const DProd*)d, E.d_plans, job_list((const Job*)(d + jo)), P.ntl,
                         unpack_smem_bytes(b), 0, st));
    CUDA_TRY(launch_jobs(JK_CARRY, (const DProd*)d, E.d_plans, job_list((const Job*)(d + jo) + P.ntl), 1, 0, 0, st));
    CUDA_TRY(launch_jobs(JK_CARRYFIX, (const DProd*)d, E.d_plans, job_list((const Job*)(d + jo)), P.ntl, 0, 0, st));
    g_launches += 3;
    CUDA_TRY(cudaStreamSynchronize(st));
    return NBG_OK;
}

// ---- plans / tuning ---------------------------------------------------------

int nbg_plan_info(int64_t N, int32_t* nst, int32_t* npass, int32_t* stage_m, int32_t* pass_end, int32_t cap) {
    if (!nst || !npass) return fail(NBG_EINVAL, "bad argument");
    API_LOCK_DEV();
    PlanRec* pr;
    int rc = g_eng.get_plan(N, 0, &pr);
    if (rc) return rc;
    *nst = pr->d.nst;
    *npass = pr->d.npass;
    for (int i = 0; stage_m && i < pr->d.nst && i < cap; i++) stage_m[i] = pr->d.st[i].m;
    for (int i = 0; pass_end && i < pr->d.npass && i < cap; i++) pass_end[i] = pr->d.pass[i].sb;
    return NBG_OK;
}

int nbg_plan_layout(int64_t N, int32_t sqr, int64_t* stages, int32_t* nst, int64_t* passes, int32_t* npass,
                    int32_t* rounds, int32_t cap) {
    if (!stages || !nst || !passes || !npass || cap < 1) return fail(NBG_EINVAL, "bad argument");
    API_LOCK();
    DPlan d;
    int rc = plan_structure(N, sqr, g_eng.tun, d);
    if (rc) return rc;
    if (d.nst > cap || d.npass > cap) return fail(NBG_EINVAL, "cap too small");
    for (int i = 0; i < d.nst; i++) {
        stages[3 * i] = d.st[i].m;
        stages[3 * i + 1] = d.st[i].L;
        stages[3 * i + 2] = d.st[i].Q;
    }
    for (int j = 0; j < d.npass; j++) {
        const DPass& p = d.pass[j];
        int64_t* o = passes + 7 * j;
        o[0] = p.sa; o[1] = p.sb; o[2] = p.G; o[3] = p.C; o[4] = p.Qb; o[5] = p.ntiles; o[6] = p.nrounds;
        if (rounds)
            for (int r = 0; r < p.nrounds && r < cap; r++) rounds[j * cap + r] = (p.rkind[r] << 8) | p.rstage[r];
    }
    *nst = d.nst;
    *npass = d.npass;
    return NBG_OK;
}

int nbg_set_tuning(const char* json) {
    if (!json) return fail(NBG_EINVAL, "null json");
    std::lock_guard<std::recursive_mutex> lk(g_eng.mu);
    int rc = g_eng.tun.from_json(json);
    if (rc) return rc;
    g_eng.drop_plans();
    return NBG_OK;
}

int nbg_get_tuning(char* buf, int64_t cap) {
    if (!buf || cap < 2) return fail(NBG_EINVAL, "bad argument");
    std::lock_guard<std::recursive_mutex> lk(g_eng.mu);
    std::string s = g_eng.tun.to_json();
    if ((int64_t)s.size() + 1 > cap) return fail(NBG_EINVAL, "buffer too small");
    memcpy(buf, s.c_str(), s.size() + 1);
    return NBG_OK;
}

}  // extern "C"
