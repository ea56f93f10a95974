// noalloc.cu — nbg_mul_dev_noalloc: one product whose whole workspace lives in
// a fixed device array compiled into the library, for callers that cannot
// allocate GPU memory.
//
// Who needs it: code that runs where cudaMalloc is unavailable or forbidden —
// inside a memory pool or arena that owns all device memory, under an
// allocator hook that must not be re-entered, in a process whose memory budget
// is fully committed, or from a foreign runtime (a Julia or other FFI host)
// that manages device memory itself and only lends out input and output
// buffers.  The regular entry points allocate a workspace pool, pinned
// staging and per-length twiddle tables on first use; this one allocates
// nothing: no cudaMalloc, no cudaFree, no pinned host memory and no library
// allocator (torch's included).
//
// Scratch: g_noalloc_scratch, NOALLOC_SCRATCH_BYTES (16 MiB), holds the plan,
// the product descriptor, the twiddle tables, the job lists, both primes'
// transform buffers and the carry aggregates.  Every GPU that loads the
// library keeps these 16 MiB until the process exits.  Products whose layout
// does not fit are rejected with NBG_ENOMEM and a message naming the bytes
// needed: transform lengths above about 3.4e5 points for products (balanced
// operands above about 2^16 limbs) or 5.2e5 points for squares.
//
// The array's name in host code is only a host-side stand-in, never a device
// address: the set-up below asks the runtime for the real address with
// cudaGetSymbolAddress, once per device, with that device current, on the
// first call made on the device.  Make that first call before any stream
// capture begins.  The address and the kernels' settings are kept for the
// life of the process, so the library must not outlive a cudaDeviceReset of
// a device it has used.
//
// Every call waits for its stream once: it copies the operands' top limbs to
// the host to size the transform (fp_ntt_params needs their magnitude bits),
// and a call that builds new twiddle tables waits once more per prime.
//
// All calls share the one array and it keeps the last call's contents: the
// twiddle tables of the last transform length are reused when the next call
// has the same length, and everything else is fully rewritten by each call
// (no buffer relies on starting at zero).  Calls that overlap on the GPU —
// issued on different streams, or from several host threads without ordering
// — race on the array and corrupt each other's results; order them on one
// stream.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/nbgpu.h"
#include "consts.h"
#include "engine.h"
#include "kernels.h"

namespace nbg {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(16) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

constexpr int NOALLOC_MAX_DEVICES = 64;
struct NoallocDevice {
    bool ready = false;
    unsigned char* base = nullptr;  // device address of g_noalloc_scratch on this device
    int64_t tables_N = 0;           // transform length whose tables the array holds
};
static NoallocDevice g_na[NOALLOC_MAX_DEVICES];
static std::mutex g_na_mu;
// host-side power tables for one twiddle build (nhi <= 4096 entries at the largest admitted length)
static double g_na_hilo[4096 + 4096];

// jobs[i] for one launch over the operands of a single product (pass jobs
// cover both primes; nprimes is 1 for them): i = ((f * nops) + op) * ntiles + t
__global__ void k_noalloc_jobs(Job* __restrict__ jobs, int64_t ntiles, int nprimes, int nops, int pass) {
    const int64_t n = ntiles * nprimes * nops;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = i % ntiles;
        const int64_t q = i / ntiles;
        const int op = (int)(q % nops), f = (int)(q / nops);
        jobs[i] = Job{0, f | (op << 1) | (pass << 8), t};
    }
}

namespace {

inline size_t up256(size_t x) { return (x + 255) / 256 * 256; }

#define NA_TRY(x)                                                                           \
    do {                                                                                    \
        cudaError_t e_ = (x);                                                               \
        if (e_ != cudaSuccess) return fail(NBG_ECUDA, "%s: %s", #x, cudaGetErrorString(e_)); \
    } while (0)

int noalloc_setup(int dev, NoallocDevice& D) {
    if (D.ready) return NBG_OK;
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        return fail(NBG_ECUDA, "cudaGetSymbolAddress(g_noalloc_scratch) on device %d: %s", dev, cudaGetErrorString(e));
    NA_TRY(kernels_init((double)P1_U, (double)P2_U));
    D.base = (unsigned char*)p;
    D.tables_N = 0;
    D.ready = true;
    return NBG_OK;
}

int read_top_bits(const uint64_t* x, int64_t n, cudaStream_t st, int64_t* bits) {
    uint64_t top = 0;
    NA_TRY(cudaMemcpyAsync(&top, x + n - 1, sizeof top, cudaMemcpyDeviceToHost, st));
    NA_TRY(cudaStreamSynchronize(st));
    *bits = 64 * (n - 1) + (top ? 64 - __builtin_clzll(top) : 0);
    return NBG_OK;
}

}  // namespace
}  // namespace nbg

using namespace nbg;

extern "C" int nbg_mul_dev_noalloc(uint64_t* r, const uint64_t* a, int64_t m, const uint64_t* b, int64_t n,
                                   void* stream) {
    if (!r || !a) return fail(NBG_EINVAL, "null pointer");
    if (m < 1) return fail(NBG_EINVAL, "operand length %lld < 1", (long long)m);
    const bool sqr = (b == nullptr) || (b == a && n == m);
    if (sqr) n = m;
    if (n < 1) return fail(NBG_EINVAL, "operand length %lld < 1", (long long)n);
    {
        const char* rp = (const char*)r;
        const char* ap = (const char*)a;
        const char* bp = (const char*)b;
        const size_t rb = 8 * (size_t)(m + n);
        if ((rp < ap + 8 * (size_t)m && ap < rp + rb) || (!sqr && rp < bp + 8 * (size_t)n && bp < rp + rb))
            return fail(NBG_EINVAL, "r must not alias a or b");
    }
    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0;
    NA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return fail(NBG_EINVAL, "device %d out of range", dev);
    std::lock_guard<std::mutex> lk(g_na_mu);
    NoallocDevice& D = g_na[dev];
    int rc = noalloc_setup(dev, D);
    if (rc) return rc;

    // admission (fp_ntt_params, src/fpntt.jl:964-977) from the operands' top limbs
    int64_t bits_a = 0, bits_b = 0;
    rc = read_top_bits(a, m, st, &bits_a);
    if (rc) return rc;
    if (sqr) bits_b = bits_a;
    else if ((rc = read_top_bits(b, n, st, &bits_b))) return rc;
    if (bits_a < 1 || bits_b < 1) return fail(NBG_EINVAL, "zero operand");
    int bch = 0;
    int64_t N = 0;
    if ((rc = ntt_params(bits_a, bits_b, &bch, &N))) return rc;
    DPlan d;
    const Tuning tun;  // default pass split
    if ((rc = plan_structure(N, sqr ? 1 : 0, tun, d))) return rc;
    const int S = d.nst, P = d.npass;

    // scratch layout: [plan | product | tables (both primes) | power tables | jobs | xa | xb | agg]
    size_t per = 0;
    for (int s = 0; s < S; s++)
        if (d.st[s].m != 2) per += (size_t)(d.st[s].m - 1) * (size_t)d.st[s].Q;
    const int64_t nhi = (N + 4095) / 4096;
    const int nops = sqr ? 1 : 2;
    int64_t njobs = 0;
    // pass jobs cover one tile of both primes
    for (int p = 0; p < P - 1; p++) njobs += nops * d.pass[p].ntiles + d.pass[p].ntiles;
    njobs += d.pass[P - 1].ntiles;
    const int64_t rn = m + n;
    const int64_t ntl = (rn + UNPACK_TL - 1) / UNPACK_TL;
    njobs += ntl + 1;
    size_t off = 0;
    const size_t o_plan = off;
    off = up256(off + sizeof(DPlan));
    const size_t o_prod = off;
    off = up256(off + sizeof(DProd));
    const size_t o_tab = off;
    off = up256(off + sizeof(double) * 2 * per);
    const size_t o_hilo = off;
    off = up256(off + sizeof(double) * (size_t)(nhi + 4096));
    const size_t o_jobs = off;
    off = up256(off + sizeof(Job) * (size_t)njobs);
    const size_t o_xa = off;
    off = up256(off + sizeof(double) * 2 * (size_t)N);
    const size_t o_xb = off;
    if (P > 1 && !sqr) off = up256(off + sizeof(double) * 2 * (size_t)N);
    const size_t o_agg = off;
    off = up256(off + sizeof(uint32_t) * (size_t)ntl);
    if (off > NOALLOC_SCRATCH_BYTES || nhi > 4096)
        return fail(NBG_ENOMEM,
                    "product needs %zu bytes of scratch (transform length %lld); nbg_mul_dev_noalloc holds %zu",
                    off, (long long)N, NOALLOC_SCRATCH_BYTES);
    unsigned char* base = D.base;

    // twiddle tables: exact minimal-balanced powers, rebuilt only when N changes
    {
        size_t toff = 0;
        for (int f = 0; f < 2; f++) {
            for (int s = 0; s < S; s++) {
                if (d.st[s].m == 2) {
                    d.st[s].tw[f] = nullptr;
                    continue;
                }
                d.st[s].tw[f] = (const double*)(base + o_tab) + toff;
                toff += (size_t)(d.st[s].m - 1) * (size_t)d.st[s].Q;
            }
        }
    }
    if (D.tables_N != N) {
        D.tables_N = 0;
        const uint64_t PR[2] = {P1_U, P2_U};
        static const uint64_t FACS[2][5] = {{2, 3, 5, 7, 23}, {2, 3, 5, 7, 13}};
        typedef unsigned __int128 u128;
        auto mulmod = [](uint64_t x, uint64_t y, uint64_t p) { return (uint64_t)(((u128)x * y) % p); };
        auto powmod = [&](uint64_t x, uint64_t e, uint64_t p) {
            uint64_t acc = 1;
            x %= p;
            while (e) {
                if (e & 1) acc = mulmod(acc, x, p);
                x = mulmod(x, x, p);
                e >>= 1;
            }
            return acc;
        };
        double* dhilo = (double*)(base + o_hilo);
        for (int f = 0; f < 2; f++) {
            const uint64_t p = PR[f];
            const double Pd = (double)p;
            uint64_t g = 0;  // fp_generator (src/fpntt.jl:50-56)
            for (uint64_t c = 3; c <= 63 && !g; c++) {
                bool ok = true;
                for (int i = 0; i < 5; i++)
                    if (powmod(c, (p - 1) / FACS[f][i], p) == 1) ok = false;
                if (ok) g = c;
            }
            const uint64_t w = powmod(g, (p - 1) / (uint64_t)N, p);
            const uint64_t w4096 = powmod(w, 4096, p);
            auto minbal = [&](uint64_t x) { return x > p / 2 ? (double)x - Pd : (double)x; };
            uint64_t x = 1;
            for (int64_t i = 0; i < nhi; i++, x = mulmod(x, w4096, p)) g_na_hilo[i] = minbal(x);
            x = 1;
            for (int i = 0; i < 4096; i++, x = mulmod(x, w, p)) g_na_hilo[nhi + i] = minbal(x);
            NA_TRY(cudaMemcpyAsync(dhilo, g_na_hilo, sizeof(double) * (size_t)(nhi + 4096), cudaMemcpyHostToDevice,
                                   st));
            for (int s = 0; s < S; s++) {
                if (d.st[s].m == 2) continue;
                NA_TRY(launch_twiddle((double*)d.st[s].tw[f], d.st[s].m, d.st[s].Q, N / d.st[s].L, dhilo,
                                      dhilo + nhi, f, st));
            }
            // g_na_hilo is reused for the next prime
            NA_TRY(cudaStreamSynchronize(st));
        }
        D.tables_N = N;
    }

    // product descriptor
    DProd Pd;
    memset(&Pd, 0, sizeof Pd);
    Pd.a = a;
    Pd.b = sqr ? a : b;
    Pd.r = r;
    Pd.m = m;
    Pd.n = n;
    Pd.rn = rn;
    Pd.bch = bch;
    Pd.sqr = sqr ? 1 : 0;
    Pd.nca = (bits_a + bch - 1) / bch;
    Pd.ncb = sqr ? Pd.nca : (bits_b + bch - 1) / bch;
    Pd.nconv = Pd.nca + Pd.ncb - 1;
    Pd.plan = 0;
    Pd.npass = P;
    Pd.xa[0] = (double*)(base + o_xa);
    Pd.xa[1] = Pd.xa[0] + N;
    if (P > 1 && !sqr) {
        Pd.xb[0] = (double*)(base + o_xb);
        Pd.xb[1] = Pd.xb[0] + N;
    }
    Pd.agg = (uint32_t*)(base + o_agg);
    Pd.ntl = ntl;
    const DPlan* dplan = (const DPlan*)(base + o_plan);
    const DProd* dprod = (const DProd*)(base + o_prod);
    NA_TRY(cudaMemcpyAsync(base + o_plan, &d, sizeof d, cudaMemcpyHostToDevice, st));
    NA_TRY(cudaMemcpyAsync(base + o_prod, &Pd, sizeof Pd, cudaMemcpyHostToDevice, st));

    // the launch sequence of one product (same kernels and order as a batch)
    Job* jobs = (Job*)(base + o_jobs);
    int64_t jo = 0;
    auto fill = [&](int64_t ntiles, int nprimes, int nj_ops, int pass) -> cudaError_t {
        int64_t cnt = ntiles * nprimes * nj_ops;
        int64_t blocks = (cnt + 255) / 256;
        if (blocks > 4096) blocks = 4096;
        k_noalloc_jobs<<<(unsigned)blocks, 256, 0, st>>>(jobs + jo, ntiles, nprimes, nj_ops, pass);
        return cudaGetLastError();
    };
    auto run = [&](int kind, int64_t cnt, size_t smem) -> cudaError_t {
        cudaError_t e = launch_jobs(kind, dprod, dplan, job_list(jobs + jo), cnt, smem, 0, st);
        jo += cnt;
        return e;
    };
    for (int p = 0; p < P - 1; p++) {
        const DPass& ps = d.pass[p];
        const size_t tile = sizeof(double) * (size_t)tile_stride_doubles(ps.G * ps.C);
        NA_TRY(fill(ps.ntiles, 1, nops, p));
        NA_TRY(run(JK_FWD, nops * ps.ntiles, 2 * tile));
    }
    {
        const DPass& ps = d.pass[P - 1];
        const size_t tile = sizeof(double) * (size_t)tile_stride_doubles(ps.G * ps.C);
        NA_TRY(fill(ps.ntiles, 1, 1, P - 1));
        NA_TRY(run(JK_PWR, ps.ntiles, 2 * nops * tile));
    }
    for (int p = P - 2; p >= 0; p--) {
        const DPass& ps = d.pass[p];
        const size_t tile = sizeof(double) * (size_t)tile_stride_doubles(ps.G * ps.C);
        NA_TRY(fill(ps.ntiles, 1, 1, p));
        NA_TRY(run(JK_REV, ps.ntiles, 2 * tile));
    }
    NA_TRY(fill(ntl, 1, 1, 0));
    const int64_t jo_unpack = jo;
    NA_TRY(run(JK_UNPACK, ntl, unpack_smem_bytes(bch)));
    if (ntl > 1) {
        NA_TRY(fill(1, 1, 1, 0));
        NA_TRY(run(JK_CARRY, 1, 0));
        // carries through runs of all-ones limbs, over the unpack's tile jobs
        NA_TRY(launch_jobs(JK_CARRYFIX, dprod, dplan, job_list(jobs + jo_unpack), ntl, 0, 0, st));
    }
    return NBG_OK;
}
