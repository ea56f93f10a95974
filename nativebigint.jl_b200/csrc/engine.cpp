// engine.cpp — host side of libnbgpu.so: admission, plans, batch work queues
// and the C ABI declared in include/nbgpu.h.
//
// Host restatements (all exact, same results as the reference):
//   magnitude_bits      src/kernels/addsub.jl:150
//   ntt_len             src/fpntt.jl:927-951
//   fp_ntt_params       src/fpntt.jl:953-977
//   plan / constants    src/fpntt.jl:50-79 (primes, generator), :123-168
//                       (Winograd constants), :191-271 (stage list)
// This file is compiled with -ffp-contract=off so the double arithmetic that
// builds the combine constants matches the reference's bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include <cudaTypedefs.h>

#include "../../include/nbgpu.h"
#include "engine.h"
#include "consts.h"
#include "kernels.h"

namespace nbg {

// ---------------------------------------------------------------------------
// errors

static thread_local std::string t_err;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    t_err = buf;
    return code;
}
const char* last_error() { return t_err.c_str(); }

#define CUDA_TRY(x)                                                                         \
    do {                                                                                    \
        cudaError_t e_ = (x);                                                               \
        if (e_ != cudaSuccess) return fail(NBG_ECUDA, "%s: %s", #x, cudaGetErrorString(e_)); \
    } while (0)

std::atomic<int64_t> g_launches{0};

// ---------------------------------------------------------------------------
// exact host arithmetic

typedef unsigned __int128 u128;
static inline uint64_t mulmod_u(uint64_t a, uint64_t b, uint64_t p) { return (uint64_t)(((u128)a * b) % p); }
static uint64_t powmod_u(uint64_t a, uint64_t e, uint64_t p) {
    uint64_t r = 1 % p;
    a %= p;
    while (e) {
        if (e & 1) r = mulmod_u(r, a, p);
        a = mulmod_u(a, a, p);
        e >>= 1;
    }
    return r;
}
static uint64_t invmod_u(uint64_t a, uint64_t p) { return powmod_u(a, p - 2, p); }

static const uint64_t PR[2] = {P1_U, P2_U};
static const int TWOADIC[2] = {34, 38};
static const uint64_t FACS[2][5] = {{2, 3, 5, 7, 23}, {2, 3, 5, 7, 13}};

// fp_generator (fpntt.jl:50-56)
static uint64_t generator(int f) {
    static uint64_t g[2] = {0, 0};
    if (!g[f]) {
        uint64_t p = PR[f];
        for (uint64_t c = 3; c <= 63; c++) {
            bool ok = true;
            for (int i = 0; i < 5; i++)
                if (powmod_u(c, (p - 1) / FACS[f][i], p) == 1) ok = false;
            if (ok) { g[f] = c; break; }
        }
    }
    return g[f];
}

// host field ops (fpntt.jl:81-121)
static inline double h_round(double v) { return (v + FP_MAGIC) - FP_MAGIC; }
static inline double h_reduce(double x, double P) {
    double q = h_round(x * (1.0 / P));
    return std::fma(q, -P, x);
}
static inline double h_mulmod(double x, double y, double P) {
    double h = x * y;
    double l = std::fma(x, y, -h);
    return h_reduce(h, P) + l;
}
static inline double h_minbal(double x, double P) { return x > P / 2 ? x - P : (x < -P / 2 ? x + P : x); }

// fp_dft5_consts (fpntt.jl:127-136)
static void dft5_consts(uint64_t c, double P, uint64_t p, double* out) {
    double inv2 = (double)invmod_u(2, p);
    double c1 = h_reduce((double)c, P);
    double c2 = h_mulmod(c1, c1, P), c3 = h_mulmod(c2, c1, P), c4 = h_mulmod(c3, c1, P);
    double inv4 = h_mulmod(inv2, inv2, P);
    out[0] = h_minbal(-inv4, P);
    out[1] = h_minbal(h_mulmod((c1 + c4) - (c2 + c3), inv4, P), P);
    out[2] = h_minbal(h_mulmod(c1 - c4, inv2, P), P);
    out[3] = h_minbal(h_mulmod(c2 - c3, inv2, P), P);
}

// fp_dft7_consts (fpntt.jl:151-168)
static void dft7_consts(uint64_t c, double P, uint64_t p, double* out) {
    double inv2 = (double)invmod_u(2, p), inv3 = (double)invmod_u(3, p);
    double cj[7];
    for (int j = 1; j <= 6; j++) cj[j] = (double)powmod_u(c, (uint64_t)j, p);
    auto A = [&](int j) { return h_mulmod(cj[j] + cj[7 - j], inv2, P); };
    auto B = [&](int j) { return h_mulmod(cj[j] - cj[7 - j], inv2, P); };
    double a0 = A(1), a1 = A(3), a2 = A(2);
    double b0 = B(1), b1 = B(3), b2 = B(2);
    double bp0 = h_minbal(h_mulmod(a0 - a2, inv3, P), P);
    double bp1 = h_minbal(h_mulmod(a1 - a2, inv3, P), P);
    double n0 = h_minbal(h_mulmod(b0 - b2, inv3, P), P);
    double n1 = h_minbal(h_mulmod(b1 + b2, inv3, P), P);
    out[0] = h_minbal(h_mulmod((a0 + a1) + a2, inv3, P), P);
    out[1] = bp0;
    out[2] = bp1;
    out[3] = h_minbal(bp0 + bp1, P);
    out[4] = h_minbal(h_mulmod((b0 + b2) - b1, inv3, P), P);
    out[5] = n0;
    out[6] = n1;
    out[7] = h_minbal(n0 + n1, P);
}

// ---------------------------------------------------------------------------
// admission

static inline int tsb64(uint64_t x) { return x ? 64 - __builtin_clzll(x) : 0; }
static inline int tsb128(u128 x) {
    uint64_t hi = (uint64_t)(x >> 64);
    return hi ? 64 + tsb64(hi) : tsb64((uint64_t)x);
}

int64_t magnitude_bits(const uint64_t* a, int64_t n) { return 64 * (n - 1) + tsb64(a[n - 1]); }

int64_t ntt_len(int64_t T) {
    static const int64_t SMALL[] = {1, 3, 5, 9}, MID[] = {1, 3, 5, 7, 9, 15, 21, 105},
                         LARGE[] = {1, 3, 5, 7, 9, 15, 21, 35, 45, 63, 105, 315};
    const int maxk = std::min(TWOADIC[0], TWOADIC[1]);
    const int64_t* ms;
    int nm;
    if (T <= (int64_t(1) << 14)) { ms = SMALL; nm = 4; }
    else if (T <= (int64_t(1) << 20)) { ms = MID; nm = 8; }
    else { ms = LARGE; nm = 12; }
    int64_t best = INT64_MAX;
    for (int i = 0; i < nm; i++) {
        int64_t m = ms[i];
        int64_t cl = (T + m - 1) / m;
        int k = std::max(tsb64((uint64_t)(cl - 1)), 2);
        if (k > maxk) continue;
        best = std::min(best, m << k);
    }
    return best == INT64_MAX ? -1 : best;
}

int ntt_params(int64_t bits_a, int64_t bits_b, int* b_out, int64_t* N_out) {
    const u128 pp = (u128)PR[0] * PR[1] - 1;
    const int maxb = tsb64(std::min(PR[0], PR[1])) - 1;
    const int64_t mn = std::min(bits_a, bits_b);
    const int nclow = tsb64((uint64_t)((mn + maxb - 1) / maxb));
    const int bstart = std::min(maxb, (tsb128(pp) - nclow + 3) >> 1);
    for (int b = bstart; b >= 1; b--) {
        int64_t nca = (bits_a + b - 1) / b, ncb = (bits_b + b - 1) / b;
        u128 w = (u128)((1ULL << b) - 1);
        if ((u128)std::min(nca, ncb) <= pp / (w * w)) {
            int64_t N = ntt_len(nca + ncb - 1);
            if (N < 0) return fail(NBG_ERANGE, "fp NTT length %lld exceeds the 315*2^34 the primes support",
                                   (long long)(nca + ncb - 1));
            *b_out = b;
            *N_out = N;
            return NBG_OK;
        }
    }
    return fail(NBG_ERANGE, "no admissible chunk width");
}

// ---------------------------------------------------------------------------
// tuning

static int64_t pow2floor(int64_t x) {
    int64_t r = 1;
    while (r * 2 <= x) r *= 2;
    return r;
}

std::string Tuning::to_json() const {
    char buf[512];
    snprintf(buf, sizeof buf,
             "{\"full_max_mul\": %d, \"full_max_sqr\": %d, \"last_max\": %d, \"last_max_sqr\": %d, "
             "\"early_gmax\": %d, \"tile_target\": %d, \"cmax\": %d, \"tma\": %d, \"queue\": %d, "
             "\"overrides\": [",
             full_max_mul, full_max_sqr, last_max, last_max_sqr, early_gmax, tile_target, cmax, tma, queue);
    std::string out = buf;
    bool first = true;
    for (const auto& kv : overrides) {
        out += first ? "" : ", ";
        first = false;
        snprintf(buf, sizeof buf, "{\"N\": %lld, \"sqr\": %d, \"tile_target\": %d, \"cmax\": %d, \"pass_ends\": [",
                 (long long)(kv.first / 2), (int)(kv.first & 1), kv.second.tile_target, kv.second.cmax);
        out += buf;
        for (size_t i = 0; i < kv.second.pass_ends.size(); i++) {
            out += (i ? ", " : "") + std::to_string(kv.second.pass_ends[i]);
        }
        out += "]}";
    }
    out += "]}";
    return out;
}

// Minimal reader for the flat JSON objects this library writes: "key": int.
static bool json_int(const char* js, const char* end, const char* key, long long* out) {
    std::string k = std::string("\"") + key + "\"";
    const char* p = js;
    for (;;) {
        p = strstr(p, k.c_str());
        if (!p || p >= end) return false;
        const char* q = p + k.size();
        while (q < end && (*q == ' ' || *q == '\t' || *q == '\n')) q++;
        if (q < end && *q == ':') {
            char* e = nullptr;
            long long v = strtoll(q + 1, &e, 10);
            if (e == q + 1) return false;
            *out = v;
            return true;
        }
        p = q;
    }
}
static bool json_int(const char* js, const char* key, int* out) {
    long long v;
    if (!json_int(js, js + strlen(js), key, &v)) return false;
    *out = (int)v;
    return true;
}

// matching bracket/brace end of the value starting at p (p points at '[' or '{')
static const char* json_close(const char* p) {
    const char open = *p, close = open == '[' ? ']' : '}';
    int depth = 0;
    for (; *p; p++) {
        if (*p == open) depth++;
        else if (*p == close && --depth == 0) return p;
    }
    return nullptr;
}

int Tuning::from_json(const char* js) {
    Tuning t = *this;
    // top-level scalars: read only the part before "overrides"
    std::string head = js;
    const char* ov = strstr(js, "\"overrides\"");
    if (ov) head = std::string(js, ov);
    json_int(head.c_str(), "full_max_mul", &t.full_max_mul);
    json_int(head.c_str(), "full_max_sqr", &t.full_max_sqr);
    json_int(head.c_str(), "last_max", &t.last_max);
    json_int(head.c_str(), "last_max_sqr", &t.last_max_sqr);
    json_int(head.c_str(), "early_gmax", &t.early_gmax);
    json_int(head.c_str(), "tile_target", &t.tile_target);
    json_int(head.c_str(), "cmax", &t.cmax);
    json_int(head.c_str(), "tma", &t.tma);
    json_int(head.c_str(), "queue", &t.queue);
    auto pow2 = [](int v) { return v >= 1 && (v & (v - 1)) == 0; };
    // shared memory bounds: a product's last pass holds 4 tiles (a, b per
    // prime), a square's 2; column passes hold 2 tiles of <= tile_target or G.
    if (!pow2(t.cmax) || t.last_max < 4 || t.last_max_sqr < 4 || t.early_gmax < 2 || t.tile_target < 1 ||
        t.full_max_mul < 4 || t.full_max_sqr < 4 || t.full_max_mul > 4096 || t.full_max_sqr > 8192 ||
        t.last_max > 4096 || t.last_max_sqr > 8192 || t.early_gmax > 1024 || t.tile_target > 8192 ||
        (t.tma != 0 && t.tma != 1) || t.queue < 0 || t.queue > 64)
        return fail(NBG_EINVAL, "tuning out of range");
    if (ov) {
        t.overrides.clear();
        const char* lb = strchr(ov, '[');
        const char* le = lb ? json_close(lb) : nullptr;
        if (!lb || !le) return fail(NBG_EINVAL, "tuning: malformed overrides");
        const char* p = lb + 1;
        while (p < le) {
            const char* ob = strchr(p, '{');
            if (!ob || ob > le) break;
            const char* oe = json_close(ob);
            if (!oe || oe > le) return fail(NBG_EINVAL, "tuning: malformed override");
            long long N = 0, sq = 0, tt = 0, cm = 0;
            if (!json_int(ob, oe, "N", &N) || N < 4) return fail(NBG_EINVAL, "tuning: override without N");
            json_int(ob, oe, "sqr", &sq);
            json_int(ob, oe, "tile_target", &tt);
            json_int(ob, oe, "cmax", &cm);
            SplitOverride so;
            so.tile_target = (int)tt;
            so.cmax = (int)cm;
            if ((so.cmax && !pow2(so.cmax)) || so.tile_target < 0 || so.tile_target > 8192 || so.cmax > 1024)
                return fail(NBG_EINVAL, "tuning: override knobs out of range");
            const char* pe = strstr(ob, "\"pass_ends\"");
            if (!pe || pe > oe) return fail(NBG_EINVAL, "tuning: override without pass_ends");
            const char* ab = strchr(pe, '[');
            const char* ae = ab ? json_close(ab) : nullptr;
            if (!ab || !ae || ae > oe) return fail(NBG_EINVAL, "tuning: malformed pass_ends");
            for (const char* q = ab + 1; q < ae;) {
                char* e = nullptr;
                long v = strtol(q, &e, 10);
                if (e == q) { q++; continue; }
                so.pass_ends.push_back((int)v);
                q = e;
            }
            t.overrides[N * 2 + (sq ? 1 : 0)] = so;
            p = oe + 1;
        }
    }
    *this = t;
    return NBG_OK;
}

// ---------------------------------------------------------------------------
// engine

Engine g_eng;

int Engine::init(int device) {
    if (ready) {
        if (device != dev) return fail(NBG_EINVAL, "engine already bound to device %d", dev);
        return NBG_OK;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(NBG_ENODEV, "no CUDA device");
    if (device < 0 || device >= ndev) return fail(NBG_EINVAL, "device %d out of range", device);
    CUDA_TRY(cudaSetDevice(device));
    CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    CUDA_TRY(cudaStreamCreateWithFlags(&copy_in, cudaStreamNonBlocking));
    CUDA_TRY(cudaStreamCreateWithFlags(&copy_out, cudaStreamNonBlocking));
    for (cudaStream_t& s : side) CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    for (auto& row : hb_ev)
        for (cudaEvent_t& e : row) CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    CUDA_TRY(kernels_init((double)PR[0], (double)PR[1]));
    CUDA_TRY(cudaMalloc(&d_plans, sizeof(DPlan) * (size_t)plan_cap));
    CUDA_TRY(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device));
    smem_optin = kernels_smem_optin();
    dev = device;
    ready = true;
    return NBG_OK;
}

void autoload_tuning_hook();

int Engine::ensure() {
    if (ready) {
        cudaSetDevice(dev);
        return NBG_OK;
    }
    int rc = init(0);
    if (!rc) autoload_tuning_hook();
    return rc;
}

// Stage list, combine constants and pass split for length N (build_fp_plan,
// fpntt.jl:236-271).  Host only; the twiddle tables are added by build_plan.
int plan_structure(int64_t N, int for_sqr, const Tuning& tun, DPlan& d) {
    if (N < 4) return fail(NBG_EINVAL, "transform length %lld < 4", (long long)N);
    const int k = __builtin_ctzll((uint64_t)N);
    const int64_t m = N >> k;
    static const int64_t okm[] = {1, 3, 5, 7, 9, 15, 21, 35, 45, 63, 105, 315};
    bool okm_hit = false;
    for (int64_t v : okm) okm_hit |= (m == v);
    if (!okm_hit || !(m == 1 || k >= 2) || k > std::min(TWOADIC[0], TWOADIC[1]))
        return fail(NBG_EINVAL, "inadmissible transform length %lld", (long long)N);
    // Tile coordinates and in-tile offsets are 32-bit, global offsets 64-bit:
    // lengths up to 2^32 points (a square there needs about 140 GB of HBM).
    if (N > (int64_t(1) << 32))
        return fail(NBG_ENOMEM, "transform length %lld is beyond one GPU (at most 2^32 points)", (long long)N);

    memset(&d, 0, sizeof d);
    d.N = N;
    struct HS { int m; int64_t L, Q; };
    std::vector<HS> hs;
    int64_t span = N, mm = m;
    for (int mf : {7, 5, 3, 3})
        if (mm % mf == 0) {
            hs.push_back({mf, span, span / mf});
            span /= mf;
            mm /= mf;
        }
    const int64_t N2 = span;
    for (int64_t L = N2; L >= 4; L >>= 2) hs.push_back({4, L, L / 4});
    if (__builtin_ctzll((uint64_t)N2) & 1) hs.push_back({2, 2, 1});
    const int S = (int)hs.size();
    if (S > MAXST) return fail(NBG_EINVAL, "too many stages");
    d.nst = S;
    for (int s = 0; s < S; s++) {
        d.st[s].m = hs[s].m;
        d.st[s].L = hs[s].L;
        d.st[s].Q = hs[s].Q;
    }

    // combine constants per prime
    for (int f = 0; f < 2; f++) {
        const uint64_t p = PR[f];
        const double P = (double)p;
        uint64_t r = powmod_u(generator(f), (p - 1) / (uint64_t)N, p);
        int s = 0;
        for (; s < S && hs[s].m != 4 && hs[s].m != 2; s++) {
            uint64_t c = powmod_u(r, (uint64_t)hs[s].Q, p);
            double* rot = d.st[s].rot[f];
            if (hs[s].m == 5) dft5_consts(c, P, p, rot);
            else if (hs[s].m == 7) dft7_consts(c, P, p, rot);
            else
                for (int t = 1; t < hs[s].m; t++) rot[t - 1] = h_reduce((double)powmod_u(c, (uint64_t)t, p), P);
            r = powmod_u(r, (uint64_t)hs[s].m, p);
        }
        double wi = N2 >= 4 ? h_reduce((double)powmod_u(r, (uint64_t)(N2 >> 2), p), P) : 1.0;
        for (; s < S; s++) d.st[s].rot[f][0] = (hs[s].m == 4) ? wi : 0.0;
        d.ninv[f] = h_reduce((double)invmod_u((uint64_t)N % p, p), P);
        d.ninvp[f] = d.ninv[f] / P;
    }

    // pass split: an autotuned override for this class, else the last pass is
    // the longest suffix whose span fits last_max (a contiguous block, C = 1)
    // and earlier stages are grouped greedily into column passes of at most
    // early_gmax rows.
    const int ntiles_last = for_sqr ? 2 : 4;
    auto ov = tun.overrides.find(N * 2 + (for_sqr ? 1 : 0));
    if (ov != tun.overrides.end()) {
        const SplitOverride& so = ov->second;
        const int tt = so.tile_target ? so.tile_target : tun.tile_target;
        const int cm = so.cmax ? so.cmax : tun.cmax;
        const int np = (int)so.pass_ends.size();
        if (np < 1 || np > MAXPASS || so.pass_ends.back() != S - 1)
            return fail(NBG_EINVAL, "tuning override for N=%lld: bad pass_ends", (long long)N);
        int sa = 0;
        for (int p = 0; p < np; p++) {
            const int sb = so.pass_ends[p];
            if (sb < sa || sb >= S) return fail(NBG_EINVAL, "tuning override for N=%lld: bad pass_ends", (long long)N);
            DPass& ps = d.pass[p];
            ps.sa = sa;
            ps.sb = sb;
            ps.Qb = hs[sb].Q;
            ps.G = (int32_t)(hs[sa].L / ps.Qb);
            if (p == np - 1) {
                ps.C = 1;
                if ((size_t)ntiles_last * tile_stride_doubles(ps.G) * sizeof(double) > PASS_SMEM_LIMIT)
                    return fail(NBG_EINVAL, "tuning override for N=%lld: last pass too large", (long long)N);
            } else {
                const int64_t low = ps.Qb & -ps.Qb;
                ps.C = (int32_t)std::min<int64_t>(low, std::min<int64_t>(cm, pow2floor(std::max<int64_t>(1, tt / ps.G))));
                if (2 * (size_t)tile_stride_doubles(ps.G * ps.C) * sizeof(double) > PASS_SMEM_LIMIT)
                    return fail(NBG_EINVAL, "tuning override for N=%lld: column tile too large", (long long)N);
            }
            ps.ntiles = (N / hs[sa].L) * (ps.Qb / ps.C);
            sa = sb + 1;
        }
        d.npass = np;
        return plan_rounds(d);
    }
    const int full_max = for_sqr ? tun.full_max_sqr : tun.full_max_mul;
    const int last_max = for_sqr ? tun.last_max_sqr : tun.last_max;
    int a = 0;
    if (N > full_max) {
        a = S - 1;
        for (int s = 0; s < S; s++)
            if (hs[s].L <= last_max) { a = s; break; }
        if (a == 0) a = 1;
    }
    int np = 0;
    int sa = 0;
    while (sa < a) {
        int sb = sa;
        while (sb + 1 < a && hs[sa].L / hs[sb + 1].Q <= tun.early_gmax) sb++;
        const int64_t Qb = hs[sb].Q;
        const int64_t G = hs[sa].L / Qb;
        const int64_t low = Qb & -Qb;
        int64_t C = std::min<int64_t>(low, std::min<int64_t>(tun.cmax, pow2floor(std::max<int64_t>(1, tun.tile_target / G))));
        if (np >= MAXPASS - 1) return fail(NBG_EINVAL, "too many passes for N=%lld", (long long)N);
        DPass& ps = d.pass[np++];
        ps.sa = sa;
        ps.sb = sb;
        ps.G = (int32_t)G;
        ps.C = (int32_t)C;
        ps.Qb = Qb;
        ps.ntiles = (N / hs[sa].L) * (Qb / C);
        sa = sb + 1;
    }
    {
        DPass& ps = d.pass[np++];
        ps.sa = a;
        ps.sb = S - 1;
        ps.G = (int32_t)hs[a].L;
        ps.C = 1;
        ps.Qb = 1;
        ps.ntiles = N / hs[a].L;
    }
    d.npass = np;
    return plan_rounds(d);
}

// Rounds of every pass: odd stages one by one; the pass's radix-4 run is
// paired from its smallest span upwards (radix-8 round for the span-8 stage
// and radix-2 when the transform ends with one), a leftover radix-4 at the
// top alone.
int plan_rounds(DPlan& d) {
    for (int p = 0; p < d.npass; p++) {
        DPass& ps = d.pass[p];
        int nr = 0;
        int s = ps.sa;
        for (; s <= ps.sb && (d.st[s].m == 3 || d.st[s].m == 5 || d.st[s].m == 7); s++) {
            ps.rkind[nr] = RK_ODD;
            ps.rstage[nr++] = (int8_t)s;
        }
        int8_t kind[MAXST], first[MAXST];
        int nb = 0;
        int e = ps.sb;
        if (e >= s && d.st[e].m == 2) {
            if (e - 1 >= s && d.st[e - 1].m == 4 && d.st[e - 1].L == 8) {
                kind[nb] = RK_R8;
                first[nb++] = (int8_t)(e - 1);
                e -= 2;
            } else {
                kind[nb] = RK_R2;
                first[nb++] = (int8_t)e;
                e -= 1;
            }
        }
        while (e - 1 >= s) {
            kind[nb] = RK_R16;
            first[nb++] = (int8_t)(e - 1);
            e -= 2;
        }
        if (e == s) {
            kind[nb] = RK_R4;
            first[nb++] = (int8_t)s;
        }
        for (int i = nb - 1; i >= 0; i--) {
            ps.rkind[nr] = kind[i];
            ps.rstage[nr++] = first[i];
        }
        ps.nrounds = nr;
    }
    return NBG_OK;
}

// Plan with device twiddle tables (one allocation for both primes).
int Engine::build_plan(int64_t N, PlanRec& pr, int for_sqr) {
    DPlan& d = pr.d;
    int prc = plan_structure(N, for_sqr, tun, d);
    if (prc) return prc;
    const int S = d.nst;
    struct HS { int m; int64_t L, Q; };
    std::vector<HS> hs((size_t)S);
    for (int s = 0; s < S; s++) hs[(size_t)s] = {d.st[s].m, d.st[s].L, d.st[s].Q};

    // twiddle tables: per prime sum_s (m_s - 1) Q_s doubles, expanded on device
    size_t per = 0;
    for (int s = 0; s < S; s++)
        if (hs[s].m != 2) per += (size_t)(hs[s].m - 1) * (size_t)hs[s].Q;
    const int64_t nhi = (N + 4095) / 4096;
    std::vector<double> hilo((size_t)(nhi + 4096));
    double* dtab = nullptr;
    double* dtmp = nullptr;
    CUDA_TRY(cudaMalloc(&dtab, sizeof(double) * 2 * per));
    if (cudaMalloc(&dtmp, sizeof(double) * hilo.size()) != cudaSuccess) {
        cudaFree(dtab);
        return fail(NBG_ENOMEM, "twiddle staging allocation failed");
    }
    int rc = NBG_OK;
    for (int f = 0; f < 2 && rc == NBG_OK; f++) {
        const uint64_t p = PR[f];
        const double P = (double)p;
        const uint64_t w = powmod_u(generator(f), (p - 1) / (uint64_t)N, p);
        const uint64_t w4096 = powmod_u(w, 4096, p);
        uint64_t x = 1;
        for (int64_t i = 0; i < nhi; i++) {
            hilo[(size_t)i] = h_minbal((double)x, P);
            x = mulmod_u(x, w4096, p);
        }
        x = 1;
        for (int i = 0; i < 4096; i++) {
            hilo[(size_t)(nhi + i)] = h_minbal((double)x, P);
            x = mulmod_u(x, w, p);
        }
        if (cudaMemcpyAsync(dtmp, hilo.data(), sizeof(double) * hilo.size(), cudaMemcpyHostToDevice, stream) !=
            cudaSuccess) {
            rc = fail(NBG_ECUDA, "twiddle upload failed");
            break;
        }
        size_t off = (size_t)f * per;
        for (int s = 0; s < S; s++) {
            if (hs[s].m == 2) {
                d.st[s].tw[f] = nullptr;
                continue;
            }
            double* out = dtab + off;
            d.st[s].tw[f] = out;
            if (launch_twiddle(out, hs[s].m, hs[s].Q, N / hs[s].L, dtmp, dtmp + nhi, f, stream) != cudaSuccess) {
                rc = fail(NBG_ECUDA, "twiddle kernel launch failed");
                break;
            }
            g_launches++;
            off += (size_t)(hs[s].m - 1) * (size_t)hs[s].Q;
        }
        // hilo is reused for the second prime: wait for the copy to finish
        if (cudaStreamSynchronize(stream) != cudaSuccess) rc = fail(NBG_ECUDA, "twiddle build failed");
    }
    cudaFree(dtmp);
    if (rc != NBG_OK) {
        cudaFree(dtab);
        return rc;
    }
    pr.dtab = dtab;
    pr.table_bytes = sizeof(double) * 2 * per;
    if (plan_used >= plan_cap) return fail(NBG_ENOMEM, "plan slots exhausted");
    pr.slot = plan_used++;
    CUDA_TRY(cudaMemcpyAsync(d_plans + pr.slot, &d, sizeof(DPlan), cudaMemcpyHostToDevice, stream));
    CUDA_TRY(cudaStreamSynchronize(stream));
    return NBG_OK;
}

int Engine::get_plan(int64_t N, int for_sqr, PlanRec** out) {
    const int64_t key = N * 2 + (for_sqr ? 1 : 0);
    auto it = plans.find(key);
    if (it != plans.end()) {
        *out = &it->second;
        return NBG_OK;
    }
    PlanRec pr;
    int rc = build_plan(N, pr, for_sqr);
    if (rc) return rc;
    auto ins = plans.emplace(key, pr);
    *out = &ins.first->second;
    return NBG_OK;
}

void Engine::drop_plans() {
    // Tables of dropped plans stay allocated: graphs of live batches may still
    // reference them.  Only the lookup is reset.
    for (auto& kv : plans) graveyard.push_back(kv.second.dtab);
    plans.clear();
}

void Engine::trim_plans() {
    cudaDeviceSynchronize();
    for (double* t : graveyard) cudaFree(t);
    graveyard.clear();
    for (auto& kv : plans) cudaFree(kv.second.dtab);
    plans.clear();
    plan_used = 0;
}

int Engine::ensure_stage(int i, size_t bytes) {
    if (bytes <= stage_bytes[i]) return NBG_OK;
    if (stage[i]) cudaFreeHost(stage[i]);
    stage[i] = nullptr;
    stage_bytes[i] = 0;
    const size_t want = std::max(bytes + bytes / 4, (size_t)1 << 20);
    if (cudaMallocHost((void**)&stage[i], want) != cudaSuccess) {
        cudaGetLastError();
        return fail(NBG_ENOMEM, "pinned staging of %zu bytes unavailable", want);
    }
    stage_bytes[i] = want;
    return NBG_OK;
}

int Engine::ensure_pool(size_t bytes) {
    if (bytes <= pool_bytes) return NBG_OK;
    if (pool) {
        cudaStreamSynchronize(stream);
        cudaFree(pool);
        pool = nullptr;
        pool_bytes = 0;
    }
    size_t want = std::max(bytes, (size_t)64 << 20);
    if (cudaMalloc(&pool, want) != cudaSuccess) {
        cudaGetLastError();
        return fail(NBG_ENOMEM, "device workspace of %zu bytes unavailable", want);
    }
    pool_bytes = want;
    return NBG_OK;
}

// ---------------------------------------------------------------------------
// TMA tensor maps (cuTensorMapEncodeTiled through the runtime's driver entry
// point, so the library needs no link against libcuda)

static PFN_cuTensorMapEncodeTiled_v12000 tma_encoder() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            p = nullptr;
        }
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// A column pass's tiles can be staged by TMA: at least 16 and at most 256
// columns (the dense shared-memory layout is free of bank conflicts from 16
// columns on; a box edge holds at most 256 elements) and at most 256 rows.
static bool tma_pass_ok(const DPass& ps) {
    return ps.C >= 16 && ps.C <= 256 && ps.G <= 256 && ps.Qb % ps.C == 0 && tma_encoder() != nullptr;
}

// The 3-D map over nbuf transform buffers of N doubles at base: dims (Qb, N/Qb,
// nbuf), box (C, G, 2): one box is one tile of both primes of one product.
static int encode_pass_map(void* out, double* base, int64_t N, int64_t nbuf, const DPass& ps) {
    auto enc = tma_encoder();
    if (!enc) return fail(NBG_ECUDA, "cuTensorMapEncodeTiled unavailable");
    const cuuint64_t dims[3] = {(cuuint64_t)ps.Qb, (cuuint64_t)(N / ps.Qb), (cuuint64_t)nbuf};
    const cuuint64_t strides[2] = {(cuuint64_t)ps.Qb * sizeof(double), (cuuint64_t)N * sizeof(double)};
    const cuuint32_t box[3] = {(cuuint32_t)ps.C, (cuuint32_t)ps.G, 2};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(reinterpret_cast<CUtensorMap*>(out), CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base, dims, strides, box,
                     estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(NBG_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return NBG_OK;
}

// ---------------------------------------------------------------------------
// batch construction

static inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

int build_batch(Engine& E, const ProdIn* in, int64_t count, BatchBuild& bb) {
    bb = BatchBuild();
    if (count <= 0) return fail(NBG_EINVAL, "empty batch");
    bb.prods.resize((size_t)count);
    std::vector<int> npass((size_t)count);
    int pmax = 1;
    int bmin = 64;
    size_t work = 0, aggw = 0;
    std::vector<size_t> xa_off((size_t)count), xb_off((size_t)count), agg_off((size_t)count);
    for (int64_t k = 0; k < count; k++) {
        const ProdIn& q = in[k];
        DProd& P = bb.prods[(size_t)k];
        memset(&P, 0, sizeof P);
        // magnitude bits must describe the buffers: the packer reads limb
        // (bits-1)/64 at most.  A zero operand (no set bit) is the caller's
        // case to handle, as NBig * does before reaching the engine.
        if (q.bits_a < 1 || q.bits_a > 64 * q.m || (!q.sqr && (q.bits_b < 1 || q.bits_b > 64 * q.n)))
            return fail(NBG_EINVAL, "product %lld: magnitude bits out of range (zero operand?)", (long long)k);
        int bch;
        int64_t N;
        int rc = ntt_params(q.bits_a, q.sqr ? q.bits_a : q.bits_b, &bch, &N);
        if (rc) return rc;
        PlanRec* pr;
        rc = E.get_plan(N, q.sqr, &pr);
        if (rc) return rc;
        P.a = q.a;
        P.b = q.sqr ? q.a : q.b;
        P.r = q.r;
        P.m = q.m;
        P.n = q.sqr ? q.m : q.n;
        P.rn = P.m + P.n;
        P.bch = bch;
        P.sqr = q.sqr;
        P.nca = (q.bits_a + bch - 1) / bch;
        P.ncb = q.sqr ? P.nca : (q.bits_b + bch - 1) / bch;
        P.nconv = P.nca + P.ncb - 1;
        P.plan = pr->slot;
        P.npass = pr->d.npass;
        P.flags = 0;
        P.ntl = (P.rn + UNPACK_TL - 1) / UNPACK_TL;
        npass[(size_t)k] = P.npass;
        pmax = std::max(pmax, P.npass);
        bmin = std::min(bmin, bch);
        if (q.keep_b && (P.npass != 1 || P.sqr))
            return fail(NBG_EINVAL, "product %lld: a kept operand spectrum needs a one-pass product", (long long)k);
        if (q.keep_b) P.flags |= PF_BSAVE;
        agg_off[(size_t)k] = aggw;
        aggw += (size_t)P.ntl;
        bb.plan_of.push_back(pr);
    }
    bb.agg_words = aggw;
    bb.agg_off = agg_off;

    // Jobs of one pipeline step, grouped by kernel and shared-memory size: a
    // launch reserves its largest job's shared memory for every CTA, so a
    // few big-tile jobs must not lower the occupancy of the rest.
    // algorithmic FP64 instructions per butterfly of the reference schedule
    // (fwd, rev), counted on the oracle's restatement: radix-2 10, radix-3 32,
    // radix-4 40, radix-5 94/98, radix-7 173/201; pointwise 7 per point; the
    // Garner unpack 28 per coefficient.
    auto bfly_ops = [](int m, bool fwd_dir) -> double {
        switch (m) {
            case 2: return 10;
            case 3: return 32;
            case 4: return 40;
            case 5: return fwd_dir ? 94 : 98;
            default: return fwd_dir ? 173 : 201;
        }
    };
    auto pass_ops = [&](const DPlan& pl, const DPass& ps, bool fwd_dir) {  // per tile, one prime
        double o = 0;
        for (int s = ps.sa; s <= ps.sb; s++) o += bfly_ops(pl.st[s].m, fwd_dir) * (double)ps.G * ps.C / pl.st[s].m;
        return o;
    };
    struct Group {
        std::vector<JobSeg> segs;
        std::vector<int32_t> plist;
        int64_t njobs = 0;
        int mode = JM_SEGS;
        double ops = 0, bytes = 0;
    };
    // key: (step order, kind, smem, odd stages present)
    std::map<std::tuple<int, int, size_t, int>, Group> groups;
    auto group_of = [&](int order, int kind, size_t smem, bool odd = false) -> Group& {
        return groups[std::make_tuple(order, kind, smem, odd ? 1 : 0)];
    };
    auto pass_odd = [](const DPlan& pl, const DPass& ps) {
        for (int st = ps.sa; st <= ps.sb; st++)
            if (pl.st[st].m & 1) return true;
        return false;
    };
    // step order: forward steps 0..pmax-2, the pointwise step pmax-1, reverse
    // steps pmax..2pmax-2, unpack 2pmax-1, carry 2pmax
    //
    // Products of one plan share every pass shape, so transform jobs are
    // emitted per plan class, with no per-job sorting: classes by transform
    // length (longest first, so the tail of each launch is short), then tile,
    // then operand, then product.  CTAs that run together read the same
    // twiddle slice, which comes from DRAM once and from L2 for the rest.
    std::vector<int32_t> byclass((size_t)count);
    for (int64_t k = 0; k < count; k++) byclass[(size_t)k] = (int32_t)k;
    std::stable_sort(byclass.begin(), byclass.end(), [&](int32_t x, int32_t y) {
        const int64_t nx = bb.plan_of[(size_t)x]->d.N, ny = bb.plan_of[(size_t)y]->d.N;
        if (nx != ny) return nx > ny;
        const int px = bb.prods[(size_t)x].plan, py = bb.prods[(size_t)y].plan;
        if (px != py) return px < py;
        return (bb.prods[(size_t)x].flags & PF_BSAVE) < (bb.prods[(size_t)y].flags & PF_BSAVE);
    });
    std::vector<int32_t> cls;
    bb.class_of.assign((size_t)count, -1);
    const Tuning& tun = E.tun;
    // A batch whose last-pass tiles are fewer than one wave of CTAs (3 per SM)
    // gives each prime of a tile its own CTA: twice the CTAs, half the
    // critical path each (small batches are latency-bound).
    int64_t pwr_tiles = 0;
    for (int64_t k = 0; k < count; k++) {
        const DPlan& pl = bb.plan_of[(size_t)k]->d;
        pwr_tiles += pl.pass[pl.npass - 1].ntiles;
    }
    const bool split_pwr = pwr_tiles < 3 * (int64_t)std::max(E.num_sms, 1);
    for (size_t i = 0; i < byclass.size();) {
        const int slot = bb.prods[(size_t)byclass[i]].plan;
        const int keep0 = bb.prods[(size_t)byclass[i]].flags & PF_BSAVE;
        cls.clear();
        double sum_bch = 0;
        while (i < byclass.size() && bb.prods[(size_t)byclass[i]].plan == slot &&
               (bb.prods[(size_t)byclass[i]].flags & PF_BSAVE) == keep0) {
            sum_bch += bb.prods[(size_t)byclass[i]].bch;
            cls.push_back(byclass[i++]);
        }
        const DProd& P0 = bb.prods[(size_t)cls[0]];
        const DPlan& pl = bb.plan_of[(size_t)cls[0]]->d;
        const int Pn = P0.npass;
        const int nop = P0.sqr ? 1 : 2;
        const double nc = (double)cls.size();
        // the class's transform buffers are contiguous: [xa of each product][xb of each product]
        {
            const size_t N2 = 2 * (size_t)pl.N;
            const bool has_b = (Pn > 1 && !P0.sqr) || keep0;
            BatchBuild::ClassRec cr;
            cr.xa0 = work;
            cr.xb0 = has_b ? work + N2 * cls.size() : SIZE_MAX;
            cr.nprod = (int32_t)cls.size();
            cr.plan = bb.plan_of[(size_t)cls[0]];
            for (size_t j = 0; j < cls.size(); j++) {
                xa_off[(size_t)cls[j]] = cr.xa0 + N2 * j;
                xb_off[(size_t)cls[j]] = has_b ? cr.xb0 + N2 * j : SIZE_MAX;
                bb.prods[(size_t)cls[j]].tslot = (int32_t)j;
            }
            work += N2 * cls.size() * (has_b ? 2 : 1);
            for (int p = 0; p < Pn - 1; p++) {
                if (!tun.tma || !tma_pass_ok(pl.pass[p])) continue;
                cr.tma_mask |= 1u << p;
                if (cr.map0 < 0) {
                    cr.map0 = bb.ntmaps;
                    bb.ntmaps += 2 * (Pn - 1);
                }
            }
            bb.classes.push_back(cr);
            for (int32_t k : cls) bb.class_of[(size_t)k] = (int32_t)bb.classes.size() - 1;
        }
        const uint32_t tmask = bb.classes.back().tma_mask;
        auto emit = [&](Group& g, const DPass& ps, int nopnd, int sub_base) {
            JobSeg sg;
            const int64_t per = ps.Qb / ps.C, nblk = ps.ntiles / per;
            const bool colmajor = per > 1 && nblk > 1;
            sg.per = colmajor ? (int32_t)per : 0;
            sg.nblk = colmajor ? (int32_t)nblk : 0;
            sg.begin = g.njobs;
            sg.ntiles = ps.ntiles;
            sg.nop = nopnd;
            sg.nprod = (int32_t)cls.size();
            sg.first = (int32_t)g.plist.size();
            sg.sub_base = sub_base;
            g.segs.push_back(sg);
            g.plist.insert(g.plist.end(), cls.begin(), cls.end());
            g.njobs += ps.ntiles * nopnd * (int64_t)cls.size();
        };
        for (int p = 0; p < Pn - 1; p++) {
            const DPass& ps = pl.pass[p];
            const bool tp = (tmask >> p) & 1u;
            const size_t smem = tp ? 128 + sizeof(double) * 2 * (size_t)(ps.G * ps.C)
                                   : sizeof(double) * 2 * (size_t)tile_stride_doubles(ps.G * ps.C);
            const double pts = (double)ps.G * ps.C;
            const double jobs = (double)ps.ntiles * nop * nc;
            Group& g = group_of(pmax - Pn + p, tp ? JK_FWD_TMA : JK_FWD, smem, pass_odd(pl, ps));
            emit(g, ps, nop, p << 8);
            g.ops += jobs * 2.0 * pass_ops(pl, ps, true);
            // first pass reads packed limbs (bch bits per point), later ones both primes' doubles
            const double in_b = p == 0 ? (double)ps.ntiles * nop * pts * sum_bch / 8.0 : jobs * 2.0 * 8.0 * pts;
            g.bytes += in_b + jobs * 2.0 * 8.0 * pts;
        }
        {
            const DPass& ps = pl.pass[Pn - 1];
            // splitting pays only where a tile set holds more 16-point units
            // than a CTA has threads (smaller tiles just repeat the pack)
            const bool keep = keep0 != 0;
            const bool split = !keep && split_pwr && (int64_t)ps.G * ps.C * 2 * nop > 16 * PASS_THREADS;
            const size_t smem = sizeof(double) * (P0.sqr ? 1 : 2) * (split ? 1 : 2) *
                                (size_t)tile_stride_doubles(ps.G * ps.C);
            const double pts = (double)ps.G * ps.C;
            const double jobs = (double)ps.ntiles * nc;  // tiles of both primes (the work, split or not)
            Group& g = group_of(pmax - 1, keep ? JK_PWR_KEEP : split ? JK_PWR_SPLIT : JK_PWR, smem, pass_odd(pl, ps));
            emit(g, ps, split ? 2 : 1, (Pn - 1) << 8);  // split: "operand" is the prime
            g.ops += jobs * 2.0 * (nop * pass_ops(pl, ps, true) + 7.0 * pts + pass_ops(pl, ps, false));
            const double in_b = Pn == 1 ? (double)ps.ntiles * nop * pts * sum_bch / 8.0 : jobs * 2.0 * nop * 8.0 * pts;
            g.bytes += in_b + jobs * 2.0 * 8.0 * pts;
        }
        for (int p = Pn - 2; p >= 0; p--) {
            const DPass& ps = pl.pass[p];
            const bool tp = (tmask >> p) & 1u;
            const size_t smem = tp ? 128 + sizeof(double) * 2 * (size_t)(ps.G * ps.C)
                                   : sizeof(double) * 2 * (size_t)tile_stride_doubles(ps.G * ps.C);
            const double pts = (double)ps.G * ps.C;
            const double jobs = (double)ps.ntiles * nc;
            Group& g = group_of(pmax + (Pn - 2 - p), tp ? JK_REV_TMA : JK_REV, smem, pass_odd(pl, ps));
            emit(g, ps, 1, p << 8);
            g.ops += jobs * 2.0 * pass_ops(pl, ps, false);
            g.bytes += jobs * 2.0 * 16.0 * pts;
        }
    }
    bb.work_doubles = work;
    bb.xa_off = xa_off;
    bb.xb_off = xb_off;
    const size_t unp_smem = unpack_smem_bytes(bmin);
    // unpack: product k owns tiles [agg_off[k], agg_off[k] + ntl); carry: one CTA per product
    Group& gu = group_of(2 * pmax - 1, JK_UNPACK, unp_smem);
    gu.mode = JM_TILES;
    gu.njobs = (int64_t)aggw;
    bool any_carry = false;
    double carry_bytes = 0;
    for (int64_t k = 0; k < count; k++) {
        const DProd& P = bb.prods[(size_t)k];
        gu.ops += 28.0 * (double)P.nconv;
        gu.bytes += 16.0 * (double)P.nconv + 8.0 * (double)P.rn;
        if (P.ntl > 1) {
            any_carry = true;
            carry_bytes += 4.0 * (double)P.ntl;
        }
    }
    if (any_carry) {
        Group& gc = group_of(2 * pmax, JK_CARRY, 0);
        gc.mode = JM_PERPROD;
        gc.njobs = count;
        gc.bytes = carry_bytes;
        Group& gf = group_of(2 * pmax + 1, JK_CARRYFIX, 0);  // the unpack's tiles again
        gf.mode = JM_TILES;
        gf.njobs = (int64_t)aggw;
    }
    // job table: [segments | product list] per launch, then the unpack tile starts
    size_t tb = 0;
    for (auto& kv : groups) {
        const Group& g = kv.second;
        const int kind = std::get<1>(kv.first);
        Launch L{kind, bb.total_jobs, g.njobs, std::get<2>(kv.first)};
        L.odd = std::get<3>(kv.first) != 0;
        bb.total_jobs += g.njobs;
        L.step = std::get<0>(kv.first);
        L.alg_ops = g.ops;
        L.alg_bytes = g.bytes;
        L.mode = g.mode;
        if ((int)L.smem > E.smem_optin) return fail(NBG_EINVAL, "tile needs %zu bytes of shared memory", L.smem);
        if (g.mode == JM_SEGS) {
            L.nseg = (int)g.segs.size();
            L.seg_off = tb;
            tb = align_up(tb + sizeof(JobSeg) * g.segs.size(), 16);
            L.plist_off = tb;
            tb = align_up(tb + sizeof(int32_t) * g.plist.size(), 16);
        }
        bb.launches.push_back(L);
    }
    bb.tstart_off = tb;
    tb = align_up(tb + sizeof(int64_t) * ((size_t)count + 1), 128);
    bb.tmap_off = tb;  // 128-byte tensor maps, written by bind_batch
    tb = align_up(tb + 128 * (size_t)bb.ntmaps, 16);
    bb.expand_off = tb;
    tb = align_up(tb + sizeof(ExpandEntry) * bb.launches.size(), 16);
    bb.table.assign(tb, 0);
    {
        size_t li = 0;
        for (auto& kv : groups) {
            const Group& g = kv.second;
            const Launch& L = bb.launches[li++];
            if (g.mode != JM_SEGS) continue;
            memcpy(bb.table.data() + L.seg_off, g.segs.data(), sizeof(JobSeg) * g.segs.size());
            memcpy(bb.table.data() + L.plist_off, g.plist.data(), sizeof(int32_t) * g.plist.size());
        }
        int64_t* ts = (int64_t*)(bb.table.data() + bb.tstart_off);
        for (int64_t k = 0; k < count; k++) ts[k] = (int64_t)agg_off[(size_t)k];
        ts[count] = (int64_t)aggw;
    }

    // device layout: [prods | jobs | work | agg]
    bb.off_prods = 0;
    bb.off_jobs = align_up(sizeof(DProd) * (size_t)count, 256);
    bb.head_bytes = bb.off_jobs + bb.table.size();
    bb.off_joblist = align_up(bb.head_bytes, 256);
    bb.off_work = align_up(bb.off_joblist + sizeof(Job) * (size_t)bb.total_jobs, 256);
    bb.off_agg = align_up(bb.off_work + sizeof(double) * work, 256);
    bb.dev_bytes = align_up(bb.off_agg + sizeof(uint32_t) * aggw, 256);
    return NBG_OK;
}

int bind_batch(BatchBuild& bb, char* dbase) {
    double* work = (double*)(dbase + bb.off_work);
    uint32_t* agg = (uint32_t*)(dbase + bb.off_agg);
    // tensor maps of the TMA column passes, per class [pass][operand]
    for (const BatchBuild::ClassRec& cr : bb.classes) {
        if (cr.map0 < 0) continue;
        const DPlan& pl = cr.plan->d;
        for (int p = 0; p + 1 < pl.npass; p++) {
            if (!((cr.tma_mask >> p) & 1u)) continue;
            for (int op = 0; op < 2; op++) {
                const size_t off = op ? cr.xb0 : cr.xa0;
                if (off == SIZE_MAX) continue;
                char* dst = bb.table.data() + bb.tmap_off + 128 * (size_t)(cr.map0 + 2 * p + op);
                int rc = encode_pass_map(dst, work + off, pl.N, 2 * (int64_t)cr.nprod, pl.pass[p]);
                if (rc) return rc;
            }
        }
    }
    for (size_t k = 0; k < bb.prods.size(); k++) {
        DProd& P = bb.prods[k];
        const int64_t N = bb.plan_of[k]->d.N;
        P.xa[0] = work + bb.xa_off[k];
        P.xa[1] = P.xa[0] + N;
        if (bb.xb_off[k] != SIZE_MAX) {
            P.xb[0] = work + bb.xb_off[k];
            P.xb[1] = P.xb[0] + N;
        } else {
            P.xb[0] = P.xb[1] = nullptr;
        }
        P.agg = agg + bb.agg_off[k];
        const BatchBuild::ClassRec& cr = bb.classes[(size_t)bb.class_of[k]];
        P.tmap = cr.map0 < 0 ? nullptr : dbase + bb.off_jobs + bb.tmap_off + 128 * (size_t)cr.map0;
    }
    ExpandEntry* ex = (ExpandEntry*)(bb.table.data() + bb.expand_off);
    for (size_t i = 0; i < bb.launches.size(); i++) {
        ex[i].src = launch_src(bb, bb.launches[i], dbase);
        ex[i].begin = bb.launches[i].off;
        ex[i].n = bb.launches[i].n;
    }
    return NBG_OK;
}

void stage_batch(const BatchBuild& bb, char* host) {
    memset(host, 0, bb.head_bytes);
    memcpy(host + bb.off_prods, bb.prods.data(), sizeof(DProd) * bb.prods.size());
    if (!bb.table.empty()) memcpy(host + bb.off_jobs, bb.table.data(), bb.table.size());
}

JobSrc launch_src(const BatchBuild& bb, const Launch& L, const char* dbase) {
    JobSrc s{};
    const char* t = dbase + bb.off_jobs;
    s.mode = L.mode;
    s.segs = (const JobSeg*)(t + L.seg_off);
    s.nseg = L.nseg;
    s.plist = (const int32_t*)(t + L.plist_off);
    s.tstart = (const int64_t*)(t + bb.tstart_off);
    s.nprod = (int64_t)bb.prods.size();
    return s;
}

// Point the descriptors at the device block and upload descriptors + job table.
int upload_batch(Engine& E, BatchBuild& bb, char* dbase, cudaStream_t st) {
    int rc = bind_batch(bb, dbase);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpyAsync(dbase + bb.off_prods, bb.prods.data(), sizeof(DProd) * bb.prods.size(),
                             cudaMemcpyHostToDevice, st));
    if (!bb.table.empty())
        CUDA_TRY(cudaMemcpyAsync(dbase + bb.off_jobs, bb.table.data(), bb.table.size(),
                                 cudaMemcpyHostToDevice, st));
    (void)E;
    return NBG_OK;
}

cudaError_t expand_jobs(const BatchBuild& bb, char* dbase, cudaStream_t st) {
    return launch_expand((const ExpandEntry*)(dbase + bb.off_jobs + bb.expand_off), (int)bb.launches.size(),
                         (Job*)(dbase + bb.off_joblist), bb.total_jobs, st);
}

int run_launches(Engine& E, const BatchBuild& bb, char* dbase, cudaStream_t st, bool expand) {
    const DProd* prods = (const DProd*)(dbase + bb.off_prods);
    const Job* jobs = (const Job*)(dbase + bb.off_joblist);
    if (expand) {
        CUDA_TRY(expand_jobs(bb, dbase, st));
        g_launches++;
    }
    for (const Launch& L : bb.launches) {
        cudaError_t e = launch_jobs(L.kind, prods, E.d_plans, job_list(jobs + L.off), L.n, L.smem, 0, st, L.odd);
        if (e != cudaSuccess) return fail(NBG_ECUDA, "launch (kind %d, %lld jobs): %s", L.kind, (long long)L.n,
                                          cudaGetErrorString(e));
        g_launches++;
    }
    return NBG_OK;
}

int run_launches_branched(Engine& E, const BatchBuild& bb, char* dbase, cudaStream_t st, cudaStream_t* side,
                          int nside) {
    const DProd* prods = (const DProd*)(dbase + bb.off_prods);
    const Job* jobs = (const Job*)(dbase + bb.off_joblist);
    CUDA_TRY(expand_jobs(bb, dbase, st));
    g_launches++;
    size_t i = 0;
    while (i < bb.launches.size()) {
        size_t j = i;
        while (j < bb.launches.size() && bb.launches[j].step == bb.launches[i].step) j++;
        // launches [i, j) share a step: the first on st, the rest forked
        std::vector<cudaEvent_t> joins;
        cudaEvent_t fork = nullptr;
        if (j - i > 1) {
            CUDA_TRY(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
            CUDA_TRY(cudaEventRecord(fork, st));
        }
        for (size_t k = i; k < j; k++) {
            const Launch& L = bb.launches[k];
            cudaStream_t s = st;
            if (k > i && nside > 0) {
                s = side[(k - i - 1) % (size_t)nside];
                CUDA_TRY(cudaStreamWaitEvent(s, fork, 0));
            }
            cudaError_t e = launch_jobs(L.kind, prods, E.d_plans, job_list(jobs + L.off), L.n, L.smem, 0, s, L.odd);
            if (e != cudaSuccess)
                return fail(NBG_ECUDA, "launch (kind %d, %lld jobs): %s", L.kind, (long long)L.n, cudaGetErrorString(e));
            g_launches++;
            if (s != st) {
                cudaEvent_t jv;
                CUDA_TRY(cudaEventCreateWithFlags(&jv, cudaEventDisableTiming));
                CUDA_TRY(cudaEventRecord(jv, s));
                joins.push_back(jv);
            }
        }
        for (cudaEvent_t jv : joins) {
            CUDA_TRY(cudaStreamWaitEvent(st, jv, 0));
            cudaEventDestroy(jv);
        }
        if (fork) cudaEventDestroy(fork);
        i = j;
    }
    return NBG_OK;
}

int queue_prepare(Engine& E, const BatchBuild& bb, char* dbase, QueueRun& q, cudaStream_t st) {
    queue_free(q);
    std::vector<QLaunch> tab;
    int64_t total = 0;
    size_t smem = 0;
    for (const Launch& L : bb.launches) {
        if (L.kind == JK_CARRYFIX) continue;  // the carry job fixes its own flagged tiles
        QLaunch e{};
        e.qstart = total;
        e.off = L.off;
        e.kind = L.kind;
        e.odd = L.odd ? 1 : 0;
        tab.push_back(e);
        total += L.n;
        // k_queue's region starts 128 bytes in: column TMA sizes include that
        // header already, the unpack needs one of its two stages
        size_t need = L.smem + 128;
        if (L.kind == JK_FWD_TMA || L.kind == JK_REV_TMA) need = L.smem;
        else if (L.kind == JK_UNPACK) need = 128 + (L.smem - 128) / 2;
        else if (L.kind == JK_CARRY) need = 128;
        smem = std::max(smem, need);
    }
    QLaunch end{};
    end.qstart = total;
    end.kind = -1;
    tab.push_back(end);
    if ((int)smem > E.smem_optin) return fail(NBG_EINVAL, "queue: %zu bytes of shared memory per CTA", smem);
    const size_t nprod = bb.prods.size();
    const size_t cnt = sizeof(uint32_t) * nprod * (size_t)QSTEPS;
    q.off_done = align_up(sizeof(QState), 256);
    q.zero_bytes = q.off_done + cnt;
    q.off_need = align_up(q.zero_bytes, 256);
    q.off_ql = align_up(q.off_need + cnt, 256);
    q.bytes = q.off_ql + sizeof(QLaunch) * tab.size();
    if (cudaMalloc(&q.d, q.bytes) != cudaSuccess) {
        cudaGetLastError();
        q.d = nullptr;
        return fail(NBG_ENOMEM, "queue state of %zu bytes unavailable", q.bytes);
    }
    q.nl = (int)tab.size() - 1;
    q.total = total;
    q.smem = smem;
    q.chunk = std::max(1, E.tun.queue);
    CUDA_TRY(queue_grid(smem, &q.grid));
    CUDA_TRY(cudaMemcpyAsync(q.d + q.off_ql, tab.data(), sizeof(QLaunch) * tab.size(), cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemsetAsync(q.d + q.off_need, 0, cnt, st));
    CUDA_TRY(expand_jobs(bb, dbase, st));
    CUDA_TRY(launch_qcount((const DProd*)(dbase + bb.off_prods), (const Job*)(dbase + bb.off_joblist),
                           (const QLaunch*)(q.d + q.off_ql), q.nl, total, (uint32_t*)(q.d + q.off_need), st));
    return NBG_OK;
}

int queue_run(Engine& E, const BatchBuild& bb, char* dbase, const QueueRun& q, cudaStream_t st) {
    if (!q.d) return fail(NBG_EINVAL, "queue not prepared");
    CUDA_TRY(cudaMemsetAsync(q.d, 0, q.zero_bytes, st));
    CUDA_TRY(expand_jobs(bb, dbase, st));
    CUDA_TRY(launch_queue((const DProd*)(dbase + bb.off_prods), E.d_plans, (const Job*)(dbase + bb.off_joblist),
                          (const QLaunch*)(q.d + q.off_ql), q.nl, (QState*)q.d, (uint32_t*)(q.d + q.off_done),
                          (const uint32_t*)(q.d + q.off_need), q.smem, q.grid, q.chunk, st));
    g_launches += 2;
    return NBG_OK;
}

void queue_free(QueueRun& q) {
    if (q.d) cudaFree(q.d);
    q = QueueRun{};
}

}  // namespace nbg
