// powmod.cpp — Barrett powermod chains on the GPU (nbg_powermod_batch*).
//
// The chains follow the reference's powermod_limbs on its Barrett branch
// (src/algorithms.jl:17-107, src/barrett.jl:33-81): a sliding window over the
// exponent bits from the top, a table of odd powers, and after every multiply
// or square the reduction
//     q1 = floor(T / β^(k-1)),  q3 = floor(q1·μ / β^(k+1)),
//     r  = (T − q3·m) mod β^(k+1),  then r −= m while r ≥ m (at most twice).
// On the device every chain advances one step per exponent step: the step's
// product x·y, then q1·μ, then q3·m — three batches of fp-NTT products, one
// per chain each — and a finishing kernel for the subtraction and the
// corrections.  q1 and q3 are windows of the previous products, so no copies
// are needed between the batches.  The host derives each chain's step list
// once (the window schedule depends only on the exponent) and μ once per
// modulus.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/nbgpu.h"
#include "engine.h"
#include "powmod_kernels.h"

namespace nbg {

typedef unsigned __int128 u128;

// q[0..ulen-vlen] = floor(u / v), u[0..ulen), v[0..vlen) with v[vlen-1] != 0
// (Knuth, TAOCP vol. 2, 4.3.1, Algorithm D; base 2^64).
static void long_divide(const uint64_t* u, int64_t ulen, const uint64_t* v, int64_t vlen, uint64_t* q) {
    const int64_t n = vlen, m = ulen - vlen;
    if (n == 1) {
        u128 r = 0;
        for (int64_t j = ulen - 1; j >= 0; j--) {
            const u128 cur = (r << 64) | u[j];
            q[j] = (uint64_t)(cur / v[0]);
            r = cur % v[0];
        }
        return;
    }
    const int s = __builtin_clzll(v[n - 1]);
    std::vector<uint64_t> vn((size_t)n), un((size_t)(ulen + 1));
    for (int64_t i = n - 1; i > 0; i--) vn[(size_t)i] = (v[i] << s) | (s ? v[i - 1] >> (64 - s) : 0);
    vn[0] = v[0] << s;
    un[(size_t)ulen] = s ? u[ulen - 1] >> (64 - s) : 0;
    for (int64_t i = ulen - 1; i > 0; i--) un[(size_t)i] = (u[i] << s) | (s ? u[i - 1] >> (64 - s) : 0);
    un[0] = u[0] << s;
    const u128 B = (u128)1 << 64;
    for (int64_t j = m; j >= 0; j--) {
        const u128 num = ((u128)un[(size_t)(j + n)] << 64) | un[(size_t)(j + n - 1)];
        u128 qhat = num / vn[(size_t)(n - 1)];
        u128 rhat = num % vn[(size_t)(n - 1)];
        while (qhat >= B || qhat * vn[(size_t)(n - 2)] > ((rhat << 64) | un[(size_t)(j + n - 2)])) {
            qhat--;
            rhat += vn[(size_t)(n - 1)];
            if (rhat >= B) break;
        }
        // un[j .. j+n] -= qhat * vn
        uint64_t borrow = 0, carry = 0;
        for (int64_t i = 0; i < n; i++) {
            const u128 p = qhat * vn[(size_t)i] + carry;
            carry = (uint64_t)(p >> 64);
            const uint64_t lo = (uint64_t)p;
            const uint64_t x = un[(size_t)(i + j)];
            const uint64_t d = x - lo - borrow;
            borrow = (x < lo) || (x - lo < borrow);
            un[(size_t)(i + j)] = d;
        }
        const uint64_t x = un[(size_t)(j + n)];
        const uint64_t d = x - carry - borrow;
        const bool neg = (x < carry) || (x - carry < borrow);
        un[(size_t)(j + n)] = d;
        if (neg) {  // qhat was one too large: add v back
            qhat--;
            uint64_t c = 0;
            for (int64_t i = 0; i < n; i++) {
                const u128 t = (u128)un[(size_t)(i + j)] + vn[(size_t)i] + c;
                un[(size_t)(i + j)] = (uint64_t)t;
                c = (uint64_t)(t >> 64);
            }
            un[(size_t)(j + n)] += c;
        }
        q[j] = (uint64_t)qhat;
    }
}

// Slots of a chain: the odd-power table 0..T-1, then b^2, the accumulator,
// the raw base and the constant 1.
struct Slots {
    int T;
    int bsq() const { return T; }
    int acc() const { return T + 1; }
    int base() const { return T + 2; }
    int one() const { return T + 3; }
    int count() const { return T + 4; }
};

constexpr uint8_t OP_COPY = 255;  // PM_COPY of the device side

static inline bool expbit(const uint64_t* e, int64_t i) { return (e[i >> 6] >> (i & 63)) & 1; }

// The reference's step sequence for exponent e (algorithms.jl:22-26 window
// width, :58-72 table of odd powers, :75-103 the window scan), preceded by
// the reduction of the base (b·1 mod m) into table slot 0.
static int64_t schedule(const uint64_t* e, int64_t le, std::vector<uint8_t>& ops, int* tsize) {
    int64_t nbits = 0;
    for (int64_t i = le - 1; i >= 0; i--)
        if (e[i]) {
            nbits = 64 * i + 64 - __builtin_clzll(e[i]);
            break;
        }
    if (nbits == 0) return -NBG_EINVAL;
    const int w = nbits <= 8 ? 1 : nbits <= 24 ? 2 : nbits <= 80 ? 3 : nbits <= 240 ? 4 : 5;
    Slots S{1 << (w - 1)};
    *tsize = S.T;
    ops.clear();
    auto step = [&](int d, int a, int b) {
        ops.push_back((uint8_t)d);
        ops.push_back((uint8_t)a);
        ops.push_back((uint8_t)b);
    };
    step(0, S.base(), S.one());
    if (S.T > 1) {
        step(S.bsq(), 0, 0);
        for (int j = 1; j < S.T; j++) step(j, j - 1, S.bsq());
    }
    bool first = true;
    int64_t i = nbits - 1;
    while (i >= 0) {
        if (!expbit(e, i)) {
            if (!first) step(S.acc(), S.acc(), S.acc());
            i--;
            continue;
        }
        int64_t l = std::min<int64_t>(w, i + 1);
        while (!expbit(e, i - l + 1)) l--;  // the window ends on a set bit
        int val = 0;
        for (int64_t j = 0; j < l; j++) val = (val << 1) | (int)expbit(e, i - j);
        if (first) {
            step(S.acc(), val >> 1, OP_COPY);
            first = false;
        } else {
            for (int64_t j = 0; j < l; j++) step(S.acc(), S.acc(), S.acc());
            step(S.acc(), S.acc(), val >> 1);
        }
        i -= l;
    }
    return (int64_t)(ops.size() / 3);
}

// ---------------------------------------------------------------------------
// device run

#define PM_TRY(x)                                                                            \
    do {                                                                                     \
        cudaError_t e_ = (x);                                                                \
        if (e_ != cudaSuccess) return fail(NBG_ECUDA, "%s: %s", #x, cudaGetErrorString(e_)); \
    } while (0)

// Device allocations of one call, released on every exit path.
struct PmMem {
    std::vector<void*> blocks;
    ~PmMem() {
        for (void* p : blocks) cudaFree(p);
    }
    template <class T>
    int get(T** out, size_t count) {
        void* p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
            cudaGetLastError();
            return fail(NBG_ENOMEM, "powermod chains: device allocation of %zu bytes failed", count * sizeof(T));
        }
        blocks.push_back(p);
        *out = (T*)p;
        return NBG_OK;
    }
};

struct PmGraph {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t x = nullptr;
    ~PmGraph() {
        if (x) cudaGraphExecDestroy(x);
        if (g) cudaGraphDestroy(g);
    }
};

// Whether a product of these magnitudes runs as one pass (its operand b's
// spectrum can then be kept between runs).
static bool one_pass(Engine& E, int64_t bits_a, int64_t bits_b) {
    int b = 0;
    int64_t N = 0;
    PlanRec* pr = nullptr;
    if (ntt_params(bits_a, bits_b, &b, &N) != NBG_OK || E.get_plan(N, 0, &pr) != NBG_OK) return false;
    return pr->d.npass == 1;
}

// Steps replayed per graph launch.
constexpr int64_t PM_GRAPH_STEPS = 64;

// The chains of d[0..count) (device pointers), modulus size k; hm/he are host
// copies of each chain's modulus and exponent.  Runs on the engine stream and
// returns when the results are written.
static int powmod_run(Engine& E, const nbg_powmod_desc* d, int64_t count, int64_t k,
                      const std::vector<std::vector<uint64_t>>& hm, const std::vector<std::vector<uint64_t>>& he) {
    // step lists, remapped to one slot layout: table 0..Tmax-1, b^2, acc, base, 1
    std::vector<std::vector<uint8_t>> ops((size_t)count);
    std::vector<int> tsz((size_t)count);
    int Tmax = 1;
    int64_t max_steps = 0;
    for (int64_t c = 0; c < count; c++) {
        const int64_t n = schedule(he[(size_t)c].data(), (int64_t)he[(size_t)c].size(), ops[(size_t)c], &tsz[(size_t)c]);
        if (n < 0) return fail(NBG_EINVAL, "chain %lld: zero exponent", (long long)c);
        Tmax = std::max(Tmax, tsz[(size_t)c]);
        max_steps = std::max(max_steps, n);
    }
    const Slots S{Tmax};
    std::vector<uint8_t> hops((size_t)(count * max_steps * 3), 0);
    std::vector<int64_t> hn((size_t)count);
    for (int64_t c = 0; c < count; c++) {
        const int T = tsz[(size_t)c];
        auto remap = [&](uint8_t v) -> uint8_t { return v == OP_COPY ? v : v < T ? v : (uint8_t)(v - T + Tmax); };
        const std::vector<uint8_t>& o = ops[(size_t)c];
        for (size_t i = 0; i < o.size(); i++) hops[(size_t)(c * max_steps * 3) + i] = remap(o[i]);
        hn[(size_t)c] = (int64_t)(o.size() / 3);
    }
    // μ per chain (host long division, once per modulus)
    const int64_t lmu_max = k + 2;
    std::vector<uint64_t> hmu((size_t)(count * lmu_max), 0);
    std::vector<int64_t> lmu((size_t)count), bits_mu((size_t)count), bits_m((size_t)count);
    for (int64_t c = 0; c < count; c++) {
        const int64_t l = nbg_barrett_mu(hm[(size_t)c].data(), k, hmu.data() + c * lmu_max);
        if (l < 0) return fail(NBG_EINVAL, "chain %lld: modulus top limb is zero", (long long)c);
        lmu[(size_t)c] = l;
        bits_mu[(size_t)c] = magnitude_bits(hmu.data() + c * lmu_max, l);
        bits_m[(size_t)c] = magnitude_bits(hm[(size_t)c].data(), k);
    }
    // device state
    PmMem mem;
    PmChains C{};
    C.count = (int32_t)count;
    C.nslot = S.count();
    C.acc_slot = S.acc();
    C.one_slot = S.one();
    C.base_slot = S.base();
    C.k = k;
    C.max_steps = max_steps;
    C.prod_stride = 2 * k + 2;
    C.r2_stride = k + lmu_max;
    const int64_t q2_stride = k + 1 + lmu_max;
    uint8_t* d_ops = nullptr;
    int64_t *d_n = nullptr, *d_ctr = nullptr, *d_lb = nullptr;
    uint64_t *d_slots = nullptr, *d_prod = nullptr, *d_q2 = nullptr, *d_r2 = nullptr, *d_mod = nullptr, *d_mu = nullptr;
    int4* d_cur = nullptr;
    const uint64_t** d_bases = nullptr;
    uint64_t** d_outs = nullptr;
    int rc = 0;
    if ((rc = mem.get(&d_ops, hops.size())) || (rc = mem.get(&d_n, (size_t)count)) || (rc = mem.get(&d_ctr, 1)) ||
        (rc = mem.get(&d_lb, (size_t)count)) || (rc = mem.get(&d_slots, (size_t)(count * C.nslot * k))) ||
        (rc = mem.get(&d_prod, (size_t)(count * C.prod_stride))) || (rc = mem.get(&d_q2, (size_t)(count * q2_stride))) ||
        (rc = mem.get(&d_r2, (size_t)(count * C.r2_stride))) || (rc = mem.get(&d_mod, (size_t)(count * k))) ||
        (rc = mem.get(&d_mu, (size_t)(count * lmu_max))) || (rc = mem.get(&d_cur, (size_t)count)) ||
        (rc = mem.get(&d_bases, (size_t)count)) || (rc = mem.get(&d_outs, (size_t)count)))
        return rc;
    cudaStream_t st = E.stream;
    std::vector<const uint64_t*> hb((size_t)count);
    std::vector<uint64_t*> ho((size_t)count);
    std::vector<int64_t> hlb((size_t)count);
    for (int64_t c = 0; c < count; c++) {
        hb[(size_t)c] = d[c].b;
        ho[(size_t)c] = d[c].r;
        hlb[(size_t)c] = d[c].lb;
        PM_TRY(cudaMemcpyAsync(d_mod + c * k, hm[(size_t)c].data(), sizeof(uint64_t) * (size_t)k,
                               cudaMemcpyHostToDevice, st));
    }
    PM_TRY(cudaMemcpyAsync(d_ops, hops.data(), hops.size(), cudaMemcpyHostToDevice, st));
    PM_TRY(cudaMemcpyAsync(d_n, hn.data(), sizeof(int64_t) * (size_t)count, cudaMemcpyHostToDevice, st));
    PM_TRY(cudaMemcpyAsync(d_lb, hlb.data(), sizeof(int64_t) * (size_t)count, cudaMemcpyHostToDevice, st));
    PM_TRY(cudaMemcpyAsync(d_mu, hmu.data(), sizeof(uint64_t) * hmu.size(), cudaMemcpyHostToDevice, st));
    PM_TRY(cudaMemcpyAsync(d_bases, hb.data(), sizeof(void*) * (size_t)count, cudaMemcpyHostToDevice, st));
    PM_TRY(cudaMemcpyAsync(d_outs, ho.data(), sizeof(void*) * (size_t)count, cudaMemcpyHostToDevice, st));
    PM_TRY(cudaMemsetAsync(d_ctr, 0, sizeof(int64_t), st));
    PM_TRY(cudaMemsetAsync(d_prod, 0, sizeof(uint64_t) * (size_t)(count * C.prod_stride), st));
    C.ops = d_ops;
    C.nsteps = d_n;
    C.slots = d_slots;
    C.cur = d_cur;
    C.prod = d_prod;
    C.r2 = d_r2;
    C.mod = d_mod;
    // the three product batches: T = x*y, q2 = q1*mu, r2 = m*q3 (q1, q3 windows of T, q2)
    std::vector<ProdIn> in1((size_t)count), in2((size_t)count), in3((size_t)count);
    for (int64_t c = 0; c < count; c++) {
        uint64_t* sl = d_slots + c * C.nslot * k;
        uint64_t* T = d_prod + c * C.prod_stride;
        uint64_t* q2 = d_q2 + c * q2_stride;
        const int64_t l = lmu[(size_t)c];
        in1[(size_t)c] = ProdIn{sl + (int64_t)S.acc() * k, sl + (int64_t)S.one() * k, T, k, k, 64 * k, 64 * k, 0};
        // mu and m are the same on every step: as operand b their transforms
        // are kept from the first run (one-pass products) and reused
        in2[(size_t)c] = ProdIn{T + (k - 1), d_mu + c * lmu_max, q2, k + 1, l, 64 * (k + 1), bits_mu[(size_t)c], 0};
        in3[(size_t)c] = ProdIn{q2 + (k + 1), d_mod + c * k, d_r2 + c * C.r2_stride, l, k, 64 * l, bits_m[(size_t)c], 0};
        in2[(size_t)c].keep_b = one_pass(E, 64 * (k + 1), bits_mu[(size_t)c]);
        in3[(size_t)c].keep_b = one_pass(E, 64 * l, bits_m[(size_t)c]);
    }
    BatchBuild bb[3];
    char* reg[3];
    const std::vector<ProdIn>* ins[3] = {&in1, &in2, &in3};
    for (int i = 0; i < 3; i++) {
        if ((rc = build_batch(E, ins[i]->data(), count, bb[i]))) return rc;
        if ((rc = mem.get(&reg[i], bb[i].dev_bytes))) return rc;
        if ((rc = upload_batch(E, bb[i], reg[i], st))) return rc;
        PM_TRY(expand_jobs(bb[i], reg[i], st));
    }
    C.prods = (DProd*)(reg[0] + bb[0].off_prods);
    PM_TRY(pm_launch_init(C, d_bases, d_lb, st));
    // one run of the q1*mu and q3*m batches stores mu's and m's spectra
    // (PF_BSAVE; their other inputs are zero or already defined here), then
    // every later run loads them (PF_BSPEC)
    for (int i = 1; i < 3; i++) {
        if ((rc = run_launches(E, bb[i], reg[i], st, false))) return rc;
        bool any = false;
        for (DProd& P : bb[i].prods)
            if (P.flags & PF_BSAVE) {
                P.flags = (P.flags & ~PF_BSAVE) | PF_BSPEC;
                any = true;
            }
        if (any)
            PM_TRY(cudaMemcpyAsync(reg[i] + bb[i].off_prods, bb[i].prods.data(), sizeof(DProd) * bb[i].prods.size(),
                                   cudaMemcpyHostToDevice, st));
    }
    PM_TRY(cudaStreamSynchronize(st));  // the host copies above read bb[i].prods
    // one graph of PM_GRAPH_STEPS steps, replayed until every chain is done
    const int64_t G = std::min(PM_GRAPH_STEPS, max_steps);
    PmGraph gr;
    const int64_t l0 = g_launches.load();
    PM_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int crc = 0;
    for (int64_t s = 0; s < G && !crc; s++) {
        if (pm_launch_select(C, d_ctr, st) != cudaSuccess) crc = NBG_ECUDA;
        for (int i = 0; i < 3 && !crc; i++) crc = run_launches(E, bb[i], reg[i], st, false);
        if (!crc && pm_launch_finish(C, st) != cudaSuccess) crc = NBG_ECUDA;
        if (!crc && pm_launch_advance(d_ctr, st) != cudaSuccess) crc = NBG_ECUDA;
    }
    const cudaError_t ce = cudaStreamEndCapture(st, &gr.g);
    if (crc) return crc == NBG_ECUDA ? fail(NBG_ECUDA, "powermod step capture failed") : crc;
    PM_TRY(ce);
    PM_TRY(cudaGraphInstantiate(&gr.x, gr.g, 0));
    for (int64_t done = 0; done < max_steps; done += G) PM_TRY(cudaGraphLaunch(gr.x, st));
    PM_TRY(pm_launch_output(C, d_outs, st));
    PM_TRY(cudaStreamSynchronize(st));
    // launches per replay: the batches' (counted once while capturing) and 3 per step
    const int64_t per_replay = (g_launches.load() - l0) + 3 * G;
    g_launches += ((max_steps + G - 1) / G) * per_replay - (per_replay - 3 * G) + 3 + 2;
    return NBG_OK;
}

}  // namespace nbg

using namespace nbg;

extern "C" {

int64_t nbg_barrett_mu(const uint64_t* m, int64_t k, uint64_t* mu) {
    if (!m || !mu || k < 1 || m[k - 1] == 0) return -(int64_t)fail(NBG_EINVAL, "modulus needs k >= 1 limbs, top limb nonzero");
    std::vector<uint64_t> num((size_t)(2 * k + 1), 0);
    num[(size_t)(2 * k)] = 1;
    std::vector<uint64_t> q((size_t)(k + 2), 0);
    long_divide(num.data(), 2 * k + 1, m, k, q.data());
    memcpy(mu, q.data(), sizeof(uint64_t) * (size_t)(k + 2));
    int64_t l = k + 2;
    while (l > 0 && mu[l - 1] == 0) l--;
    return l;
}

int64_t nbg_powmod_schedule(const uint64_t* e, int64_t le, uint8_t* ops, int64_t cap, int32_t* tsize) {
    if (!e || le < 1 || !tsize) return -(int64_t)fail(NBG_EINVAL, "bad argument");
    std::vector<uint8_t> v;
    int T = 0;
    const int64_t n = schedule(e, le, v, &T);
    if (n < 0) return -(int64_t)fail(NBG_EINVAL, "zero exponent");
    *tsize = T;
    if (ops && cap > 0) memcpy(ops, v.data(), (size_t)std::min(n, cap) * 3);
    return n;
}

static int check_chains(const nbg_powmod_desc* d, int64_t count, int64_t k) {
    if (!d || count < 1 || count > (int64_t)1 << 30 || k < 1) return fail(NBG_EINVAL, "bad chain batch");
    for (int64_t c = 0; c < count; c++)
        if (!d[c].r || !d[c].b || !d[c].e || !d[c].m || d[c].lb < 1 || d[c].lb > k || d[c].le < 1)
            return fail(NBG_EINVAL, "chain %lld: bad descriptor (null pointer, lb outside [1, k] or le < 1)",
                        (long long)c);
    return NBG_OK;
}

static int check_modulus(const std::vector<uint64_t>& m, int64_t c) {
    const int64_t k = (int64_t)m.size();
    if (m[(size_t)(k - 1)] == 0) return fail(NBG_EINVAL, "chain %lld: modulus top limb is zero", (long long)c);
    if (k == 1 && m[0] < 2) return fail(NBG_EINVAL, "chain %lld: modulus must exceed 1", (long long)c);
    return NBG_OK;
}

int nbg_powermod_batch_dev(const nbg_powmod_desc* d, int64_t count, int64_t k, void* stream) {
    int rc = check_chains(d, count, k);
    if (rc) return rc;
    std::lock_guard<std::recursive_mutex> lk(g_eng.mu);
    if ((rc = g_eng.ensure())) return rc;
    cudaStream_t cs = (cudaStream_t)stream;
    PM_TRY(cudaStreamSynchronize(cs));  // inputs written on the caller's stream
    std::vector<std::vector<uint64_t>> hm((size_t)count), he((size_t)count);
    for (int64_t c = 0; c < count; c++) {
        hm[(size_t)c].resize((size_t)k);
        he[(size_t)c].resize((size_t)d[c].le);
        PM_TRY(cudaMemcpy(hm[(size_t)c].data(), d[c].m, sizeof(uint64_t) * (size_t)k, cudaMemcpyDeviceToHost));
        PM_TRY(cudaMemcpy(he[(size_t)c].data(), d[c].e, sizeof(uint64_t) * (size_t)d[c].le, cudaMemcpyDeviceToHost));
        if ((rc = check_modulus(hm[(size_t)c], c))) return rc;
    }
    return powmod_run(g_eng, d, count, k, hm, he);
}

int nbg_powermod_batch(const nbg_powmod_desc* d, int64_t count, int64_t k) {
    int rc = check_chains(d, count, k);
    if (rc) return rc;
    std::lock_guard<std::recursive_mutex> lk(g_eng.mu);
    if ((rc = g_eng.ensure())) return rc;
    std::vector<std::vector<uint64_t>> hm((size_t)count), he((size_t)count);
    for (int64_t c = 0; c < count; c++) {
        hm[(size_t)c].assign(d[c].m, d[c].m + k);
        he[(size_t)c].assign(d[c].e, d[c].e + d[c].le);
        if ((rc = check_modulus(hm[(size_t)c], c))) return rc;
    }
    // device copies of the bases; results come back into the caller's buffers
    PmMem mem;
    uint64_t *db = nullptr, *dr = nullptr;
    if ((rc = mem.get(&db, (size_t)(count * k))) || (rc = mem.get(&dr, (size_t)(count * k)))) return rc;
    std::vector<nbg_powmod_desc> dd(d, d + count);
    for (int64_t c = 0; c < count; c++) {
        PM_TRY(cudaMemcpyAsync(db + c * k, d[c].b, sizeof(uint64_t) * (size_t)d[c].lb, cudaMemcpyHostToDevice,
                               g_eng.stream));
        dd[(size_t)c].b = db + c * k;
        dd[(size_t)c].r = dr + c * k;
    }
    if ((rc = powmod_run(g_eng, dd.data(), count, k, hm, he))) return rc;
    for (int64_t c = 0; c < count; c++)
        PM_TRY(cudaMemcpy(d[c].r, dr + c * k, sizeof(uint64_t) * (size_t)k, cudaMemcpyDeviceToHost));
    return NBG_OK;
}

}  // extern "C"
