// linalg.cu — sums of products on the GPU for the reference's HGCD callers:
// the 2x2 matrix product M <- M * M1 (hgcd_matrix_mul!, src/gcd.jl:371-389,
// eight independent mul! plus four additions) and the cofactor update
// r = a*x + b*y (cof_mul2!, src/gcd.jl:571-598).  The products of a call run
// as one fp-NTT batch; the additions are a tile-parallel carry-lookahead sum:
// each CTA adds a 1024-limb tile of the two terms and records whether the
// tile generates or propagates a carry, then one CTA per output scans the
// tiles' (generate, propagate) pairs and adds the incoming carries.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/nbgpu.h"
#include "engine.h"

namespace nbg {

constexpr int SUM_TL = 1024;     // limbs per tile
constexpr int SUM_THREADS = 256;  // 4 limbs per thread

// One sum: r[0..rn) = x[0..nx) + y[0..ny) (missing limbs zero); agg holds one
// (generate | propagate << 1) pair per tile.
struct SumJob {
    uint64_t* r;
    const uint64_t* x;
    const uint64_t* y;
    int64_t rn, nx, ny;
    uint32_t* agg;
    int64_t ntl;
    int64_t tile0;  // first global tile index of this sum
};

__device__ __forceinline__ uint32_t sum_gp(uint32_t lower, uint32_t upper) {
    const uint32_t g = (upper & 1u) | ((upper >> 1) & lower & 1u);
    const uint32_t p = (upper >> 1) & (lower >> 1) & 1u;
    return g | (p << 1);
}

// tile t of the launch -> its sum (binary search over tile0)
__device__ __forceinline__ int sum_of_tile(const SumJob* jobs, int njobs, int64_t t) {
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].tile0 <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(SUM_THREADS) k_sum_tiles(const SumJob* __restrict__ jobs, int njobs) {
    __shared__ uint32_t wagg[SUM_THREADS / 32];
    __shared__ uint32_t carry_in[SUM_THREADS / 32];
    const int64_t t = blockIdx.x;
    const SumJob J = jobs[sum_of_tile(jobs, njobs, t)];
    const int64_t tl = t - J.tile0;
    const int64_t w0 = tl * SUM_TL + 4 * (int64_t)threadIdx.x;
    uint64_t s[4];
    uint32_t ov = 0;        // bit q: a + b overflowed at limb q
    uint32_t g = 0, p = 1;  // this thread's 4 limbs: carry out with carry in 0 / propagate
    for (int q = 0; q < 4; q++) {
        const int64_t w = w0 + q;
        const uint64_t a = w < J.nx && w < J.rn ? J.x[w] : 0;
        const uint64_t b = w < J.ny && w < J.rn ? J.y[w] : 0;
        s[q] = a + b;
        const uint32_t gq = s[q] < a;        // this limb generates
        ov |= gq << q;
        const uint32_t pq = s[q] == ~0ULL;   // passes a carry on
        const uint32_t ng = gq | (pq & g), np = pq & p;
        g = ng;
        p = np;
    }
    // block scan of (g, p): inclusive within warps, then across warps
    uint32_t mine = g | (p << 1);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t incl = mine;
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl = sum_gp(o, incl);
    }
    if (lane == 31) wagg[wid] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 2u;  // identity: propagate, no generate
        for (int k = 0; k < SUM_THREADS / 32; k++) {
            carry_in[k] = run & 1u;
            run = sum_gp(run, wagg[k]);
        }
        J.agg[tl] = run;
    }
    __syncthreads();
    uint32_t excl = __shfl_up_sync(0xffffffffu, incl, 1);
    if (lane == 0) excl = 2u;
    // carry into this thread from the warps below and the lanes below
    uint32_t c = (excl & 1u) | ((excl >> 1) & carry_in[wid]);
    for (int q = 0; q < 4; q++) {
        const int64_t w = w0 + q;
        const uint64_t v = s[q] + c;
        c = ((ov >> q) & 1u) | (v < s[q] ? 1u : 0u);  // a + b overflowed, or the carry rippled through
        if (w < J.rn) J.r[w] = v;
    }
}

// One CTA per sum: carries between tiles (the tile sums above assumed carry-in 0).
__global__ void __launch_bounds__(256) k_sum_carry(const SumJob* __restrict__ jobs) {
    __shared__ uint32_t wagg[8];
    const SumJob J = jobs[blockIdx.x];
    const int64_t nt = J.ntl;
    if (nt <= 1) return;
    const int t = threadIdx.x;
    const int64_t per = (nt + blockDim.x - 1) / blockDim.x;
    const int64_t t0 = (int64_t)t * per, t1 = min(t0 + per, nt);
    uint32_t agg = 2u;
    for (int64_t k = t0; k < t1; k++) agg = sum_gp(agg, J.agg[k]);
    const int lane = t & 31, wid = t >> 5;
    uint32_t incl = agg;
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl = sum_gp(o, incl);
    }
    if (lane == 31) wagg[wid] = incl;
    __syncthreads();
    uint32_t wpre = 2u;
    for (int k = 0; k < wid; k++) wpre = sum_gp(wpre, wagg[k]);
    uint32_t excl = __shfl_up_sync(0xffffffffu, incl, 1);
    if (lane == 0) excl = 2u;
    excl = sum_gp(wpre, excl);
    uint32_t cin = excl & 1u;
    for (int64_t k = t0; k < t1; k++) {
        const uint32_t a = J.agg[k];
        if (cin) {
            int64_t w = k * SUM_TL;
            const int64_t we = min(w + (int64_t)SUM_TL, J.rn);
            while (w < we && J.r[w] == ~0ULL) {
                J.r[w] = 0;
                w++;
            }
            if (w < we) J.r[w] += 1;
        }
        cin = (a & 1u) | ((a >> 1) & cin);
    }
}

}  // namespace nbg

namespace nbg {

// Magnitude bits of each buffer (0 for an all-zero buffer): one CTA per buffer.
__global__ void __launch_bounds__(256) k_magbits(const uint64_t* const* __restrict__ bufs,
                                                 const int64_t* __restrict__ lens, int64_t* __restrict__ bits) {
    __shared__ int64_t best[8];
    const uint64_t* x = bufs[blockIdx.x];
    const int64_t n = lens[blockIdx.x];
    int64_t top = -1;  // highest nonzero limb this thread saw
    for (int64_t w = threadIdx.x; w < n; w += blockDim.x)
        if (x[w]) top = w;
    for (int off = 16; off; off >>= 1) top = max(top, (int64_t)__shfl_xor_sync(0xffffffffu, top, off));
    if ((threadIdx.x & 31) == 0) best[threadIdx.x >> 5] = top;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < 8; k++) top = max(top, best[k]);
        bits[blockIdx.x] = top < 0 ? 0 : 64 * top + 64 - __clzll((long long)x[top]);
    }
}

// Radix combine, first level: node i = value of the base-bb chunks
// c[32i .. 32i+31] (chunks past n read as zero) by Horner's rule, one thread
// per node, into out[32i .. 32i+31] (the value is below bb^32 < 2^2048).
__global__ void __launch_bounds__(128) k_horner32(const uint64_t* __restrict__ c, int64_t n, uint64_t bb,
                                                  uint64_t* __restrict__ out, int64_t nodes) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nodes) return;
    uint64_t* v = out + 32 * i;
    for (int w = 0; w < 32; w++) v[w] = 0;
    int len = 0;  // limbs of v in use
    for (int j = 31; j >= 0; j--) {
        const int64_t idx = 32 * i + j;
        uint64_t carry = idx < n ? c[idx] : 0;  // v = v * bb + c_j
        for (int w = 0; w < len; w++) {
            const unsigned __int128 t = (unsigned __int128)v[w] * bb + carry;
            v[w] = (uint64_t)t;
            carry = (uint64_t)(t >> 64);
        }
        if (carry && len < 32) v[len++] = carry;
    }
}

}  // namespace nbg

using namespace nbg;

namespace {

#define LA_TRY(x)                                                                            \
    do {                                                                                     \
        cudaError_t e_ = (x);                                                                \
        if (e_ != cudaSuccess) return fail(NBG_ECUDA, "%s: %s", #x, cudaGetErrorString(e_)); \
    } while (0)

// out[k] = Σ over terms t with owner[t] == k of a_t * b_t, plus addend[k]
// when given (device buffers, nonnegative), out[k] holding outlen[k] limbs.
// At most two summands per output.
int sum_products(const std::vector<nbg_desc>& terms, const std::vector<int>& owner,
                 const std::vector<uint64_t*>& out, const std::vector<int64_t>& outlen, cudaStream_t st,
                 const std::vector<std::pair<const uint64_t*, int64_t>>* addend = nullptr) {
    const int nt = (int)terms.size(), no = (int)out.size();
    // magnitude bits of every operand, read on the device
    std::vector<const uint64_t*> bufs(2 * (size_t)nt);
    std::vector<int64_t> lens(2 * (size_t)nt), bits(2 * (size_t)nt);
    for (int t = 0; t < nt; t++) {
        bufs[2 * t] = terms[t].a;
        lens[2 * t] = terms[t].m;
        bufs[2 * t + 1] = terms[t].b;
        lens[2 * t + 1] = terms[t].n;
    }
    size_t prod_limbs = 0;
    for (const nbg_desc& d : terms) prod_limbs += (size_t)(d.m + d.n);
    size_t tiles = 0;
    for (int k = 0; k < no; k++) tiles += (size_t)((outlen[k] + SUM_TL - 1) / SUM_TL);
    const size_t off_bufs = 0, off_lens = off_bufs + 16 * (size_t)nt, off_bits = off_lens + 16 * (size_t)nt;
    const size_t off_jobs = (off_bits + 16 * (size_t)nt + 255) / 256 * 256;
    const size_t off_agg = (off_jobs + sizeof(SumJob) * (size_t)no + 255) / 256 * 256;
    const size_t off_prod = (off_agg + 4 * tiles + 255) / 256 * 256;
    const size_t bytes = off_prod + 8 * prod_limbs;
    char* d = nullptr;
    LA_TRY(cudaMallocAsync((void**)&d, bytes, st));
    struct Free {
        char* p;
        cudaStream_t s;
        ~Free() { cudaFreeAsync(p, s); }
    } guard{d, st};
    if (nt > 0) {
        LA_TRY(cudaMemcpyAsync(d + off_bufs, bufs.data(), 8 * bufs.size(), cudaMemcpyHostToDevice, st));
        LA_TRY(cudaMemcpyAsync(d + off_lens, lens.data(), 8 * lens.size(), cudaMemcpyHostToDevice, st));
        k_magbits<<<(unsigned)(2 * nt), 256, 0, st>>>((const uint64_t* const*)(d + off_bufs),
                                                       (const int64_t*)(d + off_lens), (int64_t*)(d + off_bits));
        LA_TRY(cudaGetLastError());
        LA_TRY(cudaMemcpyAsync(bits.data(), d + off_bits, 8 * bits.size(), cudaMemcpyDeviceToHost, st));
        LA_TRY(cudaStreamSynchronize(st));
    }
    // nonzero products into the scratch; zero ones drop out of their sums
    std::vector<nbg_desc> live;
    std::vector<const uint64_t*> prod_of((size_t)nt, nullptr);
    std::vector<int64_t> prod_len((size_t)nt, 0);
    uint64_t* pbase = (uint64_t*)(d + off_prod);
    size_t po = 0;
    for (int t = 0; t < nt; t++) {
        const nbg_desc& x = terms[t];
        if (bits[2 * t] && bits[2 * t + 1]) {
            const int64_t la = (bits[2 * t] + 63) / 64, lb = (bits[2 * t + 1] + 63) / 64;
            nbg_desc q{pbase + po, x.a, x.b, la, lb, bits[2 * t], bits[2 * t + 1]};
            live.push_back(q);
            prod_of[(size_t)t] = pbase + po;
            prod_len[(size_t)t] = la + lb;
            po += (size_t)(la + lb);
        }
    }
    if (!live.empty()) {
        int rc = nbg_mul_batch_dev(live.data(), (int64_t)live.size(), st);
        if (rc) return rc;
    }
    // the sums
    std::vector<SumJob> jobs((size_t)no);
    int64_t tile0 = 0;
    uint32_t* agg = (uint32_t*)(d + off_agg);
    for (int k = 0; k < no; k++) {
        SumJob& J = jobs[(size_t)k];
        J.r = out[(size_t)k];
        J.rn = outlen[(size_t)k];
        J.x = nullptr;
        J.y = nullptr;
        J.nx = J.ny = 0;
        for (int t = 0; t < nt; t++) {
            if (owner[(size_t)t] != k || !prod_of[(size_t)t]) continue;
            if (!J.x) {
                J.x = prod_of[(size_t)t];
                J.nx = prod_len[(size_t)t];
            } else {
                J.y = prod_of[(size_t)t];
                J.ny = prod_len[(size_t)t];
            }
        }
        if (addend && (*addend)[(size_t)k].first) {
            const auto& ad = (*addend)[(size_t)k];
            if (!J.x) {
                J.x = ad.first;
                J.nx = ad.second;
            } else {
                J.y = ad.first;
                J.ny = ad.second;
            }
        }
        J.ntl = (J.rn + SUM_TL - 1) / SUM_TL;
        J.agg = agg + tile0;
        J.tile0 = tile0;
        tile0 += J.ntl;
    }
    LA_TRY(cudaMemcpyAsync(d + off_jobs, jobs.data(), sizeof(SumJob) * jobs.size(), cudaMemcpyHostToDevice, st));
    if (tile0 > 0) {
        k_sum_tiles<<<(unsigned)tile0, SUM_THREADS, 0, st>>>((const SumJob*)(d + off_jobs), no);
        LA_TRY(cudaGetLastError());
        k_sum_carry<<<(unsigned)no, 256, 0, st>>>((const SumJob*)(d + off_jobs));
        LA_TRY(cudaGetLastError());
        g_launches += 3;
    }
    // the host vectors above are read by the copies: wait before they go
    LA_TRY(cudaStreamSynchronize(st));
    return NBG_OK;
}

}  // namespace

extern "C" {

int nbg_matrix22_mul_dev(uint64_t* const* m, int64_t n, const uint64_t* const* m1, int64_t n1, void* stream) {
    if (!m || !m1 || n < 1 || n1 < 1) return fail(NBG_EINVAL, "bad argument");
    for (int i = 0; i < 4; i++)
        if (!m[i] || !m1[i]) return fail(NBG_EINVAL, "null matrix entry");
    cudaStream_t st = (cudaStream_t)stream;
    // rows (m00, m01) and (m10, m11) times the columns of M1 (hgcd_matrix_mul!)
    std::vector<nbg_desc> terms;
    std::vector<int> owner;
    for (int row = 0; row < 2; row++)
        for (int col = 0; col < 2; col++)
            for (int j = 0; j < 2; j++) {
                terms.push_back(nbg_desc{nullptr, m[2 * row + j], m1[2 * j + col], n, n1, 0, 0});
                owner.push_back(2 * row + col);
            }
    std::vector<uint64_t*> out(m, m + 4);
    std::vector<int64_t> outlen(4, n + n1 + 1);
    return sum_products(terms, owner, out, outlen, st);
}

int nbg_mul2add_dev(uint64_t* r, int64_t rn, const uint64_t* a, int64_t la, const uint64_t* x, int64_t lx,
                    const uint64_t* b, int64_t lb, const uint64_t* y, int64_t ly, void* stream) {
    if (!r || !a || !x || !b || !y || la < 1 || lx < 1 || lb < 1 || ly < 1 ||
        rn < std::max(la + lx, lb + ly) + 1)
        return fail(NBG_EINVAL, "bad argument (r needs max(la+lx, lb+ly)+1 limbs)");
    std::vector<nbg_desc> terms{nbg_desc{nullptr, a, x, la, lx, 0, 0}, nbg_desc{nullptr, b, y, lb, ly, 0, 0}};
    return sum_products(terms, std::vector<int>{0, 0}, std::vector<uint64_t*>{r}, std::vector<int64_t>{rn},
                        (cudaStream_t)stream);
}

}  // extern "C"

namespace {

// bb^32 on the host (32 limbs), the first entry of the power table.
void pow32(uint64_t bb, uint64_t* p) {
    memset(p, 0, 32 * sizeof(uint64_t));
    p[0] = 1;
    for (int k = 0; k < 32; k++) {
        uint64_t carry = 0;
        for (int w = 0; w < 32; w++) {
            const unsigned __int128 t = (unsigned __int128)p[w] * bb + carry;
            p[w] = (uint64_t)t;
            carry = (uint64_t)(t >> 64);
        }
    }
}

// Value of the little-endian base-bb chunks c[0..n) (device) into the device
// buffer *res (*res_limbs limbs, zero-padded): radix_combine of the reference
// (src/nbig.jl:410-417) level by level.  Level 5 (32 chunks per node) is one
// Horner kernel; every higher level is one batch of products high * bb^(2^(l-1))
// plus the low halves, the power table built by repeated GPU squaring as the
// reference's radix_chunks_dc builds it (src/nbig.jl:396-399).
int radix_combine_run(const uint64_t* d_c, int64_t n, uint64_t bb, std::vector<void*>& keep, uint64_t** res,
                      int64_t* res_limbs, cudaStream_t st) {
    int64_t M = 1;
    while (M < (n + 31) / 32) M <<= 1;
    const int64_t total = 32 * M;
    uint64_t *A = nullptr, *Bf = nullptr, *P = nullptr;
    LA_TRY(cudaMalloc((void**)&A, 8 * (size_t)total));
    keep.push_back(A);
    LA_TRY(cudaMalloc((void**)&Bf, 8 * (size_t)total));
    keep.push_back(Bf);
    LA_TRY(cudaMemsetAsync(A, 0, 8 * (size_t)total, st));
    const int64_t nodes5 = (n + 31) / 32;
    k_horner32<<<(unsigned)((nodes5 + 127) / 128), 128, 0, st>>>(d_c, n, bb, A, nodes5);
    LA_TRY(cudaGetLastError());
    g_launches++;
    // P = bb^32, squared up the levels
    int64_t plen = 32;
    LA_TRY(cudaMalloc((void**)&P, 8 * 32));
    keep.push_back(P);
    {
        uint64_t h[32];
        pow32(bb, h);
        LA_TRY(cudaMemcpyAsync(P, h, sizeof h, cudaMemcpyHostToDevice, st));
        LA_TRY(cudaStreamSynchronize(st));
    }
    uint64_t *in = A, *out = Bf;
    for (int64_t s = 64; s <= total; s *= 2) {  // node size of the level being formed
        const int64_t half = s / 2, count = total / s;
        std::vector<nbg_desc> terms((size_t)count);
        std::vector<int> owner((size_t)count);
        std::vector<uint64_t*> outs((size_t)count);
        std::vector<int64_t> outlen((size_t)count, s);
        std::vector<std::pair<const uint64_t*, int64_t>> add((size_t)count);
        for (int64_t i = 0; i < count; i++) {
            terms[(size_t)i] = nbg_desc{nullptr, in + (2 * i + 1) * half, P, half, plen, 0, 0};
            owner[(size_t)i] = (int)i;
            outs[(size_t)i] = out + i * s;
            add[(size_t)i] = {in + 2 * i * half, half};
        }
        int rc = sum_products(terms, owner, outs, outlen, st, &add);
        if (rc) return rc;
        std::swap(in, out);
        if (2 * s <= total) {  // next power: P^2
            uint64_t* P2 = nullptr;
            LA_TRY(cudaMalloc((void**)&P2, 8 * (size_t)(2 * plen)));
            keep.push_back(P2);
            rc = nbg_sqr_dev(P2, P, plen, st);
            if (rc) return rc;
            P = P2;
            plen *= 2;
        }
    }
    *res = in;
    *res_limbs = total;
    return NBG_OK;
}

}  // namespace

extern "C" int nbg_radix_combine(uint64_t* out, int64_t cap, const uint64_t* chunks, int64_t n, uint64_t bb,
                                 int64_t* out_len) {
    if (!out || !chunks || !out_len || n < 1 || bb < 2 || cap < n) return fail(NBG_EINVAL, "bad argument");
    for (int64_t i = 0; i < n; i++)
        if (chunks[i] >= bb) return fail(NBG_EINVAL, "chunk %lld is not below the base", (long long)i);
    std::lock_guard<std::recursive_mutex> lk(g_eng.mu);
    int rc = g_eng.ensure();
    if (rc) return rc;
    cudaStream_t st = g_eng.stream;
    std::vector<void*> keep;
    struct Free {
        std::vector<void*>& k;
        ~Free() {
            for (void* p : k) cudaFree(p);
        }
    } guard{keep};
    uint64_t* dc = nullptr;
    LA_TRY(cudaMalloc((void**)&dc, 8 * (size_t)n));
    keep.push_back(dc);
    LA_TRY(cudaMemcpyAsync(dc, chunks, 8 * (size_t)n, cudaMemcpyHostToDevice, st));
    uint64_t* res = nullptr;
    int64_t rl = 0;
    if ((rc = radix_combine_run(dc, n, bb, keep, &res, &rl, st))) return rc;
    // the value is below bb^n < 2^(64n): its limbs are within the first n
    LA_TRY(cudaMemcpyAsync(out, res, 8 * (size_t)n, cudaMemcpyDeviceToHost, st));
    LA_TRY(cudaStreamSynchronize(st));
    int64_t l = n;
    while (l > 0 && out[l - 1] == 0) l--;
    *out_len = l;
    return NBG_OK;
}

// The power table of radix_chunks_dc (src/nbig.jl:394-399): powtab[1] = bb,
// powtab[i+1] = powtab[i]^2, extended while its last entry is <= x.  Every
// square runs on the GPU with the chain kept on the device; each new entry's
// top limb comes back to trim it to its normalized length and to decide
// whether the table goes on.
extern "C" int nbg_radix_powtab(uint64_t* out, int64_t cap, int64_t* offsets, int32_t max_entries, uint64_t bb,
                                const uint64_t* x, int64_t xn, int32_t* entries) {
    if (!out || !offsets || !entries || !x || xn < 1 || bb < 2 || max_entries < 1 || cap < 1)
        return fail(NBG_EINVAL, "bad argument");
    while (xn > 1 && x[xn - 1] == 0) xn--;
    std::lock_guard<std::recursive_mutex> lk(g_eng.mu);
    int rc = g_eng.ensure();
    if (rc) return rc;
    cudaStream_t st = g_eng.stream;
    std::vector<void*> keep;
    struct Free {
        std::vector<void*>& k;
        ~Free() {
            for (void* p : k) cudaFree(p);
        }
    } guard{keep};
    // is the n-limb value p (host copy) <= x?
    auto le_x = [&](const uint64_t* p, int64_t n) {
        if (n != xn) return n < xn;
        for (int64_t i = n - 1; i >= 0; i--)
            if (p[i] != x[i]) return p[i] < x[i];
        return true;
    };
    int32_t ne = 0;
    int64_t used = 0;
    // entry 1: bb itself
    out[0] = bb;
    offsets[0] = 0;
    used = 1;
    ne = 1;
    uint64_t* dprev = nullptr;
    int64_t plen = 1;
    LA_TRY(cudaMalloc((void**)&dprev, 8));
    keep.push_back(dprev);
    LA_TRY(cudaMemcpyAsync(dprev, &bb, 8, cudaMemcpyHostToDevice, st));
    bool more = le_x(out, 1);
    while (more) {
        if (ne >= max_entries) return fail(NBG_EINVAL, "power table needs more than %d entries", (int)max_entries);
        uint64_t* dnext = nullptr;
        LA_TRY(cudaMalloc((void**)&dnext, 8 * (size_t)(2 * plen)));
        keep.push_back(dnext);
        if ((rc = nbg_sqr_dev(dnext, dprev, plen, st))) return rc;
        int64_t nl = 2 * plen;
        uint64_t top = 0;
        LA_TRY(cudaMemcpyAsync(&top, dnext + nl - 1, 8, cudaMemcpyDeviceToHost, st));
        LA_TRY(cudaStreamSynchronize(st));
        if (top == 0) nl--;  // a square of a normalized value has 2n or 2n-1 limbs
        if (used + nl > cap) return fail(NBG_EINVAL, "output needs more than %lld limbs", (long long)cap);
        LA_TRY(cudaMemcpyAsync(out + used, dnext, 8 * (size_t)nl, cudaMemcpyDeviceToHost, st));
        LA_TRY(cudaStreamSynchronize(st));
        offsets[ne] = used;
        more = le_x(out + used, nl);
        used += nl;
        ne++;
        dprev = dnext;
        plen = nl;
    }
    offsets[ne] = used;
    *entries = ne;
    return NBG_OK;
}
