// kernels.cu — the fp-NTT product pipeline on sm_100a FP64 cores.
//
// Kernels (each is a work-queue launch: CTA i takes Job i of a host-built list
// that may mix products of any size; pass kernels hold both primes' tiles):
//   k_fwd     forward pass of one tile; pass 0 packs limbs into b-bit chunks
//             on load (fp_ntt_pack!, src/fpntt.jl:744-768)
//   k_pwr     last pass: forward stages, pointwise product
//             (fp_ntt_pointwise!, :770-785) and the reverse's first stages on
//             the same shared-memory block; packs on load for one-pass products
//   k_rev     reverse pass of one tile (fp_ntt_rev!, :727-733)
//   k_unpack  Garner CRT (fp_unpack_coeff, :806-816) and limb assembly of a
//             1024-limb output tile with a block-wide carry-lookahead scan;
//             persistent CTAs stage the next tile's residues by bulk copy
//             while assembling the current one
//   k_carry   cross-tile carry scan and fix-up, one CTA per product
//   k_queue   a whole batch in one persistent launch: CTAs claim jobs from a
//             queue in pipeline-step order and wait, per product, for the
//             previous step's jobs (the per-kind kernels above run the same
//             job functions)
//   k_twiddle expands exact minimal-balanced twiddle tables from two small
//             power tables (twiddle values are unique residues, so any exact
//             construction equals fp_twiddles, :173-186)
//
// Within a pass the stages run as rounds (types.h RoundKind): radix-16 rounds
// hold 16 points per work unit in registers and apply two radix-4 stages
// between one shared-memory load and store; radix-8 rounds do the span-8
// radix-4 stage and the final radix-2; odd stages run one butterfly per unit.
// Every butterfly is the reference's butterfly on the reference's inputs, so
// the grouping changes no bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>

#include "butterfly.cuh"
#include "kernels.h"

// Minimum resident CTAs per SM the pass kernels are compiled for (register
// budget 65536 / (256 * minb) = 80 at 3).  Measured on B200 with the mixed
// 10,000-product batch: 3 CTAs/SM beats 2 by 10% (column passes by 20%)
// despite a few spills; 1 CTA/SM is 35% slower.
#ifndef NBG_PWR_MINB
#define NBG_PWR_MINB 3
#endif
// Column passes with tile sets up to this size run the 4-CTA/SM build.
constexpr size_t COL4_MAX_SMEM = 32 * 1024;
constexpr size_t COL4_MAX_SMEM_TMA = 32 * 1024 + 128;  // the TMA tiles plus their mbarrier line
// Rounds are inlined into the kernels; out-of-line rounds (NBG_ROUND_NOINLINE)
// measured 40% slower in k_pwr.
#ifdef NBG_ROUND_NOINLINE
#define NBG_ROUND __noinline__
#else
#define NBG_ROUND
#endif

namespace nbg {

__constant__ Fp c_fp[2];
__constant__ double c_garner[2];  // g = p1^-1 mod p2 (canonical) and g/p2

__device__ __forceinline__ Fp fpctx(int f) { return c_fp[f]; }

__device__ __forceinline__ int sp(int i) { return tile_pad_index(i); }
// tile layouts: padded (one double in 16, the cp.async tiles) or dense (the
// boxes TMA writes; column tiles with at least 16 columns, conflict-free)
template <bool PAD>
__device__ __forceinline__ int lay(int i) {
    return PAD ? tile_pad_index(i) : i;
}

// exact double of an integer below 2^52: OR it into 2^52's mantissa, subtract 2^52
__device__ __forceinline__ double small_u64_to_double(uint64_t c) {
    return __dsub_rn(__longlong_as_double((long long)(c | 0x4330000000000000ULL)), 4503599627370496.0);
}

// ---------------------------------------------------------------------------
// Pack: chunk i of an n-limb operand (fp_ntt_pack!, :744-768).  The
// reference's fast loop always ORs in the next limb; its high bits are masked
// off unless sh + b > 64, so this single form is identical.
__device__ __forceinline__ double pack_chunk(const uint64_t* __restrict__ limbs, int64_t n, int b, int64_t nch,
                                             int64_t i) {
    if (i >= nch) return 0.0;
    const uint64_t bit = (uint64_t)i * (uint32_t)b;
    const int64_t w = (int64_t)(bit >> 6);
    const int sh = (int)(bit & 63);
    uint64_t c = __ldg(limbs + w) >> sh;
    if (sh + b > 64 && w + 1 < n) c |= __ldg(limbs + w + 1) << (64 - sh);
    return small_u64_to_double(c & ((1ULL << b) - 1ULL));
}

// ---------------------------------------------------------------------------
// Tiles resident in shared memory: `ntiles` tiles of G rows x C columns
// (padded layout, row stride C), `stride` doubles apart; tile t belongs to
// prime t >> pshift.  Column c of a tile is global column j0 + c of the pass.
struct Tiles {
    double* s;
    int stride;
    int ntiles;
    int pshift;
    int G;
    int lc;   // log2 C
    int Qb;   // pass column stride (global)
    int j0;   // first global column of the tile
    int pfix; // -1: tile t is prime t >> pshift; 0 or 1: every tile is that prime
};

// unit u of a round over all tiles -> (tile, unit within tile)
__device__ __forceinline__ int split_unit(int u, int per, int& tau) {
    tau = 0;
    while (u >= per) {
        u -= per;
        tau++;
    }
    return u;
}

// Generic stage: one butterfly per unit, any radix (odd stages, lone radix-4/2).
template <int M, bool FWD, bool PAD>
__device__ NBG_ROUND void round_gen(const Tiles& T, const DStage& st) {
    const int C = 1 << T.lc;
    const int Lloc = (int)(st.L / T.Qb), Qloc = (int)(st.Q / T.Qb);
    // twiddle offsets stay below N <= 2^32: 32-bit unsigned arithmetic
    const uint32_t Q = (uint32_t)st.Q;
    const int per = (T.G / M) << T.lc;
    const int total = per * T.ntiles;
    // row / Qloc = (row >> e) / odd, odd by multiply-high (exact for rows < 2^32 / odd)
    const int e = __ffs(Qloc) - 1;
    const unsigned odd = (unsigned)(Qloc >> e);
    const unsigned mg = odd == 1 ? 0u : 0xFFFFFFFFu / odd + 1u;
    const int stride = Qloc << T.lc;
    // per-prime constants, loaded once per round
    const Fp F0 = fpctx(0), F1 = fpctx(1);
    const double* tw0 = st.tw[0];
    const double* tw1 = st.tw[1];
    for (int u = threadIdx.x; u < total; u += blockDim.x) {
        int tau;
        const int uu = split_unit(u, per, tau);
        const bool p1 = T.pfix >= 0 ? T.pfix == 1 : (tau >> T.pshift) != 0;
        const Fp F = p1 ? F1 : F0;
        double* s = T.s + tau * T.stride;
        const int c = uu & (C - 1);
        const int row = uu >> T.lc;
        const unsigned rs = (unsigned)row >> e;
        const int blk = odd == 1 ? (int)rs : (int)__umulhi(rs, mg);
        const int jl = row - blk * Qloc;
        const int base = ((blk * Lloc + jl) << T.lc) + c;
        double y[M];
#pragma unroll
        for (int t = 0; t < M; t++) y[t] = s[lay<PAD>(base + t * stride)];
        if constexpr (M == 2) {
            butterfly2(y[0], y[1], F);
        } else {
            const int j = jl * T.Qb + T.j0 + c;
            const double* tw = (p1 ? tw1 : tw0) + j;
            double w[M];
            w[0] = 0.0;
#pragma unroll
            for (int t = 1; t < M; t++) w[t] = __ldg(tw + (t - 1) * Q);
            constexpr int NR = M == 3 ? 1 : (M == 5 ? 4 : (M == 4 ? 1 : 8));
            double rot[8];
            const double* rp = st.rot[p1 ? 1 : 0];
#pragma unroll
            for (int t = 0; t < NR; t++) rot[t] = rp[t];
            butterfly<M, FWD>(y, w, rot, F);
        }
#pragma unroll
        for (int t = 0; t < M; t++) s[lay<PAD>(base + t * stride)] = y[t];
    }
}

// Radix-16 round: stages A (span L) and B (span L/4), both radix-4.  Unit
// (block b, j2 < L/16 rows, column c) holds rows b*L + j2 + t1*L/4 + t2*L/16.
// Forward: A's butterflies run over t1 for each t2 (column j2 + t2*L/16), then
// B's over t2 for each t1 (column j2).  Reverse: B then A, transposed.
template <bool FWD, bool PAD>
__device__ NBG_ROUND void round_r16(const Tiles& T, const DStage& A, const DStage& B) {
    const int C = 1 << T.lc;
    const int Lloc = (int)(A.L / T.Qb);
    const int q16 = Lloc >> 4, lq = __ffs(q16) - 1;
    // twiddle offsets (t2 * stepA + 2 * QA < L_A <= N <= 2^32): 32-bit unsigned
    const uint32_t QA = (uint32_t)A.Q, QB = (uint32_t)B.Q;
    const int per = (T.G >> 4) << T.lc;
    const int total = per * T.ntiles;
    const double wi0 = A.rot[0][0], wi1 = A.rot[1][0];  // the same 4th root for every radix-4 stage
    const double *twA0 = A.tw[0], *twA1 = A.tw[1], *twB0 = B.tw[0], *twB1 = B.tw[1];
    for (int u = threadIdx.x; u < total; u += blockDim.x) {
        int tau;
        const int uu = split_unit(u, per, tau);
        const bool p1 = T.pfix >= 0 ? T.pfix == 1 : (tau >> T.pshift) != 0;
        const Fp F = fpctx(p1 ? 1 : 0);
        const double wi = p1 ? wi1 : wi0;
        double* s = T.s + tau * T.stride;
        const int c = uu & (C - 1);
        const int r = uu >> T.lc;
        const int b = r >> lq, j2 = r & (q16 - 1);
        const int row0 = b * Lloc + j2;
        double v[16];
#pragma unroll
        for (int t1 = 0; t1 < 4; t1++)
#pragma unroll
            for (int t2 = 0; t2 < 4; t2++) v[t1 * 4 + t2] = s[lay<PAD>(((row0 + t1 * 4 * q16 + t2 * q16) << T.lc) + c)];
        const int jB = j2 * T.Qb + T.j0 + c;
        const double* twB = (p1 ? twB1 : twB0) + jB;
        const double* twA = (p1 ? twA1 : twA0) + jB;  // A's column for t2 is jB + t2*q16*Qb
        const uint32_t stepA = (uint32_t)q16 * (uint32_t)T.Qb;
        if (FWD) {
#pragma unroll
            for (int t2 = 0; t2 < 4; t2++) {
                double y[4] = {v[t2], v[4 + t2], v[8 + t2], v[12 + t2]};
                double w[4] = {0.0, __ldg(twA + t2 * stepA), __ldg(twA + t2 * stepA + QA),
                               __ldg(twA + t2 * stepA + 2 * QA)};
                butterfly<4, true>(y, w, &wi, F);
                v[t2] = y[0]; v[4 + t2] = y[1]; v[8 + t2] = y[2]; v[12 + t2] = y[3];
            }
            const double w[4] = {0.0, __ldg(twB), __ldg(twB + QB), __ldg(twB + 2 * QB)};
#pragma unroll
            for (int t1 = 0; t1 < 4; t1++) butterfly<4, true>(v + 4 * t1, w, &wi, F);
        } else {
            const double w[4] = {0.0, __ldg(twB), __ldg(twB + QB), __ldg(twB + 2 * QB)};
#pragma unroll
            for (int t1 = 0; t1 < 4; t1++) butterfly<4, false>(v + 4 * t1, w, &wi, F);
#pragma unroll
            for (int t2 = 0; t2 < 4; t2++) {
                double y[4] = {v[t2], v[4 + t2], v[8 + t2], v[12 + t2]};
                double wa[4] = {0.0, __ldg(twA + t2 * stepA), __ldg(twA + t2 * stepA + QA),
                                __ldg(twA + t2 * stepA + 2 * QA)};
                butterfly<4, false>(y, wa, &wi, F);
                v[t2] = y[0]; v[4 + t2] = y[1]; v[8 + t2] = y[2]; v[12 + t2] = y[3];
            }
        }
#pragma unroll
        for (int t1 = 0; t1 < 4; t1++)
#pragma unroll
            for (int t2 = 0; t2 < 4; t2++) s[lay<PAD>(((row0 + t1 * 4 * q16 + t2 * q16) << T.lc) + c)] = v[t1 * 4 + t2];
    }
}

// ---------------------------------------------------------------------------
// Radix-16 round on a dense tile (the TMA column passes), with the distance
// between a unit's 16 points, 2^LS elements, known at compile time and the
// prime's constants taken from constant memory by a compile-time index: every
// shared-memory access is one base register plus an immediate offset, and no
// register holds or selects the field constants.  Same butterflies, same
// inputs, same order as round_r16.

// One radix-4 butterfly of the reference on four named values (butterfly<4>).
template <bool FWD>
__device__ __forceinline__ void bf4(double& a, double& b, double& c, double& d, double w1, double w2, double w3,
                                    double wi, const Fp F) {
    if (FWD) dft4(a, b, c, d, wi, F);
    a = fp_reduce(a, F);
    b = fp_mulmod(b, w1, F);
    c = fp_mulmod(c, w2, F);
    d = fp_mulmod(d, w3, F);
    if (!FWD) dft4(a, b, c, d, wi, F);
}

template <bool FWD, int LS, int PR>
__device__ __forceinline__ void r16_unit_dense(double* __restrict__ s, const double* __restrict__ twA,
                                               const double* __restrict__ twB, uint32_t stepA, uint32_t QA,
                                               uint32_t QB, double wi) {
    const Fp F = c_fp[PR];
    double v[16];
#pragma unroll
    for (int k = 0; k < 16; k++) v[k] = s[k << LS];
    if (FWD) {
#pragma unroll
        for (int t2 = 0; t2 < 4; t2++) {
            const double* ta = twA + t2 * stepA;
            bf4<true>(v[t2], v[4 + t2], v[8 + t2], v[12 + t2], __ldg(ta), __ldg(ta + QA), __ldg(ta + 2 * QA), wi, F);
        }
        const double b1 = __ldg(twB), b2 = __ldg(twB + QB), b3 = __ldg(twB + 2 * QB);
#pragma unroll
        for (int t1 = 0; t1 < 4; t1++)
            bf4<true>(v[4 * t1], v[4 * t1 + 1], v[4 * t1 + 2], v[4 * t1 + 3], b1, b2, b3, wi, F);
    } else {
        const double b1 = __ldg(twB), b2 = __ldg(twB + QB), b3 = __ldg(twB + 2 * QB);
#pragma unroll
        for (int t1 = 0; t1 < 4; t1++)
            bf4<false>(v[4 * t1], v[4 * t1 + 1], v[4 * t1 + 2], v[4 * t1 + 3], b1, b2, b3, wi, F);
#pragma unroll
        for (int t2 = 0; t2 < 4; t2++) {
            const double* ta = twA + t2 * stepA;
            bf4<false>(v[t2], v[4 + t2], v[8 + t2], v[12 + t2], __ldg(ta), __ldg(ta + QA), __ldg(ta + 2 * QA), wi, F);
        }
    }
#pragma unroll
    for (int k = 0; k < 16; k++) s[k << LS] = v[k];
}

// Tiles: prime 0 at T.s, prime 1 at T.s + T.stride (dense, row length C = 2^lc).
template <bool FWD, int LS>
__device__ NBG_ROUND void round_r16_dense(const Tiles& T, const DStage& A, const DStage& B) {
    const int lc = T.lc;
    const int C = 1 << lc;
    const int Lloc = (int)(A.L / T.Qb);
    const int q16 = Lloc >> 4, lq = __ffs(q16) - 1;
    const int per = (T.G >> 4) << lc;
    const uint32_t QA = (uint32_t)A.Q, QB = (uint32_t)B.Q;
    const uint32_t stepA = (uint32_t)q16 * (uint32_t)T.Qb;
    const double wi0 = A.rot[0][0], wi1 = A.rot[1][0];
    const double *twA0 = A.tw[0], *twA1 = A.tw[1], *twB0 = B.tw[0], *twB1 = B.tw[1];
    for (int u = threadIdx.x; u < 2 * per; u += blockDim.x) {
        const bool p1 = u >= per;
        const int uu = p1 ? u - per : u;
        const int c = uu & (C - 1);
        const int r = uu >> lc;
        const int b = r >> lq, j2 = r & (q16 - 1);
        const int base = ((b * Lloc + j2) << lc) + c;
        const uint32_t jB = (uint32_t)j2 * (uint32_t)T.Qb + (uint32_t)(T.j0 + c);
        if (p1) r16_unit_dense<FWD, LS, 1>(T.s + T.stride + base, twA1 + jB, twB1 + jB, stepA, QA, QB, wi1);
        else r16_unit_dense<FWD, LS, 0>(T.s + base, twA0 + jB, twB0 + jB, stepA, QA, QB, wi0);
    }
}

template <bool FWD>
__device__ __forceinline__ void round_r16_dense_any(const Tiles& T, const DStage& A, const DStage& B) {
    const int ls = (__ffs((int)(A.L / T.Qb)) - 1 - 4) + T.lc;  // log2(q16 * C)
    switch (ls) {
        case 4: round_r16_dense<FWD, 4>(T, A, B); break;
        case 5: round_r16_dense<FWD, 5>(T, A, B); break;
        case 6: round_r16_dense<FWD, 6>(T, A, B); break;
        case 7: round_r16_dense<FWD, 7>(T, A, B); break;
        case 8: round_r16_dense<FWD, 8>(T, A, B); break;
        case 9: round_r16_dense<FWD, 9>(T, A, B); break;
        case 10: round_r16_dense<FWD, 10>(T, A, B); break;
        case 11: round_r16_dense<FWD, 11>(T, A, B); break;
        default: round_r16<FWD, false>(T, A, B); break;
    }
}

// Radix-8 round: the span-8 radix-4 stage A (Q = 2) and the radix-2 stage, on
// 8 consecutive points (contiguous passes only: C = 1, Qb = 1, j0 = 0).
template <bool FWD>
__device__ NBG_ROUND void round_r8(const Tiles& T, const DStage& A) {
    const int per = T.G >> 3;
    const int total = per * T.ntiles;
    const Fp F0 = fpctx(0), F1 = fpctx(1);
    const double wi0 = A.rot[0][0], wi1 = A.rot[1][0];
    const double *tw0 = A.tw[0], *tw1 = A.tw[1];
    for (int u = threadIdx.x; u < total; u += blockDim.x) {
        int tau;
        const int b = split_unit(u, per, tau);
        const bool p1 = T.pfix >= 0 ? T.pfix == 1 : (tau >> T.pshift) != 0;
        const Fp F = p1 ? F1 : F0;
        const double wi = p1 ? wi1 : wi0;
        double* s = T.s + tau * T.stride;
        double v[8];
#pragma unroll
        for (int k = 0; k < 8; k++) v[k] = s[sp(8 * b + k)];
        const double* tw = p1 ? tw1 : tw0;
        const double w0[4] = {0.0, __ldg(tw + 0), __ldg(tw + 2), __ldg(tw + 4)};
        const double w1[4] = {0.0, __ldg(tw + 1), __ldg(tw + 3), __ldg(tw + 5)};
        if (!FWD) {
#pragma unroll
            for (int i = 0; i < 4; i++) butterfly2(v[2 * i], v[2 * i + 1], F);
        }
        {
            double y[4] = {v[0], v[2], v[4], v[6]};
            butterfly<4, FWD>(y, w0, &wi, F);
            v[0] = y[0]; v[2] = y[1]; v[4] = y[2]; v[6] = y[3];
            double z[4] = {v[1], v[3], v[5], v[7]};
            butterfly<4, FWD>(z, w1, &wi, F);
            v[1] = z[0]; v[3] = z[1]; v[5] = z[2]; v[7] = z[3];
        }
        if (FWD) {
#pragma unroll
            for (int i = 0; i < 4; i++) butterfly2(v[2 * i], v[2 * i + 1], F);
        }
#pragma unroll
        for (int k = 0; k < 8; k++) s[sp(8 * b + k)] = v[k];
    }
}

// ---------------------------------------------------------------------------
// Fused middle of the last pass: the forward's last round on a and b, the
// pointwise product and the reverse's first round (the same stages,
// transposed) on the same registers.  The twiddles are loaded once.
// Tiles: a_f = T.s + f * T.stride * (sq ? 1 : 2), b_f = a_f + (sq ? 0 : T.stride).
struct FuseTiles {
    double* s;
    int stride;
    int sq;
    int G, lc, Qb, j0;
    int pfix;  // -1: tiles of both primes; 0 or 1: only that prime's (a, b) tiles
    int bspec; // b's tiles hold its spectrum already: its forward round is skipped
    int bsave; // b's spectrum is stored after this round: write its forward result back
};

__device__ __forceinline__ void pw4(double* a, const double* b, Fp F) {
#pragma unroll
    for (int t = 0; t < 4; t++) a[t] = fp_mulmod(a[t], b[t], F);
}

template <bool FWD>
__device__ __forceinline__ void r16_body(double* v, const double* twA, uint32_t stepA, uint32_t QA, const double* wB,
                                         double wi, Fp F) {
    if (FWD) {
#pragma unroll
        for (int t2 = 0; t2 < 4; t2++) {
            double y[4] = {v[t2], v[4 + t2], v[8 + t2], v[12 + t2]};
            const double w[4] = {0.0, __ldg(twA + t2 * stepA), __ldg(twA + t2 * stepA + QA),
                                 __ldg(twA + t2 * stepA + 2 * QA)};
            butterfly<4, true>(y, w, &wi, F);
            v[t2] = y[0]; v[4 + t2] = y[1]; v[8 + t2] = y[2]; v[12 + t2] = y[3];
        }
#pragma unroll
        for (int t1 = 0; t1 < 4; t1++) butterfly<4, true>(v + 4 * t1, wB, &wi, F);
    } else {
#pragma unroll
        for (int t1 = 0; t1 < 4; t1++) butterfly<4, false>(v + 4 * t1, wB, &wi, F);
#pragma unroll
        for (int t2 = 0; t2 < 4; t2++) {
            double y[4] = {v[t2], v[4 + t2], v[8 + t2], v[12 + t2]};
            const double w[4] = {0.0, __ldg(twA + t2 * stepA), __ldg(twA + t2 * stepA + QA),
                                 __ldg(twA + t2 * stepA + 2 * QA)};
            butterfly<4, false>(y, w, &wi, F);
            v[t2] = y[0]; v[4 + t2] = y[1]; v[8 + t2] = y[2]; v[12 + t2] = y[3];
        }
    }
}

__device__ NBG_ROUND void fused_r16(const FuseTiles& T, const DStage& A, const DStage& B) {
    const int C = 1 << T.lc;
    const int Lloc = (int)(A.L / T.Qb);
    const int q16 = Lloc >> 4, lq = __ffs(q16) - 1;
    const uint32_t QA = (uint32_t)A.Q, QB = (uint32_t)B.Q;
    const int per = (T.G >> 4) << T.lc;
    const int total = T.pfix >= 0 ? per : 2 * per;
    const double wi0 = A.rot[0][0], wi1 = A.rot[1][0];
    const double *twA0 = A.tw[0], *twA1 = A.tw[1], *twB0 = B.tw[0], *twB1 = B.tw[1];
    for (int u = threadIdx.x; u < total; u += blockDim.x) {
        const bool p1 = T.pfix >= 0 ? T.pfix == 1 : u >= per;
        const int uu = (T.pfix < 0 && p1) ? u - per : u;
        const Fp F = fpctx(p1 ? 1 : 0);
        const double wi = p1 ? wi1 : wi0;
        double* sa = T.s + ((T.pfix < 0 && p1) ? (T.sq ? 1 : 2) : 0) * T.stride;
        double* sb = T.sq ? sa : sa + T.stride;
        const int c = uu & (C - 1);
        const int r = uu >> T.lc;
        const int b = r >> lq, j2 = r & (q16 - 1);
        const int row0 = b * Lloc + j2;
#define NBG_OFF(k) sp(((row0 + ((k) >> 2) * 4 * q16 + ((k) & 3) * q16) << T.lc) + c)
        const int jB = j2 * T.Qb + T.j0 + c;
        const double* twB = (p1 ? twB1 : twB0) + jB;
        const double* twA = (p1 ? twA1 : twA0) + jB;
        const uint32_t stepA = (uint32_t)q16 * (uint32_t)T.Qb;
        const double wB[4] = {0.0, __ldg(twB), __ldg(twB + QB), __ldg(twB + 2 * QB)};
        double va[16];
        if (!T.sq && !T.bspec) {
            // b's forward round goes back to its own shared slots (same thread),
            // keeping one operand in registers at a time
#pragma unroll
            for (int k = 0; k < 16; k++) va[k] = sb[NBG_OFF(k)];
            r16_body<true>(va, twA, stepA, QA, wB, wi, F);
#pragma unroll
            for (int k = 0; k < 16; k++) sb[NBG_OFF(k)] = va[k];
        }
#pragma unroll
        for (int k = 0; k < 16; k++) va[k] = sa[NBG_OFF(k)];
        r16_body<true>(va, twA, stepA, QA, wB, wi, F);
        // pointwise (fp_ntt_pointwise!, :770-785)
        if (T.sq) {
#pragma unroll
            for (int k = 0; k < 16; k++) va[k] = fp_mulmod(va[k], va[k], F);
        } else {
#pragma unroll
            for (int k = 0; k < 16; k++) va[k] = fp_mulmod(va[k], sb[NBG_OFF(k)], F);
        }
        r16_body<false>(va, twA, stepA, QA, wB, wi, F);
#pragma unroll
        for (int k = 0; k < 16; k++) sa[NBG_OFF(k)] = va[k];
#undef NBG_OFF
    }
}

__device__ NBG_ROUND void fused_r8(const FuseTiles& T, const DStage& A) {
    const int per = T.G >> 3;
    const int total = T.pfix >= 0 ? per : 2 * per;
    const double wi0 = A.rot[0][0], wi1 = A.rot[1][0];
    const double *tw0 = A.tw[0], *tw1 = A.tw[1];
    for (int u = threadIdx.x; u < total; u += blockDim.x) {
        const bool p1 = T.pfix >= 0 ? T.pfix == 1 : u >= per;
        const int b = (T.pfix < 0 && p1) ? u - per : u;
        const Fp F = fpctx(p1 ? 1 : 0);
        const double wi = p1 ? wi1 : wi0;
        double* sa = T.s + ((T.pfix < 0 && p1) ? (T.sq ? 1 : 2) : 0) * T.stride;
        double* sb = T.sq ? sa : sa + T.stride;
        const double* tw = p1 ? tw1 : tw0;
        const double w0[4] = {0.0, __ldg(tw + 0), __ldg(tw + 2), __ldg(tw + 4)};
        const double w1[4] = {0.0, __ldg(tw + 1), __ldg(tw + 3), __ldg(tw + 5)};
        double va[8], vb[8];
#pragma unroll
        for (int k = 0; k < 8; k++) va[k] = sa[sp(8 * b + k)];
        if (!T.sq) {
#pragma unroll
            for (int k = 0; k < 8; k++) vb[k] = sb[sp(8 * b + k)];
        }
#pragma unroll
        for (int op = 0; op < 2; op++) {
            if (op == 1 && (T.sq || T.bspec)) break;
            double* v = op ? vb : va;
            double y[4] = {v[0], v[2], v[4], v[6]};
            butterfly<4, true>(y, w0, &wi, F);
            v[0] = y[0]; v[2] = y[1]; v[4] = y[2]; v[6] = y[3];
            double z[4] = {v[1], v[3], v[5], v[7]};
            butterfly<4, true>(z, w1, &wi, F);
            v[1] = z[0]; v[3] = z[1]; v[5] = z[2]; v[7] = z[3];
#pragma unroll
            for (int i = 0; i < 4; i++) butterfly2(v[2 * i], v[2 * i + 1], F);
        }
        if (T.bsave) {  // b's forward result lives in registers here: the stored spectrum needs it
#pragma unroll
            for (int k = 0; k < 8; k++) sb[sp(8 * b + k)] = vb[k];
        }
#pragma unroll
        for (int k = 0; k < 2; k++) pw4(va + 4 * k, T.sq ? va + 4 * k : vb + 4 * k, F);
#pragma unroll
        for (int i = 0; i < 4; i++) butterfly2(va[2 * i], va[2 * i + 1], F);
        {
            double y[4] = {va[0], va[2], va[4], va[6]};
            butterfly<4, false>(y, w0, &wi, F);
            va[0] = y[0]; va[2] = y[1]; va[4] = y[2]; va[6] = y[3];
            double z[4] = {va[1], va[3], va[5], va[7]};
            butterfly<4, false>(z, w1, &wi, F);
            va[1] = z[0]; va[3] = z[1]; va[5] = z[2]; va[7] = z[3];
        }
#pragma unroll
        for (int k = 0; k < 8; k++) sa[sp(8 * b + k)] = va[k];
    }
}

// PAD = false (dense TMA tiles) occurs only in column passes, which hold no
// radix-8 or radix-2 round (those stages end a transform: the last pass).
// ODD = false: the pass holds no radix-3/5/7 stage (every pass but the first of
// an odd-length transform), so that code and its registers are left out.
template <bool FWD, bool PAD = true, bool ODD = true>
__device__ void run_round(const Tiles& T, const DPlan& pl, int kind, int s0) {
    __syncthreads();
    const DStage& st = pl.st[s0];
    switch (kind) {
        case RK_R16:
            if (PAD) round_r16<FWD, PAD>(T, st, pl.st[s0 + 1]);
            else round_r16_dense_any<FWD>(T, st, pl.st[s0 + 1]);
            break;
        case RK_R4: round_gen<4, FWD, PAD>(T, st); break;
        case RK_R8:
            if (PAD) round_r8<FWD>(T, st);
            break;
        case RK_R2:
            if (PAD) round_gen<2, FWD, PAD>(T, st);
            break;
        default:
            if (!ODD) break;
            if (st.m == 3) round_gen<3, FWD, PAD>(T, st);
            else if (st.m == 5) round_gen<5, FWD, PAD>(T, st);
            else round_gen<7, FWD, PAD>(T, st);
            break;
    }
}

template <bool FWD, bool PAD = true, bool ODD = true>
__device__ void run_pass(const Tiles& T, const DPlan& pl, const DPass& ps) {
    if (FWD) {
        for (int r = 0; r < ps.nrounds; r++) run_round<true, PAD, ODD>(T, pl, ps.rkind[r], ps.rstage[r]);
    } else {
        for (int r = ps.nrounds - 1; r >= 0; r--) run_round<false, PAD, ODD>(T, pl, ps.rkind[r], ps.rstage[r]);
    }
    __syncthreads();
}

// Tile geometry: tile t of pass ps -> global index of its (row 0, column 0) and its first column.
__device__ __forceinline__ void tile_geo(const DPlan& pl, const DPass& ps, int64_t t, int64_t& base, int& j0) {
    const int64_t per = ps.Qb / ps.C;
    const int64_t blk = t / per;
    j0 = (int)((t - blk * per) * ps.C);
    base = blk * pl.st[ps.sa].L + j0;
}

// Asynchronous global -> shared copies (cp.async, 8 bytes each): a thread
// issues every copy of its share of the tile set before waiting once, so the
// loads of a whole tile are in flight together instead of one per thread.
__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// x[base + c + k*Qb] -> tile row k, column c (padded).  Issues only; the
// caller waits with cp_async_wait_all() and a barrier.
__device__ __forceinline__ void load_tile_async(double* s, const double* __restrict__ x, const DPass& ps,
                                                int64_t base) {
    const int lc = __ffs(ps.C) - 1;
    const int n = ps.G << lc;
    const int64_t Qb = ps.Qb;
    x += base;
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
        const int k = e >> lc, c = e & (ps.C - 1);
        cp_async8(s + sp(e), x + c + k * Qb);
    }
}
__device__ __forceinline__ void store_tile(const double* s, double* __restrict__ x, const DPass& ps, int64_t base) {
    const int lc = __ffs(ps.C) - 1;
    const int n = ps.G << lc;
    const int64_t Qb = ps.Qb;
    const int nt = blockDim.x;
    int e = threadIdx.x;
    // batches of 4 shared loads ahead of their global stores
    for (; e + 3 * nt < n; e += 4 * nt) {
        double v[4];
#pragma unroll
        for (int q = 0; q < 4; q++) v[q] = s[sp(e + q * nt)];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int ee = e + q * nt;
            x[base + (ee & (ps.C - 1)) + (ee >> lc) * Qb] = v[q];
        }
    }
    for (; e < n; e += nt) x[base + (e & (ps.C - 1)) + (e >> lc) * Qb] = s[sp(e)];
}
// one packed chunk written to both primes' tiles s0 and s1; chunks are
// processed 4 per thread at a time so their limb loads overlap
template <bool PAD = true>
__device__ __forceinline__ void pack_tile2(double* s0, double* s1, const uint64_t* __restrict__ limbs, int64_t n,
                                           int b, int64_t nch, const DPass& ps, int64_t base) {
    const int lc = __ffs(ps.C) - 1;
    const int cnt = ps.G << lc;
    const int Qb = (int)ps.Qb;
    const int nt = blockDim.x;
    const uint64_t mask = (1ULL << b) - 1ULL;
    for (int e0 = threadIdx.x; e0 < cnt; e0 += 4 * nt) {
        uint64_t lo[4], hi[4];
        int sh[4];
        bool live[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int e = e0 + q * nt;
            const int64_t i = e < cnt ? (int64_t)base + (e & (ps.C - 1)) + (int64_t)(e >> lc) * Qb : nch;
            live[q] = i < nch;
            const uint64_t bit = (uint64_t)(live[q] ? i : 0) * (uint32_t)b;
            const int64_t w = (int64_t)(bit >> 6);
            sh[q] = (int)(bit & 63);
            lo[q] = live[q] ? __ldg(limbs + w) : 0;
            hi[q] = (live[q] && sh[q] + b > 64 && w + 1 < n) ? __ldg(limbs + w + 1) : 0;
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int e = e0 + q * nt;
            if (e >= cnt) break;
            uint64_t c = lo[q] >> sh[q];
            if (sh[q]) c |= hi[q] << (64 - sh[q]);
            const double v = live[q] ? small_u64_to_double(c & mask) : 0.0;
            s0[lay<PAD>(e)] = v;
            s1[lay<PAD>(e)] = v;
        }
    }
}

__device__ __forceinline__ Tiles make_tiles(double* s, int stride, int ntiles, int pshift, const DPass& ps, int j0) {
    Tiles T;
    T.s = s;
    T.stride = stride;
    T.ntiles = ntiles;
    T.pshift = pshift;
    T.G = ps.G;
    T.lc = __ffs(ps.C) - 1;
    T.Qb = (int)ps.Qb;
    T.j0 = j0;
    T.pfix = -1;
    return T;
}

// ---------------------------------------------------------------------------
// Forward pass of one tile of one operand, both primes (tiles X0, X1): one
// job, run by the whole CTA (the per-kind kernels and the queue kernel call it).
template <bool ODD>
__device__ __forceinline__ void job_fwd(const DProd* __restrict__ prods, const DPlan* __restrict__ plans,
                                        const Job& jb, double* smem) {
    {
        const DProd& P = prods[jb.prod];
        const DPlan& pl = plans[P.plan];
        const int opb = (jb.sub >> 1) & 1, pass = (jb.sub >> 8) & 0xff;
        const DPass& ps = pl.pass[pass];
        int64_t base;
        int j0;
        tile_geo(pl, ps, jb.tile, base, j0);
        const int stride = tile_stride_doubles(ps.G * ps.C);
        double* s0 = smem;
        double* s1 = smem + stride;
        double* x0 = opb ? P.xb[0] : P.xa[0];
        double* x1 = opb ? P.xb[1] : P.xa[1];
        __syncthreads();
        if (pass == 0 && !(P.flags & PF_PRELOADED)) {
            if (opb) pack_tile2(s0, s1, P.b, P.n, P.bch, P.ncb, ps, base);
            else pack_tile2(s0, s1, P.a, P.m, P.bch, P.nca, ps, base);
        } else {
            load_tile_async(s0, x0, ps, base);
            load_tile_async(s1, x1, ps, base);
            cp_async_wait_all();
        }
        run_pass<true, true, ODD>(make_tiles(smem, stride, 2, 0, ps, j0), pl, ps);
        store_tile(s0, x0, ps, base);
        store_tile(s1, x1, ps, base);
    }
}

// MINB: CTAs per SM the register budget is cut for (3: 80 registers, 4: 64);
// launches pick 4 when the tile set is small enough for four CTAs' shared memory.
template <int MINB, bool ODD>
__global__ void __launch_bounds__(PASS_THREADS, MINB) k_fwd(const DProd* __restrict__ prods,
                                                         const DPlan* __restrict__ plans,
                                                         const Job* __restrict__ jobs, int64_t njobs) {
    extern __shared__ double smem[];
    // a run of consecutive jobs per CTA: in column passes they share twiddle
    // columns, which stay in L1 from one tile to the next
    const int64_t run = (njobs + gridDim.x - 1) / gridDim.x;
    const int64_t jend = min(njobs, ((int64_t)blockIdx.x + 1) * run);
    for (int64_t ji = (int64_t)blockIdx.x * run; ji < jend; ji++) job_fwd<ODD>(prods, plans, jobs[ji], smem);
}

// Last pass, both primes: forward on a (and b), pointwise, reverse on a.
// Tiles: products [a0, b0, a1, b1], squares [a0, a1].
// SPLIT: one CTA per prime (JK_PWR_SPLIT).  KEEPB: launches of products with
// a kept operand spectrum (JK_PWR_KEEP; PF_BSAVE / PF_BSPEC), compiled apart
// so the other launches carry none of that code.
template <bool SPLIT, bool KEEPB, bool ODD>
__device__ __forceinline__ void job_pwr(const DProd* __restrict__ prods, const DPlan* __restrict__ plans,
                                        const Job& jb, double* smem) {
    {
        const DProd& P = prods[jb.prod];
        const DPlan& pl = plans[P.plan];
        const int pass = P.npass - 1;
        const DPass& ps = pl.pass[pass];
        int64_t base;
        int j0;
        tile_geo(pl, ps, jb.tile, base, j0);
        const int stride = tile_stride_doubles(ps.G * ps.C);
        const int sq = P.sqr;
        // split launches (JK_PWR_SPLIT) give each prime (sub bit 1) its own
        // CTA: half the tiles, twice the CTAs, for batches too small to fill
        // the GPU
        const int pf = SPLIT ? (jb.sub >> 1) & 1 : -1;
        double* a0 = smem;
        double* a1 = smem + (sq ? 1 : 2) * stride;
        double* b0 = sq ? a0 : smem + stride;
        double* b1 = sq ? a1 : smem + 3 * stride;
        const int p0 = pf >= 0 ? pf : 0;
        const int cnt = ps.G * ps.C;
        // operand b's spectrum: kept from an earlier run (bspec) or to be kept (bsave)
        const bool bspec = KEEPB && !sq && (P.flags & PF_BSPEC);
        const bool bsave = KEEPB && !sq && (P.flags & PF_BSAVE);
        __syncthreads();
        if (pass == 0 && !(P.flags & PF_PRELOADED)) {
            pack_tile2(a0, pf >= 0 ? a0 : a1, P.a, P.m, P.bch, P.nca, ps, base);
            if (bspec) {
                load_tile_async(b0, P.xb[p0], ps, base);
                if (pf < 0) load_tile_async(b1, P.xb[1], ps, base);
                cp_async_wait_all();
            } else if (!sq) {
                pack_tile2(b0, pf >= 0 ? b0 : b1, P.b, P.n, P.bch, P.ncb, ps, base);
            }
        } else {
            load_tile_async(a0, P.xa[p0], ps, base);
            if (!sq) load_tile_async(b0, P.xb[p0], ps, base);
            if (pf < 0) {
                load_tile_async(a1, P.xa[1], ps, base);
                if (!sq) load_tile_async(b1, P.xb[1], ps, base);
            }
            cp_async_wait_all();
        }
        Tiles TF = pf < 0 ? make_tiles(smem, stride, sq ? 2 : 4, sq ? 0 : 1, ps, j0)
                          : make_tiles(smem, stride, sq ? 1 : 2, 30, ps, j0);
        if (bspec)  // b is transformed already: the forward rounds run on the a tiles only
            TF = pf < 0 ? make_tiles(a0, (int)(a1 - a0), 2, 0, ps, j0) : make_tiles(a0, stride, 1, 30, ps, j0);
        Tiles TR = pf < 0 ? make_tiles(a0, (int)(a1 - a0), 2, 0, ps, j0) : make_tiles(a0, stride, 1, 30, ps, j0);
        TF.pfix = pf;
        TR.pfix = pf;
        const int nr = ps.nrounds;
        const int lastk = ps.rkind[nr - 1];
        if (lastk == RK_R16 || lastk == RK_R8) {
            // forward rounds but the last, fused round, reverse rounds but the first
            for (int r = 0; r < nr - 1; r++) run_round<true, true, ODD>(TF, pl, ps.rkind[r], ps.rstage[r]);
            __syncthreads();
            FuseTiles FT;
            FT.s = smem;
            FT.stride = stride;
            FT.sq = sq;
            FT.G = ps.G;
            FT.lc = __ffs(ps.C) - 1;
            FT.Qb = (int)ps.Qb;
            FT.j0 = j0;
            FT.pfix = pf;
            FT.bspec = bspec;
            FT.bsave = bsave;
            const int s0 = ps.rstage[nr - 1];
            if (lastk == RK_R16) fused_r16(FT, pl.st[s0], pl.st[s0 + 1]);
            else fused_r8(FT, pl.st[s0]);
            if (bsave) {  // b's tiles are fully transformed now; the reverse leaves them alone
                __syncthreads();
                store_tile(b0, P.xb[p0], ps, base);
                if (pf < 0) store_tile(b1, P.xb[1], ps, base);
            }
            for (int r = nr - 2; r >= 0; r--) run_round<false, true, ODD>(TR, pl, ps.rkind[r], ps.rstage[r]);
            __syncthreads();
        } else {
            run_pass<true, true, ODD>(TF, pl, ps);
            if (bsave) {
                store_tile(b0, P.xb[p0], ps, base);
                if (pf < 0) store_tile(b1, P.xb[1], ps, base);
            }
            if (pf < 0) {
                const Fp F0 = fpctx(0), F1 = fpctx(1);
                for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
                    const int i = sp(e);
                    a0[i] = fp_mulmod(a0[i], b0[i], F0);
                    a1[i] = fp_mulmod(a1[i], b1[i], F1);
                }
            } else {
                const Fp F = fpctx(pf);
                for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
                    const int i = sp(e);
                    a0[i] = fp_mulmod(a0[i], b0[i], F);
                }
            }
            run_pass<false, true, ODD>(TR, pl, ps);
        }
        store_tile(a0, P.xa[p0], ps, base);
        if (pf < 0) store_tile(a1, P.xa[1], ps, base);
    }
}

template <bool SPLIT, bool KEEPB, bool ODD>
__global__ void __launch_bounds__(PASS_THREADS, NBG_PWR_MINB) k_pwr(const DProd* __restrict__ prods,
                                                         const DPlan* __restrict__ plans,
                                                         const Job* __restrict__ jobs, int64_t njobs) {
    extern __shared__ double smem[];
    for (int64_t ji = blockIdx.x; ji < njobs; ji += gridDim.x) job_pwr<SPLIT, KEEPB, ODD>(prods, plans, jobs[ji], smem);
}

// Reverse pass of one tile, both primes (one job).
template <bool ODD>
__device__ __forceinline__ void job_rev(const DProd* __restrict__ prods, const DPlan* __restrict__ plans,
                                        const Job& jb, double* smem) {
    {
        const DProd& P = prods[jb.prod];
        const DPlan& pl = plans[P.plan];
        const int pass = (jb.sub >> 8) & 0xff;
        const DPass& ps = pl.pass[pass];
        int64_t base;
        int j0;
        tile_geo(pl, ps, jb.tile, base, j0);
        const int stride = tile_stride_doubles(ps.G * ps.C);
        __syncthreads();
        load_tile_async(smem, P.xa[0], ps, base);
        load_tile_async(smem + stride, P.xa[1], ps, base);
        cp_async_wait_all();
        run_pass<false, true, ODD>(make_tiles(smem, stride, 2, 0, ps, j0), pl, ps);
        store_tile(smem, P.xa[0], ps, base);
        store_tile(smem + stride, P.xa[1], ps, base);
    }
}

template <int MINB, bool ODD>
__global__ void __launch_bounds__(PASS_THREADS, MINB) k_rev(const DProd* __restrict__ prods,
                                                         const DPlan* __restrict__ plans,
                                                         const Job* __restrict__ jobs, int64_t njobs) {
    extern __shared__ double smem[];
    // a run of consecutive jobs per CTA: in column passes they share twiddle
    // columns, which stay in L1 from one tile to the next
    const int64_t run = (njobs + gridDim.x - 1) / gridDim.x;
    const int64_t jend = min(njobs, ((int64_t)blockIdx.x + 1) * run);
    for (int64_t ji = (int64_t)blockIdx.x * run; ji < jend; ji++) job_rev<ODD>(prods, plans, jobs[ji], smem);
}

// ---------------------------------------------------------------------------
// Column passes staged by TMA.  The tiles of one (product class, pass,
// operand) are boxes of one 3-D tensor map over the class's transform
// buffers: x = column (Qb wide rows), y = row (N / Qb rows), z = buffer
// (2 per product: prime 0, prime 1).  One cp.async.bulk.tensor load brings both
// primes' G x C tiles into shared memory (dense, [prime][row][column]) and one
// store writes them back; tiles have at least 16 columns, so the rounds' accesses
// are free of bank conflicts without padding.  The tensor maps cover this GPU's
// own workspace only, and no load uses cluster multicast.

// mbarrier waits that gave up (the host reads and clears it: nbg_device_faults)
__device__ unsigned int g_nbg_faults = 0;

namespace tma {

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void bar_expect(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool bar_try(uint64_t* bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(saddr(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}
// Waits for the barrier's phase with a bound of about 2^32 SM clocks (two
// seconds); returns false (and counts a fault) when it gives up.
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t phase) {
    if (bar_try(bar, phase)) return true;
    const long long t0 = clock64();
    while (!bar_try(bar, phase)) {
        if (clock64() - t0 > (1LL << 32)) {
            if (threadIdx.x == 0) atomicAdd(&g_nbg_faults, 1u);
            return false;
        }
    }
    return true;
}
__device__ __forceinline__ void load3(void* dst, const void* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(saddr(dst)), "l"(map), "r"(x), "r"(y), "r"(z), "r"(saddr(bar))
        : "memory");
}
// untiled bulk copy of `bytes` (a multiple of 16) from 16-byte aligned global
// memory of this GPU into 16-byte aligned shared memory, completing on bar
__device__ __forceinline__ void load1(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(saddr(dst)), "l"(src), "r"(bytes), "r"(saddr(bar))
                 : "memory");
}
__device__ __forceinline__ void store3(const void* map, int x, int y, int z, const void* src) {
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];"
                 ::"l"(map), "r"(x), "r"(y), "r"(z), "r"(saddr(src))
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// the bulk stores issued so far have read their shared-memory source
__device__ __forceinline__ void stores_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// the bulk stores issued so far are complete
__device__ __forceinline__ void stores_done() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// generic-proxy shared-memory accesses before this point are ordered before later async-proxy ones
__device__ __forceinline__ void fence_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// a tensor map the host wrote to global memory, made visible to the tensor-map proxy
__device__ __forceinline__ void fence_map(const void* map) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(map) : "memory");
}

}  // namespace tma

// box origin of column tile t: x = first column, y = first row
__device__ __forceinline__ void tile_box(const DPass& ps, int64_t t, int& x, int& y) {
    const int64_t per = ps.Qb / ps.C;
    const int64_t blk = t / per;
    x = (int)((t - blk * per) * ps.C);
    y = (int)(blk * ps.G);
}

// One column pass (forward or reverse) of one tile of one operand, both primes,
// staged by TMA.  Dynamic shared memory: [mbarrier | 120 B | tiles].
// One tile (one job); false when the bounded wait for its load gave up.
// smem: the tile region (128-byte aligned); bar: the CTA's mbarrier, whose
// phase the caller keeps.
template <bool FWD, bool ODD>
__device__ __forceinline__ bool job_col_tma(const DProd* __restrict__ prods, const DPlan* __restrict__ plans,
                                            const Job& jb, double* smem, uint64_t* bar, uint32_t& phase) {
    {
        const DProd& P = prods[jb.prod];
        const DPlan& pl = plans[P.plan];
        const int opb = FWD ? (jb.sub >> 1) & 1 : 0;
        const int pass = (jb.sub >> 8) & 0xff;
        const DPass& ps = pl.pass[pass];
        int x, y;
        tile_box(ps, jb.tile, x, y);
        const int z = 2 * P.tslot;
        const void* map = static_cast<const char*>(P.tmap) + 128 * (2 * pass + opb);
        const int cnt = ps.G * ps.C;
        const bool pack = FWD && pass == 0 && !(P.flags & PF_PRELOADED);
        __syncthreads();  // every thread is done with the previous tile
        if (threadIdx.x == 0) {
            tma::stores_read();  // the previous tile's store has read shared memory
            if (!pack) {
                tma::fence_map(map);
                tma::bar_expect(bar, (uint32_t)(2 * cnt * sizeof(double)));
                tma::load3(smem, map, x, y, z, bar);
            }
        }
        if (pack) {
            __syncthreads();
            const int64_t base = (int64_t)(y / ps.G) * pl.st[ps.sa].L + x;
            if (opb) pack_tile2<false>(smem, smem + cnt, P.b, P.n, P.bch, P.ncb, ps, base);
            else pack_tile2<false>(smem, smem + cnt, P.a, P.m, P.bch, P.nca, ps, base);
        } else {
            if (!tma::bar_wait(bar, phase)) return false;
            phase ^= 1u;
        }
        run_pass<FWD, false, ODD>(make_tiles(smem, cnt, 2, 0, ps, x), pl, ps);
        tma::fence_async();
        __syncthreads();
        if (threadIdx.x == 0) tma::store3(map, x, y, z, smem);
    }
    return true;
}

template <int MINB, bool FWD, bool ODD>
__global__ void __launch_bounds__(PASS_THREADS, MINB) k_col_tma(const DProd* __restrict__ prods,
                                                             const DPlan* __restrict__ plans,
                                                             const Job* __restrict__ jobs, int64_t njobs) {
    extern __shared__ __align__(128) double dsm[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(dsm);
    double* smem = dsm + 16;  // tiles start 128 bytes in
    if (threadIdx.x == 0) tma::bar_init(bar);
    __syncthreads();
    uint32_t phase = 0;
    const int64_t run = (njobs + gridDim.x - 1) / gridDim.x;
    const int64_t jend = min(njobs, ((int64_t)blockIdx.x + 1) * run);
    for (int64_t ji = (int64_t)blockIdx.x * run; ji < jend; ji++)
        if (!job_col_tma<FWD, ODD>(prods, plans, jobs[ji], smem, bar, phase)) break;  // gave up (counted)
    if (threadIdx.x == 0) tma::stores_done();  // leave after the stores issued so far
}

// ---------------------------------------------------------------------------
// Unpack.  Coefficient i (value c_i = c1 + p1*u < p1*p2 < 2^100) sits at
// x[(N - i) mod N] scaled by N (fp_ntt_rev! :723-726).  The product is
// sum_i c_i 2^(b i); its limb w collects the 64-bit slices of the (at most
// five) coefficients overlapping bits [64w, 64w+64).  This equals the
// reference's S1 + p1*S2 fold (:793-795, :923) as an integer, so the limbs are
// identical.
__device__ __forceinline__ void garner_xy(double x1v, double x2v, const DPlan& pl, uint64_t& lo, uint64_t& hi) {
    const Fp F1 = fpctx(0), F2 = fpctx(1);
    double v1 = fp_mulmod4(x1v, pl.ninv[0], pl.ninvp[0], F1);
    v1 = v1 < 0.0 ? dadd(v1, F1.p) : v1;
    double v2 = fp_mulmod4(x2v, pl.ninv[1], pl.ninvp[1], F2);
    double u = fp_mulmod4(dsub(v2, fp_reduce(v1, F2)), c_garner[0], c_garner[1], F2);
    u = u < 0.0 ? dadd(u, F2.p) : u;
    // canonical values are < 2^50: adding 1.5*2^52 leaves them in the low 51
    // mantissa bits (the reference's vector unpack does the same, :897-901)
    const uint64_t m51 = (1ULL << 51) - 1ULL;
    uint64_t c1 = (uint64_t)__double_as_longlong(dadd(v1, FP_MAGIC)) & m51;
    uint64_t uu = (uint64_t)__double_as_longlong(dadd(u, FP_MAGIC)) & m51;
    // c = c1 + p1*uu  (128-bit)
    uint64_t plo = uu * P1_U;
    uint64_t phi = __umul64hi(uu, P1_U);
    lo = plo + c1;
    hi = phi + (lo < plo ? 1ULL : 0ULL);
}

constexpr int UNPACK_THREADS = 256;
constexpr int LIMBS_PER_THREAD = UNPACK_TL / UNPACK_THREADS;
static_assert(LIMBS_PER_THREAD == 4, "the limb window below is written for 4 limbs per thread");

__device__ __forceinline__ uint32_t gp_compose(uint32_t lower, uint32_t upper) {
    // (g,p) pairs packed as bit0 = generate, bit1 = propagate; lower then upper.
    uint32_t g = (upper & 1u) | ((upper >> 1) & lower & 1u);
    uint32_t p = (upper >> 1) & (lower >> 1) & 1u;
    return g | (p << 1);
}

// 3-word window W += c * 2^d, c = (lo, hi) < 2^100, 0 <= d < 64 (the sum stays below 2^192)
__device__ __forceinline__ void window_add(uint64_t& W0, uint64_t& W1, uint64_t& W2, uint64_t lo, uint64_t hi,
                                           uint32_t d) {
    const uint64_t a0 = lo << d;
    const uint64_t a1 = ((lo >> 1) >> (63 - d)) | (hi << d);
    const uint64_t a2 = (hi >> 1) >> (63 - d);
    asm("add.cc.u64 %0, %0, %3;\n\t"
        "addc.cc.u64 %1, %1, %4;\n\t"
        "addc.u64 %2, %2, %5;"
        : "+l"(W0), "+l"(W1), "+l"(W2)
        : "l"(a0), "l"(a1), "l"(a2));
}

// Limbs [wt, wt + 4) of the sum of the tile's coefficients k..kend (those that
// start in bits [64 wt, 64 (wt + 4)); d = b i - 64 wt), streamed through a
// 3-word window; the part above the range comes back as the spill (s0, s1),
// limbs wt + 4 and wt + 5.  OWN = false keeps only the spill.  Coefficient k's
// 128-bit value is (u1[top1 - k], u2[top2 - k]).
template <bool OWN>
__device__ __forceinline__ void range_limbs(const uint64_t* __restrict__ u1, const uint64_t* __restrict__ u2,
                                            int top1, int top2, int k, int kend, uint32_t d, uint32_t b,
                                            uint64_t* own, uint64_t& s0, uint64_t& s1) {
    uint64_t W0 = 0, W1 = 0, W2 = 0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        while (k <= kend && d < 64) {
            window_add(W0, W1, W2, u1[top1 - k], u2[top2 - k], d);
            k++;
            d += b;
        }
        if (OWN) own[q] = W0;
        W0 = W1;
        W1 = W2;
        W2 = 0;
        d -= 64;
    }
    s0 = W0;
    s1 = W1;
}

// floor(x / b) for 0 <= x < 2^50 and 1 <= b <= 52 without a 64-bit integer
// division: the double quotient is off by at most one, fixed by an exact check.
__device__ __forceinline__ int64_t div_b(int64_t x, int b, double rb) {
    int64_t q = (int64_t)__dmul_rn((double)x, rb);
    if (q * b > x) q--;
    else if ((q + 1) * b <= x) q++;
    return q;
}

// One unpack tile: output limbs [w0, w1) and the coefficients ilo..ihi that
// start in bits [64 wlo, 64 w1), wlo = w0 - 4 (the 4-limb range below the tile
// spills into limbs w0 and w0 + 1).
struct UTile {
    int64_t w0, w1, wlo, ilo, ihi, ncoef;
};

__device__ __forceinline__ UTile unpack_tile(const DProd& P, int64_t tile) {
    const int b = P.bch;
    const double rb = 1.0 / (double)b;
    UTile g;
    g.w0 = tile * UNPACK_TL;
    g.w1 = min(g.w0 + (int64_t)UNPACK_TL, P.rn);
    g.wlo = g.w0 >= 4 ? g.w0 - 4 : 0;
    g.ilo = div_b(64 * g.wlo + b - 1, b, rb);
    g.ihi = min(div_b(64 * g.w1 - 1, b, rb), P.nconv - 1);
    g.ncoef = g.ihi >= g.ilo ? g.ihi - g.ilo + 1 : 0;
    return g;
}

// Coefficient i > 0 has its residues at x[N - i], so the tile's residues
// (i = 0 apart: x[0], read directly) are the contiguous run x[N - ihi ..
// N - max(ilo, 1)], descending in i.  One untiled bulk copy per prime stages
// the run, widened to 16-byte boundaries (a 16-byte block holding a valid
// double lies inside the same allocation); the run starts `lead` (0 or 1)
// doubles into the stage.
__device__ __forceinline__ int stage_lead(const double* x, int64_t N, const UTile& g) {
    return (int)((reinterpret_cast<uintptr_t>(x + (N - g.ihi)) >> 3) & 1);
}

__device__ __forceinline__ void unpack_issue(const DProd& P, int64_t N, const UTile& g, double* st1, double* st2,
                                             uint64_t* bar) {
    const int64_t cnt = g.ncoef - (g.ilo == 0 ? 1 : 0);
    if (cnt <= 0) {
        tma::bar_expect(bar, 0);  // nothing to stage: the phase completes with this arrival
        return;
    }
    uintptr_t src[2];
    uint32_t bytes[2];
#pragma unroll
    for (int f = 0; f < 2; f++) {
        const uintptr_t a = reinterpret_cast<uintptr_t>(P.xa[f] + (N - g.ihi));
        src[f] = a & ~(uintptr_t)15;
        bytes[f] = (uint32_t)(((a + 8 * (uintptr_t)cnt + 15) & ~(uintptr_t)15) - src[f]);
    }
    tma::bar_expect(bar, bytes[0] + bytes[1]);
    tma::load1(st1, reinterpret_cast<const void*>(src[0]), bytes[0], bar);
    tma::load1(st2, reinterpret_cast<const void*>(src[1]), bytes[1], bar);
}

// Phases after the tile's residues are staged (st1, st2: prime 1 and 2, each
// run starting `lead` doubles in): Garner in place, the per-thread limb
// windows, the spill exchange, the block carry-lookahead scan, the limb
// stores and the tile aggregate.  The stage's last read (and write) comes
// before a block barrier inside, after a proxy fence, so a bulk copy issued
// after this returns may refill it.
__device__ __forceinline__ void unpack_assemble(const DProd& P, const DPlan& pl, const Job& jb, const UTile& g,
                                                double* st1, double* st2, uint32_t* wagg, uint64_t (*spill)[2]) {
    const int t = threadIdx.x;
    const int b = P.bch;
    const int64_t N = pl.N;
    const int nc = (int)g.ncoef;
    const int top1 = stage_lead(P.xa[0], N, g) + nc - 1;
    const int top2 = stage_lead(P.xa[1], N, g) + nc - 1;
    uint64_t* const u1 = reinterpret_cast<uint64_t*>(st1);
    uint64_t* const u2 = reinterpret_cast<uint64_t*>(st2);
    // Garner in place: coefficient k's two residues become its (lo, hi)
    for (int k0 = t; k0 < nc; k0 += 8 * UNPACK_THREADS) {
        double a1[8], a2[8];
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const int k = k0 + q * UNPACK_THREADS;
            a1[q] = 0.0;
            a2[q] = 0.0;
            if (k < nc) {
                if (k == 0 && g.ilo == 0) {
                    a1[q] = P.xa[0][0];  // plain loads: in the queue kernel this launch wrote them
                    a2[q] = P.xa[1][0];
                } else {
                    a1[q] = st1[top1 - k];
                    a2[q] = st2[top2 - k];
                }
            }
        }
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const int k = k0 + q * UNPACK_THREADS;
            if (k < nc) {
                uint64_t lo, hi;
                garner_xy(a1[q], a2[q], pl, lo, hi);
                u1[top1 - k] = lo;
                u2[top2 - k] = hi;
            }
        }
    }
    __syncthreads();
    const int64_t w0 = g.w0, w1 = g.w1, ilo = g.ilo, ihi = g.ihi;
    const double rb = 1.0 / (double)b;
    const int64_t wt = w0 + 4 * (int64_t)t;
    uint64_t own[4], s0, s1;
    {
        const int64_t i0 = div_b(64 * wt + b - 1, b, rb);
        const int64_t i1 = min(div_b(64 * (wt + 4) - 1, b, rb), ihi);
        range_limbs<true>(u1, u2, top1, top2, (int)(i0 - ilo), (int)(i1 - ilo), (uint32_t)(b * i0 - 64 * wt),
                          (uint32_t)b, own, s0, s1);
    }
    spill[t + 1][0] = s0;
    spill[t + 1][1] = s1;
    if (t == 0) {
        uint64_t p0 = 0, p1 = 0;
        if (w0 > 0) {  // the spill of the range [w0 - 4, w0) into limbs w0, w0 + 1
            const int64_t i1 = min(div_b(64 * w0 - 1, b, rb), ihi);
            range_limbs<false>(u1, u2, top1, top2, 0, (int)(i1 - ilo), (uint32_t)(b * ilo - 64 * g.wlo),
                               (uint32_t)b, nullptr, p0, p1);
        }
        spill[0][0] = p0;
        spill[0][1] = p1;
    }
    // this stage's generic-proxy accesses come before the bulk copy that
    // refills it (issued after the barrier below)
    tma::fence_async();
    __syncthreads();
    // own + the spill from below: a carry (0 or 1) out of the 4 limbs, then
    // generate / propagate across threads
    uint32_t gen;
    {
        const uint64_t a0 = spill[t][0], a1 = spill[t][1];
        uint32_t c;
        asm("add.cc.u64 %0, %0, %5;\n\t"
            "addc.cc.u64 %1, %1, %6;\n\t"
            "addc.cc.u64 %2, %2, %7;\n\t"
            "addc.cc.u64 %3, %3, %7;\n\t"
            "addc.u32 %4, %8, %8;"
            : "+l"(own[0]), "+l"(own[1]), "+l"(own[2]), "+l"(own[3]), "=r"(c)
            : "l"(a0), "l"(a1), "l"(0ULL), "r"(0u));
        gen = c;
    }
    // limbs past the product's end are zero and must not propagate
    uint32_t prop = 1u;
#pragma unroll
    for (int q = 0; q < 4; q++) prop &= (wt + q < w1 && own[q] == ~0ULL) ? 1u : 0u;
    const uint32_t agg = gen | (prop << 1);
    // block exclusive scan of agg (carry-in to each thread, tile carry-in 0)
    const int lane = t & 31, wid = t >> 5;
    uint32_t incl = agg;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        uint32_t o = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl = gp_compose(o, incl);
    }
    if (lane == 31) wagg[wid] = incl;
    __syncthreads();
    uint32_t wpre = 2u;
    for (int k = 0; k < wid; k++) wpre = gp_compose(wpre, wagg[k]);
    uint32_t excl = __shfl_up_sync(0xffffffffu, incl, 1);
    if (lane == 0) excl = 2u;
    excl = gp_compose(wpre, excl);
    const uint64_t cin = excl & 1u;  // tile carry-in assumed 0
    asm("add.cc.u64 %0, %0, %4;\n\t"
        "addc.cc.u64 %1, %1, %5;\n\t"
        "addc.cc.u64 %2, %2, %5;\n\t"
        "addc.u64 %3, %3, %5;"
        : "+l"(own[0]), "+l"(own[1]), "+l"(own[2]), "+l"(own[3])
        : "l"(cin), "l"(0ULL));
    if (wt + 3 < w1) {
        ulonglong2* dst = reinterpret_cast<ulonglong2*>(P.r + wt);
        if ((reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
            dst[0] = make_ulonglong2(own[0], own[1]);
            dst[1] = make_ulonglong2(own[2], own[3]);
        } else {
#pragma unroll
            for (int q = 0; q < 4; q++) P.r[wt + q] = own[q];
        }
    } else {
#pragma unroll
        for (int q = 0; q < 4; q++)
            if (wt + q < w1) P.r[wt + q] = own[q];
    }
    if (t == blockDim.x - 1 && P.agg) {
        uint32_t tot = 2u;
        for (int k = 0; k < UNPACK_THREADS / 32; k++) tot = gp_compose(tot, wagg[k]);
        P.agg[jb.tile] = tot;
    }
}

// Persistent: CTA c assembles tiles c, c + G, c + 2G, ... (G = gridDim.x); the
// next tile's residues are in flight (bulk copy into the other stage) while
// this one is assembled.  Dynamic shared memory: [2 mbarriers | 112 B |
// stage 0 (prime 1, prime 2) | stage 1], each prime's part `cap` doubles.
__global__ void __launch_bounds__(UNPACK_THREADS, 3) k_unpack(const DProd* __restrict__ prods,
                                                              const DPlan* __restrict__ plans,
                                                              const Job* __restrict__ jobs, int64_t njobs) {
    extern __shared__ __align__(128) double dsm[];
    __shared__ uint32_t wagg[UNPACK_THREADS / 32];
    __shared__ uint64_t spill[UNPACK_THREADS + 1][2];
    uint64_t* bar = reinterpret_cast<uint64_t*>(dsm);
    uint32_t dsz;
    asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dsz));
    const int cap = (int)((dsz - 128) / 32);
    double* const stg = dsm + 16;
    const int t = threadIdx.x;
    if (t == 0) {
        tma::bar_init(bar);
        tma::bar_init(bar + 1);
    }
    __syncthreads();
    int j = 0;
    for (int64_t ji = blockIdx.x; ji < njobs; ji += gridDim.x, j++) {
        const int s = j & 1;
        double* const st1 = stg + (size_t)s * 2 * cap;
        double* const st2 = st1 + cap;
        const Job jb = jobs[ji];
        const DProd& P = prods[jb.prod];
        const DPlan& pl = plans[P.plan];
        const int64_t N = pl.N;
        const UTile g = unpack_tile(P, jb.tile);
        const int64_t jn = ji + gridDim.x;
        if (t == 0) {
            if (j == 0) unpack_issue(P, N, g, st1, st2, bar + s);
            if (jn < njobs) {  // stage s ^ 1 was last read before the previous tile's spill exchange
                const Job jx = jobs[jn];
                const DProd& Px = prods[jx.prod];
                double* const nx = stg + (size_t)(s ^ 1) * 2 * cap;
                unpack_issue(Px, plans[Px.plan].N, unpack_tile(Px, jx.tile), nx, nx + cap, bar + (s ^ 1));
            }
        }
        if (!tma::bar_wait(bar + s, (uint32_t)(j >> 1) & 1u)) {
            // gave up (counted): let the copy in flight into the other stage land first
            if (jn < njobs) tma::bar_wait(bar + (s ^ 1), (uint32_t)((j + 1) >> 1) & 1u);
            return;
        }
        unpack_assemble(P, pl, jb, g, st1, st2, wagg, spill);
    }
}

// Cross-tile carries of one product (one CTA).  Each thread composes a run of
// tile aggregates, the block scans them, and every tile whose true carry-in is
// 1 gets +1 propagated from its first limb (limbs equal to 2^64-1 wrap to 0).
__device__ __forceinline__ void carry_product(const DProd& P, uint32_t* wagg) {
    const int64_t nt = P.ntl;
    if (nt <= 1) return;  // one tile: no carry crosses a tile boundary
    const int t = threadIdx.x;
    const int64_t per = (nt + blockDim.x - 1) / blockDim.x;
    const int64_t t0 = (int64_t)t * per, t1 = min(t0 + per, nt);
    uint32_t agg = 2u;
    for (int64_t k = t0; k < t1; k++) agg = gp_compose(agg, P.agg[k]);
    const int lane = t & 31, wid = t >> 5;
    uint32_t incl = agg;
    for (int off = 1; off < 32; off <<= 1) {
        uint32_t o = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl = gp_compose(o, incl);
    }
    __syncthreads();
    if (lane == 31) wagg[wid] = incl;
    __syncthreads();
    uint32_t wpre = 2u;
    for (int k = 0; k < wid; k++) wpre = gp_compose(wpre, wagg[k]);
    uint32_t excl = __shfl_up_sync(0xffffffffu, incl, 1);
    if (lane == 0) excl = 2u;
    excl = gp_compose(wpre, excl);
    uint32_t cin = excl & 1u;
    for (int64_t k = t0; k < t1; k++) {
        uint32_t a = P.agg[k];
        if (cin) {
            // the carry stops at the tile's first limb unless that limb is
            // all ones; such tiles are flagged for carry_fix_tile, which
            // walks the run of all-ones limbs with a whole warp
            const int64_t w = k * UNPACK_TL;
            if (P.r[w] != ~0ULL) P.r[w] += 1;
            else P.agg[k] = a | 4u;
        }
        cin = (a & 1u) | ((a >> 1) & cin);
    }
}

__global__ void __launch_bounds__(256) k_carry(const DProd* __restrict__ prods, const Job* __restrict__ jobs,
                                               int64_t njobs) {
    __shared__ uint32_t wagg[8];
    for (int64_t ji = blockIdx.x; ji < njobs; ji += gridDim.x) carry_product(prods[jobs[ji].prod], wagg);
}

// A tile that carry_product flagged (bit 2 of its aggregate): the incoming
// carry runs through the tile's leading all-ones limbs.  One warp: the tile
// is read 32 limbs at a time until the first limb that is not all ones (it
// absorbs the +1), the run before it zeroed; a tile that is all ones passes
// the carry on, which the cross-tile scan already credited to the next tile.
__device__ __forceinline__ void carry_fix_tile(const DProd& P, int64_t tile, int lane) {
    const int64_t w0 = tile * UNPACK_TL, we = min(w0 + (int64_t)UNPACK_TL, P.rn);
    for (int64_t w = w0; w < we; w += 32) {
        const int64_t wl = w + lane;
        const uint64_t v = wl < we ? P.r[wl] : 0ULL;  // past the tile: stops the run
        const unsigned notones = __ballot_sync(0xffffffffu, v != ~0ULL);
        if (notones) {
            const int k = __ffs(notones) - 1;
            if (lane < k) P.r[wl] = 0;
            else if (lane == k && wl < we) P.r[wl] = v + 1;
            break;
        }
        P.r[wl] = 0;  // all 32 are all ones (and inside the tile)
    }
}

// Flagged tiles, one warp per tile (most tiles are left at once).  Jobs are
// the unpack's (product, tile) list.
__global__ void __launch_bounds__(256) k_carry_fix(const DProd* __restrict__ prods, const Job* __restrict__ jobs,
                                                   int64_t njobs) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t ji = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); ji < njobs; ji += nw) {
        const Job jb = jobs[ji];
        const DProd& P = prods[jb.prod];
        if (P.ntl <= 1 || !(P.agg[jb.tile] & 4u)) continue;
        carry_fix_tile(P, jb.tile, lane);
    }
}

// ---------------------------------------------------------------------------
// Work-queue execution: one persistent launch runs a whole batch.  Each CTA
// claims the next queue positions (an atomic counter), waits until the job's
// product has finished its previous pipeline step (per product and step, a
// count of finished jobs against the count the step has), runs the job and
// counts it finished.  Positions are claimed in pipeline-step order, so every
// job a CTA waits for was claimed earlier by a CTA that is running: the
// earliest unfinished job never waits, and the queue drains.  Waits are
// bounded: one that gives up counts a fault and raises the abort flag, on
// which every CTA leaves.

__device__ __forceinline__ int queue_step(int kind, const Job& jb, int npass) {
    switch (kind) {
        case JK_FWD:
        case JK_FWD_TMA: return (jb.sub >> 8) & 0xff;
        case JK_PWR:
        case JK_PWR_SPLIT:
        case JK_PWR_KEEP: return npass - 1;
        case JK_REV:
        case JK_REV_TMA: return 2 * npass - 2 - ((jb.sub >> 8) & 0xff);
        case JK_UNPACK: return 2 * npass - 1;
        default: return 2 * npass;  // JK_CARRY
    }
}

__device__ __forceinline__ int queue_entry(const QLaunch* __restrict__ ql, int nl, int64_t g) {
    int lo = 0, hi = nl - 1;  // last entry with qstart <= g
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (ql[mid].qstart <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ bool queue_aborted(const QState* qs) {
    return *reinterpret_cast<const volatile unsigned int*>(&qs->abort) != 0u;
}

// Waits (bounded: about 2^31 SM clocks, a second) until *cnt >= want.
__device__ __forceinline__ bool queue_wait(const uint32_t* cnt, uint32_t want, QState* qs) {
    if (ld_acquire(cnt) >= want) return true;
    const long long t0 = clock64();
    for (;;) {
        __nanosleep(100);
        if (ld_acquire(cnt) >= want) return true;
        if (queue_aborted(qs)) return false;
        if (clock64() - t0 > (1LL << 31)) {
            atomicAdd(&g_nbg_faults, 1u);
            atomicExch(&qs->abort, 1u);
            return false;
        }
    }
}

// One unpack tile, its residues staged by bulk copy into `reg` (one stage).
__device__ __forceinline__ bool job_unpack(const DProd* __restrict__ prods, const DPlan* __restrict__ plans,
                                           const Job& jb, double* reg, uint64_t* bar, uint32_t& phase,
                                           uint32_t* wagg, uint64_t (*spill)[2]) {
    const DProd& P = prods[jb.prod];
    const DPlan& pl = plans[P.plan];
    const UTile g = unpack_tile(P, jb.tile);
    const int cap = (int)unpack_stage_doubles(P.bch);
    double* const st1 = reg;
    double* const st2 = reg + cap;
    if (threadIdx.x == 0) unpack_issue(P, pl.N, g, st1, st2, bar);
    if (!tma::bar_wait(bar, phase)) return false;
    phase ^= 1u;
    unpack_assemble(P, pl, jb, g, st1, st2, wagg, spill);
    return true;
}

// The cross-tile carries of one product and the tiles they flag.
__device__ __forceinline__ void job_carry(const DProd& P, uint32_t* wagg) {
    if (P.ntl <= 1) return;
    carry_product(P, wagg);
    __syncthreads();  // the flags and +1s are written
    const int lane = threadIdx.x & 31;
    for (int64_t k0 = (int64_t)(threadIdx.x >> 5) * 32; k0 < P.ntl; k0 += (int64_t)(blockDim.x >> 5) * 32) {
        const int64_t k = k0 + lane;
        unsigned f = __ballot_sync(0xffffffffu, k < P.ntl && (P.agg[k] & 4u));
        for (; f; f &= f - 1) carry_fix_tile(P, k0 + __ffs(f) - 1, lane);
    }
}

// Publishes this CTA's finished jobs of one (product, step): their column
// tiles' bulk stores have landed, and their results are visible before the
// count that releases them.
__device__ __forceinline__ void queue_publish(uint32_t* done, int64_t pend_c, uint32_t& pend_n) {
    if (pend_n == 0) return;
    tma::stores_done();
    asm volatile("fence.proxy.async.global;" ::: "memory");
    __threadfence();
    atomicAdd(done + pend_c, pend_n);
    pend_n = 0;
}

// The queue kernel's dynamic shared memory, named at file scope so that the
// job functions below address it as shared memory without a pointer argument:
// [mbarrier | 120 B | region].
extern __shared__ __align__(128) double q_dsm[];

// One job of each kind, each compiled as a function of its own: a job then has
// the kernel's whole register budget, and only the queue loop's few values are
// saved around the call.  Column and unpack jobs return the mbarrier phase
// after the job in bit 0 and success in bit 1.
template <bool ODD>
__device__ __noinline__ void qj_fwd(const DProd* __restrict__ prods, const DPlan* __restrict__ plans, Job jb) {
    job_fwd<ODD>(prods, plans, jb, q_dsm + 16);
}
template <bool ODD>
__device__ __noinline__ void qj_rev(const DProd* __restrict__ prods, const DPlan* __restrict__ plans, Job jb) {
    job_rev<ODD>(prods, plans, jb, q_dsm + 16);
}
template <bool SPLIT, bool KEEPB, bool ODD>
__device__ __noinline__ void qj_pwr(const DProd* __restrict__ prods, const DPlan* __restrict__ plans, Job jb) {
    job_pwr<SPLIT, KEEPB, ODD>(prods, plans, jb, q_dsm + 16);
}
template <bool FWD, bool ODD>
__device__ __noinline__ uint32_t qj_col(const DProd* __restrict__ prods, const DPlan* __restrict__ plans, Job jb,
                                        uint32_t phase) {
    const bool ok = job_col_tma<FWD, ODD>(prods, plans, jb, q_dsm + 16, reinterpret_cast<uint64_t*>(q_dsm), phase);
    return (phase & 1u) | (ok ? 2u : 0u);
}
__device__ __noinline__ uint32_t qj_unpack(const DProd* __restrict__ prods, const DPlan* __restrict__ plans, Job jb,
                                           uint32_t phase) {
    __shared__ uint32_t wagg[UNPACK_THREADS / 32];
    __shared__ uint64_t spill[UNPACK_THREADS + 1][2];
    const bool ok = job_unpack(prods, plans, jb, q_dsm + 16, reinterpret_cast<uint64_t*>(q_dsm), phase, wagg, spill);
    return (phase & 1u) | (ok ? 2u : 0u);
}
__device__ __noinline__ void qj_carry(const DProd* __restrict__ prods, Job jb) {
    __shared__ uint32_t wagg[UNPACK_THREADS / 32];
    job_carry(prods[jb.prod], wagg);
}

// The region holds the largest tile set of the batch's launches and one
// unpack stage.  A CTA
// claims `chunk` consecutive queue positions at a time (one atomic); thread 0
// checks each job's dependency (an acquire only when the count it needs was
// not seen complete before) and publishes finished jobs in runs of one
// (product, step), always before it waits, so no CTA waits on a count that
// a waiting CTA holds back.
__global__ void __launch_bounds__(PASS_THREADS, 3) k_queue(const DProd* __restrict__ prods,
                                                          const DPlan* __restrict__ plans,
                                                          const Job* __restrict__ jobs,
                                                          const QLaunch* __restrict__ ql, int nl, QState* qs,
                                                          uint32_t* done, const uint32_t* __restrict__ need,
                                                          int chunk) {
    __shared__ int64_t s_g;
    __shared__ int s_n, s_k, s_ok;
    uint64_t* bar = reinterpret_cast<uint64_t*>(q_dsm);
    const int t = threadIdx.x;
    if (t == 0) tma::bar_init(bar);
    __syncthreads();
    uint32_t phase = 0;
    const int64_t total = ql[nl].qstart;
    // thread 0: the (product, step) counter of finished, unpublished jobs, and
    // the last dependency counter seen complete
    int64_t pend_c = -1, seen_c = -1;
    uint32_t pend_n = 0;
    int k = 0;
    for (;;) {
        if (t == 0) {
            int64_t g = -1;
            int n = 0;
            if (!queue_aborted(qs)) {
                g = (int64_t)atomicAdd(&qs->head, (unsigned long long)chunk);
                if (g < total) {
                    n = (int)min((int64_t)chunk, total - g);
                    k = queue_entry(ql, nl, g);
                } else {
                    g = -1;
                }
            }
            s_g = g;
            s_n = n;
        }
        __syncthreads();
        const int64_t g0 = s_g;
        const int n = s_n;
        if (g0 < 0) break;
        bool ok = true;
        for (int i = 0; i < n; i++) {
            const int64_t g = g0 + i;
            if (t == 0) {
                while (ql[k + 1].qstart <= g) k++;
                const Job jq = jobs[ql[k].off + (g - ql[k].qstart)];
                const int st = queue_step(ql[k].kind, jq, prods[jq.prod].npass);
                int good = 1;
                if (st > 0) {
                    const int64_t c = (int64_t)jq.prod * QSTEPS + st - 1;
                    if (c != seen_c) {
                        if (ld_acquire(done + c) < need[c]) {
                            queue_publish(done, pend_c, pend_n);  // never wait holding finished jobs back
                            good = queue_wait(done + c, need[c], qs) ? 1 : 0;
                        }
                        seen_c = c;
                    }
                }
                // the previous job's bulk store has read shared memory, and what
                // the acquire made visible is visible to this job's bulk loads
                tma::stores_read();
                asm volatile("fence.proxy.async.global;" ::: "memory");
                s_k = k;
                s_ok = good;
            }
            __syncthreads();
            if (!s_ok) {
                ok = false;
                break;
            }
            const QLaunch L = ql[s_k];
            const Job jb = jobs[L.off + (g - L.qstart)];
            uint32_t r = 2u | phase;
            const bool odd = L.odd != 0;
            switch (L.kind) {
                case JK_FWD:
                    if (odd) qj_fwd<true>(prods, plans, jb);
                    else qj_fwd<false>(prods, plans, jb);
                    break;
                case JK_FWD_TMA:
                    r = odd ? qj_col<true, true>(prods, plans, jb, phase) : qj_col<true, false>(prods, plans, jb, phase);
                    break;
                case JK_PWR:
                    if (odd) qj_pwr<false, false, true>(prods, plans, jb);
                    else qj_pwr<false, false, false>(prods, plans, jb);
                    break;
                case JK_PWR_SPLIT:
                    if (odd) qj_pwr<true, false, true>(prods, plans, jb);
                    else qj_pwr<true, false, false>(prods, plans, jb);
                    break;
                case JK_PWR_KEEP:
                    if (odd) qj_pwr<false, true, true>(prods, plans, jb);
                    else qj_pwr<false, true, false>(prods, plans, jb);
                    break;
                case JK_REV:
                    if (odd) qj_rev<true>(prods, plans, jb);
                    else qj_rev<false>(prods, plans, jb);
                    break;
                case JK_REV_TMA:
                    r = odd ? qj_col<false, true>(prods, plans, jb, phase)
                            : qj_col<false, false>(prods, plans, jb, phase);
                    break;
                case JK_UNPACK: r = qj_unpack(prods, plans, jb, phase); break;
                case JK_CARRY: qj_carry(prods, jb); break;
                default: break;
            }
            phase = r & 1u;
            ok = (r & 2u) != 0;
            // this job's generic shared-memory accesses come before the next
            // job's bulk copies into the region; every thread's stores are issued
            tma::fence_async();
            ok = __syncthreads_and(ok) != 0;
            if (!ok) break;
            if (t == 0) {
                const int64_t c = (int64_t)jb.prod * QSTEPS + queue_step(L.kind, jb, prods[jb.prod].npass);
                if (c != pend_c) {
                    queue_publish(done, pend_c, pend_n);
                    pend_c = c;
                }
                pend_n++;
            }
        }
        if (!ok) {
            if (t == 0) atomicExch(&qs->abort, 1u);
            break;
        }
        if (t == 0) queue_publish(done, pend_c, pend_n);
    }
    if (t == 0) tma::stores_done();
}

// need[prod * QSTEPS + step] += 1 for every queued job.
__global__ void k_qcount(const DProd* __restrict__ prods, const Job* __restrict__ jobs,
                         const QLaunch* __restrict__ ql, int nl, uint32_t* need) {
    const int64_t total = ql[nl].qstart;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < total;
         g += (int64_t)gridDim.x * blockDim.x) {
        const int k = queue_entry(ql, nl, g);
        const Job jb = jobs[ql[k].off + (g - ql[k].qstart)];
        const int s = queue_step(ql[k].kind, jb, prods[jb.prod].npass);
        atomicAdd(need + (size_t)jb.prod * QSTEPS + s, 1u);
    }
}

// ---------------------------------------------------------------------------
// Standalone pack and pointwise (the transform-level entry points).
__global__ void k_pack(double* __restrict__ x, int64_t N, const uint64_t* __restrict__ limbs, int64_t n, int b,
                       int64_t nch) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = pack_chunk(limbs, n, b, nch, i);
}
__global__ void k_pointwise(double* __restrict__ xa, const double* __restrict__ xb, int64_t N, int f) {
    const Fp F = fpctx(f);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
        xa[i] = fp_mulmod(xa[i], xb[i], F);
}
// top-limb bit lengths for device batches: bits[2k] / bits[2k+1] of operand a / b
__global__ void k_topbits(const DProd* __restrict__ prods, int64_t count, int64_t* __restrict__ bits) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < count; k += (int64_t)gridDim.x * blockDim.x) {
        const DProd& P = prods[k];
        uint64_t ta = P.a[P.m - 1];
        bits[2 * k] = 64 * (P.m - 1) + (ta ? 64 - __clzll((long long)ta) : 0);
        uint64_t tb = P.b[P.n - 1];
        bits[2 * k + 1] = 64 * (P.n - 1) + (tb ? 64 - __clzll((long long)tb) : 0);
    }
}

// ---------------------------------------------------------------------------
// Twiddle tables: tw[(t-1)*Q + j] = omega^e, e = (N/L)*t*j (< N), as
//   minbal(mulmod(HI[e >> 12], LO[e & 4095]))
// where HI/LO are exact minimal-balanced powers built on the host.  Both
// factors are <= p/2, so the mulmod is exact and |r| < p; minbal then yields
// the unique representative in [-p/2, p/2], the value fp_twiddles stores.
__global__ void k_twiddle(double* __restrict__ out, int m, int64_t Q, int64_t step, const double* __restrict__ hi,
                          const double* __restrict__ lo, int f) {
    const Fp F = fpctx(f);
    const int64_t total = (int64_t)(m - 1) * Q;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int64_t t = idx / Q + 1, j = idx - (t - 1) * Q;
        int64_t e = step * t * j;
        double v = fp_mulmod(hi[e >> 12], lo[e & 4095], F);
        out[idx] = fp_minbal(v, F);
    }
}

// ---------------------------------------------------------------------------
// Host-side launch helpers

// Written once per kernels_init with its final value, so a concurrent reader
// never sees a partial result.
static std::atomic<int> g_smem_optin{0};
static std::atomic<int> g_num_sms{148};

cudaError_t kernels_init(double p1, double p2) {
    Fp h[2] = {{p1, 1.0 / p1}, {p2, 1.0 / p2}};
    cudaError_t e = cudaMemcpyToSymbol(c_fp, h, sizeof h);
    if (e != cudaSuccess) return e;
    // Garner constant g = p1^-1 mod p2 (canonical) and g/p2 (fpntt.jl:879-880)
    const uint64_t P1 = P1_U, P2 = P2_U;
    // invmod by Fermat with 128-bit products
    unsigned __int128 r = 1, a = P1 % P2;
    uint64_t ex = P2 - 2;
    while (ex) {
        if (ex & 1) r = (r * a) % P2;
        a = (a * a) % P2;
        ex >>= 1;
    }
    double g[2];
    g[0] = (double)(uint64_t)r;
    g[1] = g[0] / p2;
    e = cudaMemcpyToSymbol(c_garner, g, sizeof g);
    if (e != cudaSuccess) return e;
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const void* ks[] = {(const void*)k_fwd<3, true>, (const void*)k_fwd<4, true>, (const void*)k_fwd<3, false>,
                        (const void*)k_fwd<4, false>,
                        (const void*)k_pwr<false, false, true>, (const void*)k_pwr<true, false, true>,
                        (const void*)k_pwr<false, true, true>, (const void*)k_pwr<false, false, false>,
                        (const void*)k_pwr<true, false, false>, (const void*)k_pwr<false, true, false>,
                        (const void*)k_rev<3, true>, (const void*)k_rev<4, true>, (const void*)k_rev<3, false>,
                        (const void*)k_rev<4, false>, (const void*)k_unpack,
                        (const void*)k_col_tma<3, true, true>, (const void*)k_col_tma<4, true, true>,
                        (const void*)k_col_tma<3, false, true>, (const void*)k_col_tma<4, false, true>,
                        (const void*)k_col_tma<3, true, false>, (const void*)k_col_tma<4, true, false>,
                        (const void*)k_col_tma<3, false, false>, (const void*)k_col_tma<4, false, false>,
                        (const void*)k_queue};
    for (const void* k : ks) {
        cudaFuncAttributes fa;
        e = cudaFuncGetAttributes(&fa, k);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
        if (e != cudaSuccess) return e;
    }
    int nsm = 0;
    e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    g_num_sms.store(nsm);
    g_smem_optin.store(optin - 8192);  // headroom for the largest static allocation (k_unpack, 4.1 KB)
    return cudaSuccess;
}

int kernels_smem_optin() { return g_smem_optin.load(); }

cudaError_t kernels_take_faults(unsigned int* n) {
    unsigned int zero = 0;
    cudaError_t e = cudaMemcpyFromSymbol(n, g_nbg_faults, sizeof(unsigned int));
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(g_nbg_faults, &zero, sizeof zero);
}

cudaError_t kernels_binary_version(int* version) {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, (const void*)k_pwr<false, false, false>);
    if (e != cudaSuccess) return e;
    *version = fa.binaryVersion;
    return cudaSuccess;
}

cudaError_t launch_jobs(int kind, const DProd* prods, const DPlan* plans, const JobSrc& src, int64_t njobs,
                        size_t smem, int grid_cap, cudaStream_t st, bool odd) {
    // the kernels read an explicit job list (batches expand theirs on the device first)
    if (src.mode != JM_LIST) return cudaErrorInvalidValue;
    const Job* jobs = src.list;
    if (njobs <= 0) return cudaSuccess;
    int64_t grid64 = njobs;
    if (kind == JK_FWD || kind == JK_REV || kind == JK_FWD_TMA || kind == JK_REV_TMA) {
        // up to 8 consecutive jobs per CTA while keeping >= 4 waves of 3 CTAs per SM
        const int64_t k = std::max<int64_t>(1, std::min<int64_t>(8, njobs / (148 * 3 * 4)));
        grid64 = (njobs + k - 1) / k;
    }
    if (grid_cap > 0 && grid64 > grid_cap) grid64 = grid_cap;
    if (grid64 > 0x7fffffff) grid64 = 0x7fffffff;
    const unsigned grid = (unsigned)grid64;
#define NBG_ODD(KERNEL, ...)                                                                      \
    do {                                                                                          \
        if (odd) KERNEL<__VA_ARGS__, true><<<grid, 256, smem, st>>>(prods, plans, jobs, njobs);   \
        else KERNEL<__VA_ARGS__, false><<<grid, 256, smem, st>>>(prods, plans, jobs, njobs);      \
    } while (0)
    const bool c4 = smem <= COL4_MAX_SMEM, c4t = smem <= COL4_MAX_SMEM_TMA;
    switch (kind) {
        case JK_FWD:
            if (c4) NBG_ODD(k_fwd, 4);
            else NBG_ODD(k_fwd, 3);
            break;
        // passes with radix-3/5/7 rounds take the 80-register build whatever
        // their tile size (the 64-register one spills there)
        case JK_FWD_TMA:
            if (c4t && !odd) NBG_ODD(k_col_tma, 4, true);
            else NBG_ODD(k_col_tma, 3, true);
            break;
        case JK_REV_TMA:
            if (c4t && !odd) NBG_ODD(k_col_tma, 4, false);
            else NBG_ODD(k_col_tma, 3, false);
            break;
        case JK_PWR: NBG_ODD(k_pwr, false, false); break;
        case JK_PWR_SPLIT: NBG_ODD(k_pwr, true, false); break;
        case JK_PWR_KEEP: NBG_ODD(k_pwr, false, true); break;
        case JK_REV:
            if (c4) NBG_ODD(k_rev, 4);
            else NBG_ODD(k_rev, 3);
            break;
        case JK_UNPACK: {
            // persistent: as many CTAs as fit on the GPU at once, each streaming its tiles
            int nb = 0;
            cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_unpack, UNPACK_THREADS, smem);
            if (e != cudaSuccess) return e;
            const unsigned g = (unsigned)std::min<int64_t>(grid, (int64_t)std::max(nb, 1) * g_num_sms.load());
            k_unpack<<<g, UNPACK_THREADS, smem, st>>>(prods, plans, jobs, njobs);
            break;
        }
        case JK_CARRY: k_carry<<<grid, 256, 0, st>>>(prods, jobs, njobs); break;
        case JK_CARRYFIX: {
            // one warp per tile (most tiles are left at once)
            const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>((njobs + 7) / 8, 148 * 32));
            k_carry_fix<<<g, 256, 0, st>>>(prods, jobs, njobs);
            break;
        }
        default: return cudaErrorInvalidValue;
    }
#undef NBG_ODD
    return cudaGetLastError();
}

cudaError_t launch_qcount(const DProd* prods, const Job* jobs, const QLaunch* ql, int nl, int64_t total,
                          uint32_t* need, cudaStream_t st) {
    if (total <= 0) return cudaSuccess;
    const unsigned grid = (unsigned)std::min<int64_t>((total + 255) / 256, 148 * 8);
    k_qcount<<<grid, 256, 0, st>>>(prods, jobs, ql, nl, need);
    return cudaGetLastError();
}

cudaError_t queue_grid(size_t smem, int* grid) {
    int nb = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_queue, PASS_THREADS, smem);
    if (e != cudaSuccess) return e;
    *grid = std::max(nb, 1) * g_num_sms.load();
    return cudaSuccess;
}

cudaError_t launch_queue(const DProd* prods, const DPlan* plans, const Job* jobs, const QLaunch* ql, int nl,
                         QState* qs, uint32_t* done, const uint32_t* need, size_t smem, int grid, int chunk,
                         cudaStream_t st) {
    k_queue<<<(unsigned)grid, PASS_THREADS, smem, st>>>(prods, plans, jobs, ql, nl, qs, done, need, chunk);
    return cudaGetLastError();
}

// One thread per job: find the launch owning job g, decode it, store it.
__global__ void __launch_bounds__(256) k_expand(const ExpandEntry* __restrict__ entries, int nentries,
                                                Job* __restrict__ out, int64_t total) {
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < total;
         g += (int64_t)gridDim.x * blockDim.x) {
        int lo = 0, hi = nentries - 1;  // last entry with begin <= g
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (entries[mid].begin <= g) lo = mid;
            else hi = mid - 1;
        }
        out[g] = job_at(entries[lo].src, g - entries[lo].begin);
    }
}

cudaError_t launch_expand(const ExpandEntry* entries, int nentries, Job* out, int64_t total, cudaStream_t st) {
    if (total <= 0 || nentries <= 0) return cudaSuccess;
    int64_t b = (total + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    k_expand<<<(unsigned)b, 256, 0, st>>>(entries, nentries, out, total);
    return cudaGetLastError();
}

static unsigned grid_for(int64_t n) {
    int64_t b = (n + 255) / 256;
    if (b > 148 * 32) b = 148 * 32;
    return (unsigned)(b < 1 ? 1 : b);
}

cudaError_t launch_pack(double* x, int64_t N, const uint64_t* limbs, int64_t n, int b, int64_t nch, cudaStream_t st) {
    k_pack<<<grid_for(N), 256, 0, st>>>(x, N, limbs, n, b, nch);
    return cudaGetLastError();
}
cudaError_t launch_pointwise(double* xa, const double* xb, int64_t N, int f, cudaStream_t st) {
    k_pointwise<<<grid_for(N), 256, 0, st>>>(xa, xb, N, f);
    return cudaGetLastError();
}
cudaError_t launch_topbits(const DProd* prods, int64_t count, int64_t* bits, cudaStream_t st) {
    k_topbits<<<grid_for(count), 256, 0, st>>>(prods, count, bits);
    return cudaGetLastError();
}

cudaError_t launch_twiddle(double* out, int m, int64_t Q, int64_t step, const double* hi, const double* lo, int f,
                           cudaStream_t st) {
    int64_t total = (int64_t)(m - 1) * Q;
    int64_t blocks = (total + 255) / 256;
    if (blocks > 148 * 64) blocks = 148 * 64;
    if (blocks < 1) blocks = 1;
    k_twiddle<<<(unsigned)blocks, 256, 0, st>>>(out, m, Q, step, hi, lo, f);
    return cudaGetLastError();
}

}  // namespace nbg
