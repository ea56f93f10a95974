/*
 * fpntt_oracle.c — CPU restatement of the reference's two-prime Float64 NTT
 * multiplication engine (NativeBigInt.jl, src/fpntt.jl), used ONLY as the test
 * oracle and as the timed CPU baseline.  Nothing in the product library links
 * or calls this file.
 *
 * Parity status: pinned.  The restatement is checked (tests/test_oracle.py)
 * against (1) the reference's own known-answer tables from
 * test/test_fpntt.jl (ntt_len table, prime identities, 2-adic cap, root
 * orders), (2) its property tests (field-range sweep, round trip,
 * convolution, Garner CRT, adversarial operands, b = 49 all-ones), and
 * (3) GMP 6.3 mpn_mul / mpn_sqr, the same arithmetic Julia's BigInt uses.
 * Julia itself is not available, so the reference cannot be executed.
 *
 * Every routine is a scalar restatement.  The reference's SIMD paths are
 * elementwise identical to its scalar paths (test/test_fpntt.jl:70-82 pins
 * this), so each intermediate double here equals the reference's bit for
 * bit, provided the compiler neither contracts a*b+c nor reassociates:
 * build with -O2 -ffp-contract=off -fno-fast-math.
 *
 * With -DORC_COUNT every DADD/DMUL/DFMA of the transform, pointwise and
 * unpack stages bumps orc_op_count, giving the algorithmic FP64 op count of
 * the reference schedule.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

#ifdef ORC_COUNT
static volatile uint64_t orc_op_count_v = 0;
#define OPS(k) (orc_op_count_v += (uint64_t)(k))
#else
#define OPS(k) ((void)0)
#endif

uint64_t orc_op_count(void) {
#ifdef ORC_COUNT
    return orc_op_count_v;
#else
    return 0;
#endif
}
void orc_op_count_reset(void) {
#ifdef ORC_COUNT
    orc_op_count_v = 0;
#endif
}

/* ------------------------------------------------------------------------ */
/* Primes and contexts: src/fpntt.jl:50-79                                   */

#define NPRIMES 2
static const uint64_t ORC_P[NPRIMES] = {65205ULL * (1ULL << 34) + 1ULL,   /* FP_CTX1 :78 */
                                        4095ULL * (1ULL << 38) + 1ULL};   /* FP_CTX2 :79 */
static const int ORC_TWOADIC[NPRIMES] = {34, 38};
/* odd prime factors of p-1 (the 2 is handled separately), :78-79 */
static const uint64_t ORC_FACS[NPRIMES][5] = {{2, 3, 5, 7, 23}, {2, 3, 5, 7, 13}};

static const double FP_MAGIC = 6755399441055744.0; /* 1.5 * 2^52, :81 */

static uint64_t mulmod_u(uint64_t a, uint64_t b, uint64_t p) { return (uint64_t)(((u128)a * b) % p); }
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
static uint64_t invmod_u(uint64_t a, uint64_t p) { return powmod_u(a, p - 2, p); } /* p prime */

/* fp_generator :50-56: smallest g in 3..63 with g^((p-1)/q) != 1 for all q | p-1 */
static uint64_t orc_gen[NPRIMES];
static void orc_init_gens(void) {
    static int done = 0;
    if (done) return;
    for (int f = 0; f < NPRIMES; f++) {
        uint64_t p = ORC_P[f];
        for (uint64_t g = 3; g <= 63; g++) {
            int ok = 1;
            for (int i = 0; i < 5; i++)
                if (powmod_u(g, (p - 1) / ORC_FACS[f][i], p) == 1) ok = 0;
            if (ok) { orc_gen[f] = g; break; }
        }
    }
    done = 1;
}
uint64_t orc_prime(int f) { return ORC_P[f]; }
uint64_t orc_generator(int f) { orc_init_gens(); return orc_gen[f]; }
int orc_two_adicity(int f) { return ORC_TWOADIC[f]; }

/* ------------------------------------------------------------------------ */
/* Field arithmetic: src/fpntt.jl:81-121                                     */

static inline double fp_round(double v) { OPS(2); return (v + FP_MAGIC) - FP_MAGIC; }       /* :83 */
static inline double fp_reduce(double x, double P) {                                       /* :88-91 */
    OPS(2);
    double q = fp_round(x * (1.0 / P));
    return fma(q, -P, x);
}
static inline double fp_mulmod3(double x, double y, double P) {                           /* :101-105 */
    OPS(3);
    double h = x * y;
    double l = fma(x, y, -h);
    return fp_reduce(h, P) + l;
}
static inline double fp_mulmod4(double x, double w, double wpinv, double P) {             /* :106-111 */
    OPS(5);
    double h = x * w;
    double l = fma(x, w, -h);
    double q = fp_round(x * wpinv);
    return fma(q, -P, h) + l;
}
static inline double fp_minbal(double x, double P) {                                      /* :118-119 */
    return (x > P / 2) ? x - P : ((x < -P / 2) ? x + P : x);
}

double orc_fp_round(double v) { return fp_round(v); }
double orc_fp_reduce(double x, int f) { return fp_reduce(x, (double)ORC_P[f]); }
double orc_fp_mulmod3(double x, double y, int f) { return fp_mulmod3(x, y, (double)ORC_P[f]); }
double orc_fp_mulmod4(double x, double w, double wp, int f) { return fp_mulmod4(x, w, wp, (double)ORC_P[f]); }
double orc_fp_minbal(double x, int f) { return fp_minbal(x, (double)ORC_P[f]); }

/* ------------------------------------------------------------------------ */
/* Constants and tables: src/fpntt.jl:123-186                                */

/* fp_dft5_consts :127-136 */
static void fp_dft5_consts(uint64_t c, double P, uint64_t p, double out[4]) {
    double inv2 = (double)invmod_u(2, p);
    double c1 = fp_reduce((double)c, P);
    double c2 = fp_mulmod3(c1, c1, P), c3 = fp_mulmod3(c2, c1, P), c4 = fp_mulmod3(c3, c1, P);
    double inv4 = fp_mulmod3(inv2, inv2, P);
    out[0] = fp_minbal(-inv4, P);
    out[1] = fp_minbal(fp_mulmod3((c1 + c4) - (c2 + c3), inv4, P), P);
    out[2] = fp_minbal(fp_mulmod3(c1 - c4, inv2, P), P);
    out[3] = fp_minbal(fp_mulmod3(c2 - c3, inv2, P), P);
}

/* fp_dft7_consts :151-168 */
static void fp_dft7_consts(uint64_t c, double P, uint64_t p, double out[8]) {
    double inv2 = (double)invmod_u(2, p);
    double inv3 = (double)invmod_u(3, p);
    double cj[7];
    for (int j = 1; j <= 6; j++) cj[j] = (double)powmod_u(c, (uint64_t)j, p);
#define A_(j) fp_mulmod3(cj[j] + cj[7 - (j)], inv2, P)
#define B_(j) fp_mulmod3(cj[j] - cj[7 - (j)], inv2, P)
    double a0 = A_(1), a1 = A_(3), a2 = A_(2);
    double b0 = B_(1), b1 = B_(3), b2 = B_(2);
#undef A_
#undef B_
    double bp0 = fp_minbal(fp_mulmod3(a0 - a2, inv3, P), P);
    double bp1 = fp_minbal(fp_mulmod3(a1 - a2, inv3, P), P);
    double n0 = fp_minbal(fp_mulmod3(b0 - b2, inv3, P), P);
    double n1 = fp_minbal(fp_mulmod3(b1 + b2, inv3, P), P);
    out[0] = fp_minbal(fp_mulmod3((a0 + a1) + a2, inv3, P), P);
    out[1] = bp0;
    out[2] = bp1;
    out[3] = fp_minbal(bp0 + bp1, P);
    out[4] = fp_minbal(fp_mulmod3((b0 + b2) - b1, inv3, P), P);
    out[5] = n0;
    out[6] = n1;
    out[7] = fp_minbal(n0 + n1, P);
}

/* fp_twiddles :173-186: minimal-balanced r^0..r^(n-1), 8-lane stride chain */
static double *fp_twiddles(uint64_t r, int64_t n, double P, uint64_t p) {
    int64_t np = ((n + 7) / 8) * 8;
    double *t = (double *)malloc(sizeof(double) * (size_t)(np > 0 ? np : 8));
    double r8 = fp_reduce((double)powmod_u(r, 8, p), P);
    double r8p = r8 / P;
    double v[8];
    for (int k = 0; k < 8; k++) v[k] = fp_reduce((double)powmod_u(r, (uint64_t)k, p), P);
    for (int64_t j = 0; j < np; j += 8) {
        for (int k = 0; k < 8; k++) {
            v[k] = fp_minbal(v[k], P);
            t[j + k] = v[k];
            v[k] = fp_mulmod4(v[k], r8, r8p, P);
        }
    }
    return t; /* only the first n entries are meaningful (resize! :184) */
}

/* ------------------------------------------------------------------------ */
/* Plans: src/fpntt.jl:188-271                                               */

typedef struct {
    int m;         /* radix: 2, 3, 4, 5, 7 */
    int64_t span;  /* block size L the butterflies run within (radix-2: 2) */
    int64_t Q;     /* L / m, butterfly stride */
    double rot[8]; /* DFT combine constants (radix-4: rot[0] = wi) */
    double *tw;    /* (m-1) tables of twlen entries, table t-1 at tw + (t-1)*twlen */
    int64_t twlen;
} orc_stage;

typedef struct {
    int f;            /* prime index 0/1 */
    int64_t N, N2;    /* N2 = 2^k */
    double ninv, ninvp;
    int nst;
    orc_stage st[48];
} orc_plan;

/* build_fp_4 :199-211 (stored with span L = 4q; the reference stores span N2
 * and walks the L-blocks inside it, which visits the same butterflies) */
static void build_fp_4(orc_stage *s, const double *table, int64_t N2, int64_t L, double wi) {
    int64_t q = L >> 2, st = N2 / L, len = q > 8 ? q : 8;
    s->m = 4;
    s->span = L;
    s->Q = q;
    memset(s->rot, 0, sizeof s->rot);
    s->rot[0] = wi;
    s->twlen = len;
    s->tw = (double *)malloc(sizeof(double) * 3 * (size_t)len);
    for (int64_t j = 0; j < len; j++) {
        int64_t jm = j < q ? j : j % q;
        s->tw[0 * len + j] = table[jm * st];
        s->tw[1 * len + j] = table[2 * jm * st];
        s->tw[2 * len + j] = table[3 * jm * st];
    }
}

/* build_fp_odd :213-225 */
static void build_fp_odd(orc_stage *s, int m, int64_t span, uint64_t root, double P, uint64_t p) {
    int64_t Q = span / m;
    uint64_t c = powmod_u(root, (uint64_t)Q, p);
    s->m = m;
    s->span = span;
    s->Q = Q;
    memset(s->rot, 0, sizeof s->rot);
    if (m == 5) fp_dft5_consts(c, P, p, s->rot);
    else if (m == 7) fp_dft7_consts(c, P, p, s->rot);
    else
        for (int r = 1; r <= m - 1; r++) s->rot[r - 1] = fp_reduce((double)powmod_u(c, (uint64_t)r, p), P);
    s->twlen = Q;
    s->tw = (double *)malloc(sizeof(double) * (size_t)(m - 1) * (size_t)Q);
    for (int r = 1; r <= m - 1; r++) {
        uint64_t wr = powmod_u(root, (uint64_t)r, p);
        double *t = fp_twiddles(wr, Q, P, p);
        memcpy(s->tw + (size_t)(r - 1) * (size_t)Q, t, sizeof(double) * (size_t)Q);
        free(t);
    }
}

static int ctz64(uint64_t x) { return x ? __builtin_ctzll(x) : 64; }

/* build_fp_plan :236-271.  Returns NULL if N is not an admissible length. */
orc_plan *orc_plan_build(int64_t N, int f) {
    orc_init_gens();
    if (N < 1 || f < 0 || f >= NPRIMES) return NULL;
    uint64_t p = ORC_P[f];
    double P = (double)p;
    int k = ctz64((uint64_t)N);
    int64_t m = N >> k;
    /* :242-244 preconditions */
    static const int64_t okm[] = {1, 3, 5, 7, 9, 15, 21, 35, 45, 63, 105, 315};
    int okm_hit = 0;
    for (int i = 0; i < 12; i++) okm_hit |= (m == okm[i]);
    if (!okm_hit || !(m == 1 || k >= 2) || k > ORC_TWOADIC[f]) return NULL;
    if ((p - 1) % (uint64_t)N != 0) return NULL;
    uint64_t w = powmod_u(orc_gen[f], (p - 1) / (uint64_t)N, p);

    orc_plan *pl = (orc_plan *)calloc(1, sizeof(orc_plan));
    pl->f = f;
    pl->N = N;
    int64_t span = N;
    uint64_t r = w;
    static const int mfs[4] = {7, 5, 3, 3}; /* :253 */
    for (int i = 0; i < 4; i++) {
        int mf = mfs[i];
        if (m % mf == 0) {
            build_fp_odd(&pl->st[pl->nst++], mf, span, r, P, p);
            r = powmod_u(r, (uint64_t)mf, p);
            span /= mf;
            m /= mf;
        }
    }
    double *tw = fp_twiddles(r, span, P, p);
    double wi = span >= 4 ? fp_reduce((double)powmod_u(r, (uint64_t)(span >> 2), p), P) : 1.0;
    for (int64_t L = span; L >= 4; L >>= 2) build_fp_4(&pl->st[pl->nst++], tw, span, L, wi);
    free(tw);
    /* leftover twiddle-free radix-2 (:719, :728) as an explicit span-2 stage */
    if (ctz64((uint64_t)span) & 1) {
        orc_stage *s = &pl->st[pl->nst++];
        memset(s, 0, sizeof *s);
        s->m = 2;
        s->span = 2;
        s->Q = 1;
    }
    pl->N2 = span;
    pl->ninv = fp_reduce((double)invmod_u((uint64_t)N % p, p), P); /* :269 */
    pl->ninvp = pl->ninv / P;
    return pl;
}

void orc_plan_free(orc_plan *pl) {
    if (!pl) return;
    for (int i = 0; i < pl->nst; i++) free(pl->st[i].tw);
    free(pl);
}

int orc_plan_nstages(const orc_plan *pl) { return pl->nst; }
int64_t orc_plan_N2(const orc_plan *pl) { return pl->N2; }
double orc_plan_ninv(const orc_plan *pl) { return pl->ninv; }
double orc_plan_ninvp(const orc_plan *pl) { return pl->ninvp; }
/* stage accessors for the tests: returns m, fills span/Q/twlen and rot[8] */
int orc_plan_stage(const orc_plan *pl, int i, int64_t *span, int64_t *Q, int64_t *twlen, double *rot) {
    const orc_stage *s = &pl->st[i];
    *span = s->span;
    *Q = s->Q;
    *twlen = s->twlen;
    memcpy(rot, s->rot, sizeof s->rot);
    return s->m;
}
const double *orc_plan_stage_tw(const orc_plan *pl, int i) { return pl->st[i].tw; }

/* ------------------------------------------------------------------------ */
/* Butterflies and stages: src/fpntt.jl:300-713                              */

/* fp_dft3 :305-308 */
static inline void fp_dft3(double *a, double *b, double *c, double w3, double P) {
    OPS(7);
    double u = fp_mulmod3(*b - *c, w3, P);
    double y0 = *a + (*b + *c), y1 = (*a - *c) + u, y2 = (*a - *b) - u;
    *a = y0; *b = y1; *c = y2;
}

/* fp_dft5 :371-382 */
static inline void fp_dft5(double y[5], const double k[4], double P) {
    OPS(16);
    double x0 = y[0], x1 = y[1], x2 = y[2], x3 = y[3], x4 = y[4];
    double t1 = x1 + x4, t3 = x1 - x4;
    double t2 = x2 + x3, t4 = x2 - x3;
    double S = t1 + t2, D = t1 - t2;
    double y0 = x0 + S;
    double r = fp_reduce(x0 + fp_mulmod3(S, k[0], P), P);
    double q = fp_mulmod3(D, k[1], P);
    double g1 = fp_mulmod3(t3, k[2], P) + fp_mulmod3(t4, k[3], P);
    double g2 = fp_mulmod3(t3, k[3], P) - fp_mulmod3(t4, k[2], P);
    double u = r + q, v = r - q;
    y[0] = y0; y[1] = u + g1; y[2] = v + g2; y[3] = v - g2; y[4] = u - g1;
}

/* fp_dft7 :459-492 */
static inline void fp_dft7(double y[7], const double *rot, double P, int red) {
    double x0 = y[0];
    double s1 = y[1] + y[6], d1 = y[1] - y[6];
    double s2 = y[2] + y[5], d2 = y[2] - y[5];
    double s3 = y[3] + y[4], d3 = y[3] - y[4];
    OPS(6);
    if (red) {
        s1 = fp_reduce(s1, P); s2 = fp_reduce(s2, P); s3 = fp_reduce(s3, P);
        d1 = fp_reduce(d1, P); d2 = fp_reduce(d2, P); d3 = fp_reduce(d3, P);
    }
    double S = (s1 + s2) + s3;
    double y0 = x0 + S;
    double m1 = fp_mulmod3(S, rot[0], P);
    double va = s1 - s3, vb = s2 - s3;
    double w0 = fp_mulmod3(va, rot[1], P);
    double w1 = fp_mulmod3(vb, rot[2], P);
    double w2 = fp_mulmod3(va + vb, rot[3], P);
    double mn = fp_mulmod3((d1 + d2) - d3, rot[4], P);
    double wa = d1 + d3, wb = -(d2 + d3);
    double q0 = fp_mulmod3(wa, rot[5], P);
    double q1 = fp_mulmod3(wb, rot[6], P);
    double q2 = fp_mulmod3(wa + wb, rot[7], P);
    OPS(11);
    double u1 = fp_reduce(m1 + (3 * w0 - w2), P);
    double u3 = fp_reduce((m1 + 2 * w2) - 3 * (w0 + w1), P);
    double u2 = fp_reduce(m1 + (3 * w1 - w2), P);
    double r0 = q0 - q1, r1 = q2 - q0;
    double v1 = fp_reduce(mn + (2 * r0 + r1), P);
    double v3 = fp_reduce((r0 + 2 * r1) - mn, P);
    double v2 = fp_reduce((mn - r0) + r1, P);
    double a1 = x0 + u1, a2 = x0 + u2, a3 = x0 + u3;
    OPS(30);
    y[0] = y0;
    y[1] = a1 + v1; y[2] = a2 + v2; y[3] = a3 + v3;
    y[4] = a3 - v3; y[5] = a2 - v2; y[6] = a1 - v1;
}

/* fp_dft4 :543-549 */
static inline void fp_dft4(double y[4], double wi, double P) {
    OPS(8);
    double a = y[0], b = y[1], c = y[2], d = y[3];
    double apc = a + c, amc = a - c, bpd = b + d;
    double ibmd = fp_mulmod3(b - d, wi, P);
    y[0] = apc + bpd; y[1] = amc + ibmd; y[2] = apc - bpd; y[3] = amc - ibmd;
}

/* One butterfly of an odd or radix-4 stage at block offset o, column j:
 * fp_radix3! :310-354, fp_radix5! :384-442, fp_radix7! :494-537,
 * fp_radix4! :645-701 (incl. fp_smallq! :595-624, same per-butterfly math). */
static void orc_butterfly(double *x, int64_t o, int64_t j, const orc_stage *s, double P, int fwd) {
    const int m = s->m;
    const int64_t Q = s->Q;
    double y[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int t = 0; t < m; t++) y[t] = x[o + j + t * Q];
    if (fwd) {
        if (m == 3) fp_dft3(&y[0], &y[1], &y[2], s->rot[0], P);
        else if (m == 4) fp_dft4(y, s->rot[0], P);
        else if (m == 5) fp_dft5(y, s->rot, P);
        else fp_dft7(y, s->rot, P, 0);
    }
    y[0] = fp_reduce(y[0], P);
    int64_t jt = j < s->twlen ? j : j % s->twlen;
    for (int t = 1; t < m; t++) y[t] = fp_mulmod3(y[t], s->tw[(t - 1) * s->twlen + jt], P);
    if (!fwd) {
        if (m == 3) fp_dft3(&y[0], &y[1], &y[2], s->rot[0], P);
        else if (m == 4) fp_dft4(y, s->rot[0], P);
        else if (m == 5) { fp_dft5(y, s->rot, P); y[0] = fp_reduce(y[0], P); }
        else { fp_dft7(y, s->rot, P, 1); y[0] = fp_reduce(y[0], P); }
    }
    for (int t = 0; t < m; t++) x[o + j + t * Q] = y[t];
}

/* fp_radix2! :630-638 (twiddle-free, reduced, self-transpose) */
static void fp_radix2(double *x, int64_t N, double P) {
    for (int64_t s = 0; s < N; s += 2) {
        double u = x[s], v = x[s + 1];
        OPS(2);
        x[s] = fp_reduce(u + v, P);
        x[s + 1] = fp_reduce(u - v, P);
    }
}

/* fp_stage! :703-713 for one stage of the plan, either direction */
void orc_stage_run(double *x, const orc_plan *pl, int i, int fwd) {
    const orc_stage *s = &pl->st[i];
    double P = (double)ORC_P[pl->f];
    if (s->m == 2) { fp_radix2(x, pl->N, P); return; }
    for (int64_t o = 0; o < pl->N; o += s->span)
        for (int64_t j = 0; j < s->Q; j++) orc_butterfly(x, o, j, s, P, fwd);
}

/* fp_ntt_fwd! :715-721 */
void orc_ntt_fwd(double *x, const orc_plan *pl) {
    for (int i = 0; i < pl->nst; i++) orc_stage_run(x, pl, i, 1);
}
/* fp_ntt_rev! :727-733 */
void orc_ntt_rev(double *x, const orc_plan *pl) {
    for (int i = pl->nst - 1; i >= 0; i--) orc_stage_run(x, pl, i, 0);
}

/* ------------------------------------------------------------------------ */
/* Pack and pointwise: src/fpntt.jl:744-785                                  */

/* fp_ntt_pack! :744-768 (limbs 0-based here) */
void orc_pack(double *x, int64_t N, const uint64_t *limbs, int64_t n, int b, int64_t nch) {
    uint64_t mask = (1ULL << b) - 1;
    int64_t lim = 64 * (n - 1) - 1;
    int64_t imax = lim >= 0 ? lim / b : -1; /* fld(64(n-1)-1, b) */
    if (nch - 1 < imax) imax = nch - 1;
    for (int64_t i = 0; i <= imax; i++) {
        int64_t bit = i * b, w = bit >> 6;
        int sh = (int)(bit & 63);
        uint64_t c = (limbs[w] >> sh) | (sh ? limbs[w + 1] << (64 - sh) : 0);
        x[i] = (double)(c & mask);
    }
    for (int64_t i = imax + 1; i < nch; i++) {
        int64_t bit = i * b, w = bit >> 6;
        int sh = (int)(bit & 63);
        uint64_t c = limbs[w] >> sh;
        if (sh + b > 64 && w + 2 <= n) c |= limbs[w + 1] << (64 - sh);
        x[i] = (double)(c & mask);
    }
    for (int64_t i = nch; i < N; i++) x[i] = 0.0;
}

/* fp_ntt_pointwise! :770-785 */
void orc_pointwise(double *xa, const double *xb, int64_t N, int f) {
    double P = (double)ORC_P[f];
    for (int64_t i = 0; i < N; i++) xa[i] = fp_mulmod3(xa[i], xb[i], P);
}

/* ------------------------------------------------------------------------ */
/* Garner unpack: src/fpntt.jl:787-925, addmul_1!: src/kernels/mul.jl:32-70  */

/* fp_unpack_coeff :806-816 */
static inline void fp_unpack_coeff(const double *x1, const double *x2, int64_t idx, double n1, double n1p,
                                   double n2, double n2p, double g, double gp, uint64_t *c1, uint64_t *uu) {
    const double P1 = (double)ORC_P[0], P2 = (double)ORC_P[1];
    double v1 = fp_mulmod4(x1[idx], n1, n1p, P1);
    OPS(1);
    v1 = v1 < 0 ? v1 + P1 : v1;
    double v2 = fp_mulmod4(x2[idx], n2, n2p, P2);
    OPS(2);
    double u = fp_mulmod4(v2 - fp_reduce(v1, P2), g, gp, P2);
    *c1 = (uint64_t)v1;
    *uu = (uint64_t)(u < 0 ? u + P2 : u);
}

/* addmul_1! semantics (src/kernels/mul.jl:32-70): r[0..n) += a[0..n)*b, returns carry */
static uint64_t addmul_1(uint64_t *r, const uint64_t *a, int64_t n, uint64_t b) {
    uint64_t c = 0;
    for (int64_t i = 0; i < n; i++) {
        u128 p = (u128)a[i] * b + r[i] + c;
        r[i] = (uint64_t)p;
        c = (uint64_t)(p >> 64);
    }
    return c;
}

/* fp_ntt_unpack2! :869-925 (scalar: fp_unpack_scalar! + fp_accum_words!) */
void orc_unpack2(uint64_t *r, int64_t rn, const double *x1, const double *x2, int64_t N, int64_t nconv, int b,
                 double n1, double n1p, double n2, double n2p) {
    uint64_t *s2 = (uint64_t *)calloc((size_t)(rn > 0 ? rn : 1), sizeof(uint64_t));
    const uint64_t p1 = ORC_P[0], p2 = ORC_P[1];
    double g = (double)invmod_u(p1 % p2, p2); /* :879 */
    double gp = g / (double)p2;               /* :880 */
    u128 w1 = 0, w2 = 0;
    int s = 0;
    int64_t outw = 0; /* 0-based limb the windows start at */
    for (int64_t c = 0; c < nconv; c++) {
        int64_t idx = c == 0 ? 0 : N - c; /* :830 */
        uint64_t c1, uu;
        fp_unpack_coeff(x1, x2, idx, n1, n1p, n2, n2p, g, gp, &c1, &uu);
        int sh = s; /* (i*b) & 63 */
        u128 lo1 = (u128)c1 << sh, lo2 = (u128)uu << sh;
        w1 += lo1;
        w2 += lo2;
        s += b;
        if (s >= 64) { /* fp_accum_words! flush :857-864 */
            if (outw < rn) { r[outw] = (uint64_t)w1; s2[outw] = (uint64_t)w2; }
            w1 >>= 64;
            w2 >>= 64;
            outw++;
            s -= 64;
        }
    }
    for (; outw < rn; outw++) { /* :915-922 */
        r[outw] = (uint64_t)w1;
        s2[outw] = (uint64_t)w2;
        w1 >>= 64;
        w2 >>= 64;
    }
    addmul_1(r, s2, rn, p1); /* :923 */
    free(s2);
}

/* ------------------------------------------------------------------------ */
/* Admission: src/fpntt.jl:927-977 and magnitude_bits (kernels/addsub.jl:150) */

static int top_set_bit_u64(uint64_t x) { return x ? 64 - __builtin_clzll(x) : 0; }
static int top_set_bit_u128(u128 x) {
    uint64_t hi = (uint64_t)(x >> 64);
    return hi ? 64 + top_set_bit_u64(hi) : top_set_bit_u64((uint64_t)x);
}

int64_t orc_magnitude_bits(const uint64_t *a, int64_t n) { return 64 * (n - 1) + top_set_bit_u64(a[n - 1]); }

/* ntt_len :936-951.  Returns -1 when T exceeds 315*2^34 (ArgumentError). */
int64_t orc_ntt_len(int64_t T) {
    static const int64_t SMALL[] = {1, 3, 5, 9}, MID[] = {1, 3, 5, 7, 9, 15, 21, 105},
                         LARGE[] = {1, 3, 5, 7, 9, 15, 21, 35, 45, 63, 105, 315};
    const int maxk = ORC_TWOADIC[0] < ORC_TWOADIC[1] ? ORC_TWOADIC[0] : ORC_TWOADIC[1];
    const int64_t *ms;
    int nm;
    if (T <= (1LL << 14)) { ms = SMALL; nm = 4; }
    else if (T <= (1LL << 20)) { ms = MID; nm = 8; }
    else { ms = LARGE; nm = 12; }
    int64_t best = INT64_MAX;
    for (int i = 0; i < nm; i++) {
        int64_t m = ms[i];
        int64_t cl = (T + m - 1) / m; /* cld(T, m) */
        int k = top_set_bit_u64((uint64_t)(cl - 1));
        if (k < 2) k = 2;
        if (k > maxk) continue;
        int64_t c = m << k;
        if (c < best) best = c;
    }
    return best == INT64_MAX ? -1 : best;
}

/* fp_ntt_params :964-977 */
int orc_ntt_params(int64_t bits_a, int64_t bits_b, int *b_out, int64_t *N_out) {
    const u128 pp = (u128)ORC_P[0] * ORC_P[1] - 1;
    const uint64_t pmin = ORC_P[0] < ORC_P[1] ? ORC_P[0] : ORC_P[1];
    const int maxb = top_set_bit_u64(pmin) - 1;
    int64_t mn = bits_a < bits_b ? bits_a : bits_b;
    int nclow = top_set_bit_u64((uint64_t)((mn + maxb - 1) / maxb));
    int bstart = (top_set_bit_u128(pp) - nclow + 3) >> 1;
    if (bstart > maxb) bstart = maxb;
    for (int b = bstart; b >= 1; b--) {
        int64_t nca = (bits_a + b - 1) / b, ncb = (bits_b + b - 1) / b;
        u128 m2 = (u128)((1ULL << b) - 1);
        m2 *= m2;
        int64_t mnc = nca < ncb ? nca : ncb;
        if ((u128)mnc <= pp / m2) {
            int64_t N = orc_ntt_len(nca + ncb - 1);
            if (N < 0) return -1;
            *b_out = b;
            *N_out = N;
            return 0;
        }
    }
    return -2;
}

/* ------------------------------------------------------------------------ */
/* Engine entry points: src/fpntt.jl:982-1037                                */

/* A small plan cache so repeated oracle products do not rebuild tables
 * (the reference memoizes per (N, p): :273-293).  Not thread-safe; callers
 * that run products on several threads pre-build plans with orc_plan_get
 * from one thread first. */
#define ORC_CACHE 1024
static struct { int64_t N; int f; orc_plan *pl; } orc_cache[ORC_CACHE];
static int orc_ncache = 0;
/* The cache is shared by the threads of the timed CPU baseline: one lock. */
static pthread_mutex_t orc_cache_mu = PTHREAD_MUTEX_INITIALIZER;

orc_plan *orc_plan_get(int64_t N, int f) {
    pthread_mutex_lock(&orc_cache_mu);
    for (int i = 0; i < orc_ncache; i++)
        if (orc_cache[i].N == N && orc_cache[i].f == f) {
            orc_plan *hit = orc_cache[i].pl;
            pthread_mutex_unlock(&orc_cache_mu);
            return hit;
        }
    orc_plan *pl = orc_plan_build(N, f);
    if (pl && orc_ncache < ORC_CACHE) {
        orc_cache[orc_ncache].N = N;
        orc_cache[orc_ncache].f = f;
        orc_cache[orc_ncache].pl = pl;
        orc_ncache++;
    }
    pthread_mutex_unlock(&orc_cache_mu);
    return pl;
}

/* mul_fpntt2! :982-1014.  r[0..m+n) = a[0..m) * b[0..n).  Returns 0 on success. */
int orc_mul_fpntt2(uint64_t *r, const uint64_t *a, int64_t m, const uint64_t *b, int64_t n) {
    int64_t bits_a = orc_magnitude_bits(a, m), bits_b = orc_magnitude_bits(b, n);
    int bch;
    int64_t N;
    if (orc_ntt_params(bits_a, bits_b, &bch, &N)) return -1;
    orc_plan *plan1 = orc_plan_get(N, 0), *plan2 = orc_plan_get(N, 1);
    if (!plan1 || !plan2) return -1;
    int64_t nca = (bits_a + bch - 1) / bch, ncb = (bits_b + bch - 1) / bch;
    double *buf = (double *)malloc(sizeof(double) * 3 * (size_t)N);
    if (!buf) return -3;
    double *tmp1 = buf, *tmp2 = buf + N, *tmp3 = buf + 2 * N;
    orc_pack(tmp3, N, a, m, bch, nca);
    memcpy(tmp1, tmp3, sizeof(double) * (size_t)N);
    orc_ntt_fwd(tmp1, plan1);
    orc_pack(tmp2, N, b, n, bch, ncb);
    orc_ntt_fwd(tmp2, plan1);
    orc_pointwise(tmp1, tmp2, N, 0);
    orc_ntt_rev(tmp1, plan1);
    orc_ntt_fwd(tmp3, plan2);
    orc_pack(tmp2, N, b, n, bch, ncb);
    orc_ntt_fwd(tmp2, plan2);
    orc_pointwise(tmp3, tmp2, N, 1);
    orc_ntt_rev(tmp3, plan2);
    orc_unpack2(r, m + n, tmp1, tmp3, N, nca + ncb - 1, bch, plan1->ninv, plan1->ninvp, plan2->ninv, plan2->ninvp);
    free(buf);
    return 0;
}

/* sqr_fpntt2! :1016-1037.  r[0..2n) = a[0..n)^2. */
int orc_sqr_fpntt2(uint64_t *r, const uint64_t *a, int64_t n) {
    int64_t bits = orc_magnitude_bits(a, n);
    int bch;
    int64_t N;
    if (orc_ntt_params(bits, bits, &bch, &N)) return -1;
    orc_plan *plan1 = orc_plan_get(N, 0), *plan2 = orc_plan_get(N, 1);
    if (!plan1 || !plan2) return -1;
    int64_t nca = (bits + bch - 1) / bch;
    double *buf = (double *)malloc(sizeof(double) * 2 * (size_t)N);
    if (!buf) return -3;
    double *tmp1 = buf, *tmp2 = buf + N;
    orc_pack(tmp2, N, a, n, bch, nca);
    memcpy(tmp1, tmp2, sizeof(double) * (size_t)N);
    orc_ntt_fwd(tmp1, plan1);
    orc_pointwise(tmp1, tmp1, N, 0);
    orc_ntt_rev(tmp1, plan1);
    orc_ntt_fwd(tmp2, plan2);
    orc_pointwise(tmp2, tmp2, N, 1);
    orc_ntt_rev(tmp2, plan2);
    orc_unpack2(r, 2 * n, tmp1, tmp2, N, 2 * nca - 1, bch, plan1->ninv, plan1->ninvp, plan2->ninv, plan2->ninvp);
    free(buf);
    return 0;
}

/* ---------------------------------------------------------------------------
 * Barrett powermod (the workload of the powermod chains): a restatement of
 * powermod_limbs on its Barrett branch (src/algorithms.jl:17-107) with
 * barrett_mu!/barrett_reduce! (src/barrett.jl:22-81); every product goes
 * through the fp NTT above, as the reference's mul!/sqr! do at 256 limbs.
 * ------------------------------------------------------------------------ */

static int64_t orc_normlen(const uint64_t *a, int64_t n) {
    while (n > 0 && a[n - 1] == 0) n--;
    return n;
}

/* a[0..n) >= b[0..nb), nb <= n (missing limbs zero) */
static int orc_geq(const uint64_t *a, int64_t n, const uint64_t *b, int64_t nb) {
    for (int64_t i = n - 1; i >= 0; i--) {
        uint64_t y = i < nb ? b[i] : 0;
        if (a[i] != y) return a[i] > y;
    }
    return 1;
}

/* r[0..n) = a[0..n) - b[0..nb) mod 2^(64n) */
static void orc_subn(uint64_t *r, const uint64_t *a, int64_t n, const uint64_t *b, int64_t nb) {
    uint64_t br = 0;
    for (int64_t i = 0; i < n; i++) {
        uint64_t y = i < nb ? b[i] : 0, x = a[i];
        uint64_t d = x - y - br;
        br = (x < y) || (x - y < br);
        r[i] = d;
    }
}

/* r = a * b for normalized lengths (either may be zero) into r[0..m+n) */
static void orc_mul_any(uint64_t *r, const uint64_t *a, int64_t m, const uint64_t *b, int64_t n) {
    int64_t la = orc_normlen(a, m), lb = orc_normlen(b, n);
    memset(r, 0, sizeof(uint64_t) * (size_t)(m + n));
    if (!la || !lb) return;
    if (a == b && la == lb) orc_sqr_fpntt2(r, a, la);
    else orc_mul_fpntt2(r, a, la, b, lb);
}

/* mu[0..k+2) = floor(2^(128k) / m): schoolbook division by one-limb estimates
 * corrected downward (the remainder is kept exact), divrem!'s role in
 * barrett_mu!.  Returns mu's normalized length. */
int64_t orc_barrett_mu(const uint64_t *m, int64_t k, uint64_t *mu) {
    typedef unsigned __int128 u128;
    uint64_t *rem = (uint64_t *)calloc((size_t)(k + 1), sizeof(uint64_t));
    uint64_t *t = (uint64_t *)calloc((size_t)(k + 1), sizeof(uint64_t));
    memset(mu, 0, sizeof(uint64_t) * (size_t)(k + 2));
    /* numerator digits from the top: 1 followed by 2k zero limbs */
    for (int64_t j = 2 * k; j >= 0; j--) {
        /* rem = rem * 2^64 + digit */
        memmove(rem + 1, rem, sizeof(uint64_t) * (size_t)k);
        rem[0] = j == 2 * k ? 1 : 0;
        /* q = floor(rem / m) < 2^64; estimate from the top two limbs of rem and the top limb of m */
        uint64_t q = 0;
        if (orc_geq(rem, k + 1, m, k)) {
            u128 top = ((u128)rem[k] << 64) | rem[k - 1];
            u128 est = top / ((u128)m[k - 1]);
            q = est >> 64 ? ~(uint64_t)0 : (uint64_t)est;
            for (;;) { /* t = q*m; lower q until t <= rem */
                uint64_t c = 0;
                for (int64_t i = 0; i < k; i++) {
                    u128 p = (u128)q * m[i] + c;
                    t[i] = (uint64_t)p;
                    c = (uint64_t)(p >> 64);
                }
                t[k] = c;
                if (orc_geq(rem, k + 1, t, k + 1)) break;
                /* overshoot: step q down by about (t - rem) / m */
                uint64_t *d = (uint64_t *)calloc((size_t)(k + 1), sizeof(uint64_t));
                orc_subn(d, t, k + 1, rem, k + 1);
                u128 dt = ((u128)d[k] << 64) | d[k - 1];
                u128 dec = dt / ((u128)m[k - 1] + 1) + 1;
                free(d);
                q = dec >= q ? 0 : q - (uint64_t)dec;
            }
            orc_subn(rem, rem, k + 1, t, k + 1);
            while (orc_geq(rem, k + 1, m, k)) { /* q too small */
                orc_subn(rem, rem, k + 1, m, k);
                q++;
            }
        }
        if (j < k + 2) mu[j] = q;
    }
    free(rem);
    free(t);
    return orc_normlen(mu, k + 2);
}

/* barrett_reduce! (barrett.jl:44-81): r[0..k) = T mod m, T = t[0..2k) (t[2k] = 0). */
static void orc_barrett_reduce(uint64_t *r, const uint64_t *t, const uint64_t *m, int64_t k, const uint64_t *mu,
                               int64_t lmu, uint64_t *scratch) {
    const int64_t kp1 = k + 1;
    uint64_t *q2 = scratch, *r2 = scratch + 2 * k + 3;
    int64_t l1 = orc_normlen(t + k - 1, kp1), lq3 = 0;
    if (l1 > 0) {
        orc_mul_any(q2, t + k - 1, l1, mu, lmu);
        lq3 = orc_normlen(q2 + kp1, l1 + lmu - kp1);
    }
    if (lq3 == 0) {
        memcpy(scratch, t, sizeof(uint64_t) * (size_t)kp1);
    } else {
        orc_mul_any(r2, m, k, q2 + kp1, lq3);
        orc_subn(scratch, t, kp1, r2, kp1);
    }
    int64_t lr = orc_normlen(scratch, kp1);
    while (orc_geq(scratch, kp1, m, k)) {
        orc_subn(scratch, scratch, kp1, m, k);
        lr = orc_normlen(scratch, lr);
    }
    memcpy(r, scratch, sizeof(uint64_t) * (size_t)lr);
    memset(r + lr, 0, sizeof(uint64_t) * (size_t)(k - lr));
}

static int orc_expbit(const uint64_t *e, int64_t i) { return (int)((e[i >> 6] >> (i & 63)) & 1); }

/* powermod_limbs, Barrett branch: r[0..k) = b^e mod m.  b[0..lb) with lb <= k
 * (reduced mod m first), e[0..le) nonzero, m[k-1] != 0, m > 1. */
int orc_powmod_barrett(uint64_t *r, const uint64_t *b, int64_t lb, const uint64_t *e, int64_t le, const uint64_t *m,
                       int64_t k) {
    int64_t nbits = 0;
    for (int64_t i = le - 1; i >= 0 && !nbits; i--)
        if (e[i]) nbits = 64 * i + 64 - (int64_t)__builtin_clzll(e[i]);
    if (!nbits || lb > k || !m[k - 1]) return -1;
    const int w = nbits <= 8 ? 1 : nbits <= 24 ? 2 : nbits <= 80 ? 3 : nbits <= 240 ? 4 : 5;
    const int tsize = 1 << (w - 1);
    uint64_t *mu = (uint64_t *)calloc((size_t)(k + 2), 8);
    uint64_t *scratch = (uint64_t *)calloc((size_t)(4 * k + 6), 8);
    uint64_t *prod = (uint64_t *)calloc((size_t)(2 * k + 1), 8);
    uint64_t *table = (uint64_t *)calloc((size_t)(tsize * k), 8);
    uint64_t *acc = (uint64_t *)calloc((size_t)k, 8);
    uint64_t *bsq = (uint64_t *)calloc((size_t)k, 8);
    const int64_t lmu = orc_barrett_mu(m, k, mu);
#define MULRED(dst, x, y)                                  \
    do {                                                   \
        orc_mul_any(prod, (x), k, (y), k);                 \
        prod[2 * k] = 0;                                   \
        orc_barrett_reduce((dst), prod, m, k, mu, lmu, scratch); \
    } while (0)
    /* slot 0 = b mod m (the reference reduces b before powermod_limbs) */
    memset(prod, 0, sizeof(uint64_t) * (size_t)(2 * k + 1));
    memcpy(prod, b, sizeof(uint64_t) * (size_t)lb);
    orc_barrett_reduce(table, prod, m, k, mu, lmu, scratch);
    if (tsize > 1) {
        MULRED(bsq, table, table);
        for (int j = 1; j < tsize; j++) MULRED(table + j * k, table + (j - 1) * k, bsq);
    }
    int first = 1;
    int64_t i = nbits - 1;
    while (i >= 0) {
        if (!orc_expbit(e, i)) {
            if (!first) MULRED(acc, acc, acc);
            i--;
            continue;
        }
        int64_t l = w < i + 1 ? w : i + 1;
        while (!orc_expbit(e, i - l + 1)) l--;
        int val = 0;
        for (int64_t j = 0; j < l; j++) val = (val << 1) | orc_expbit(e, i - j);
        if (first) {
            memcpy(acc, table + (val >> 1) * k, sizeof(uint64_t) * (size_t)k);
            first = 0;
        } else {
            for (int64_t j = 0; j < l; j++) MULRED(acc, acc, acc);
            MULRED(acc, acc, table + (val >> 1) * k);
        }
        i -= l;
    }
#undef MULRED
    memcpy(r, acc, sizeof(uint64_t) * (size_t)k);
    free(mu);
    free(scratch);
    free(prod);
    free(table);
    free(acc);
    free(bsq);
    return 0;
}
