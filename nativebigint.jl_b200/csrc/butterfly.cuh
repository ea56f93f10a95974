// butterfly.cuh — the reference's DFT butterflies on the FP64 cores.
//
// Restated from NativeBigInt.jl src/fpntt.jl: radix-3 (fp_dft3 :305-308,
// fp_radix3! :310-354), radix-5 (fp_dft5 :371-382, fp_radix5! :384-442),
// radix-7 (fp_dft7 :459-492, fp_radix7! :494-537), radix-4 (fp_dft4 :543-549,
// fp_radix4! :645-701) and radix-2 (fp_radix2! :630-638).  Each butterfly does
// exactly the reference's operations in the reference's order, so every
// intermediate double equals the reference's: the forward runs the combine,
// reduces lane 0 and twiddles lanes 1..m-1; the reverse twiddles first and
// combines after (radix-5/7 re-reduce lane 0; radix-7 reduces its pair sums).
#pragma once
#include "fp.cuh"

namespace nbg {

__device__ __forceinline__ void dft3(double& a, double& b, double& c, double w3, Fp F) {
    double u = fp_mulmod(dsub(b, c), w3, F);
    double y0 = dadd(a, dadd(b, c));
    double y1 = dadd(dsub(a, c), u);
    double y2 = dsub(dsub(a, b), u);
    a = y0; b = y1; c = y2;
}

__device__ __forceinline__ void dft4(double& a, double& b, double& c, double& d, double wi, Fp F) {
    double apc = dadd(a, c), amc = dsub(a, c), bpd = dadd(b, d);
    double ibmd = fp_mulmod(dsub(b, d), wi, F);
    a = dadd(apc, bpd); b = dadd(amc, ibmd); c = dsub(apc, bpd); d = dsub(amc, ibmd);
}

__device__ __forceinline__ void dft5(double* y, const double* k, Fp F) {
    double x0 = y[0], x1 = y[1], x2 = y[2], x3 = y[3], x4 = y[4];
    double t1 = dadd(x1, x4), t3 = dsub(x1, x4);
    double t2 = dadd(x2, x3), t4 = dsub(x2, x3);
    double S = dadd(t1, t2), D = dsub(t1, t2);
    double y0 = dadd(x0, S);
    double r = fp_reduce(dadd(x0, fp_mulmod(S, k[0], F)), F);
    double q = fp_mulmod(D, k[1], F);
    double g1 = dadd(fp_mulmod(t3, k[2], F), fp_mulmod(t4, k[3], F));
    double g2 = dsub(fp_mulmod(t3, k[3], F), fp_mulmod(t4, k[2], F));
    double u = dadd(r, q), v = dsub(r, q);
    y[0] = y0; y[1] = dadd(u, g1); y[2] = dadd(v, g2); y[3] = dsub(v, g2); y[4] = dsub(u, g1);
}

template <bool RED>
__device__ __forceinline__ void dft7(double* y, const double* rot, Fp F) {
    double x0 = y[0];
    double s1 = dadd(y[1], y[6]), d1 = dsub(y[1], y[6]);
    double s2 = dadd(y[2], y[5]), d2 = dsub(y[2], y[5]);
    double s3 = dadd(y[3], y[4]), d3 = dsub(y[3], y[4]);
    if (RED) {
        s1 = fp_reduce(s1, F); s2 = fp_reduce(s2, F); s3 = fp_reduce(s3, F);
        d1 = fp_reduce(d1, F); d2 = fp_reduce(d2, F); d3 = fp_reduce(d3, F);
    }
    double S = dadd(dadd(s1, s2), s3);
    double y0 = dadd(x0, S);
    double m1 = fp_mulmod(S, rot[0], F);
    double va = dsub(s1, s3), vb = dsub(s2, s3);
    double w0 = fp_mulmod(va, rot[1], F);
    double w1 = fp_mulmod(vb, rot[2], F);
    double w2 = fp_mulmod(dadd(va, vb), rot[3], F);
    double mn = fp_mulmod(dsub(dadd(d1, d2), d3), rot[4], F);
    double wa = dadd(d1, d3), wb = -dadd(d2, d3);
    double q0 = fp_mulmod(wa, rot[5], F);
    double q1 = fp_mulmod(wb, rot[6], F);
    double q2 = fp_mulmod(dadd(wa, wb), rot[7], F);
    double u1 = fp_reduce(dadd(m1, dsub(dmul(3.0, w0), w2)), F);
    double u3 = fp_reduce(dsub(dadd(m1, dmul(2.0, w2)), dmul(3.0, dadd(w0, w1))), F);
    double u2 = fp_reduce(dadd(m1, dsub(dmul(3.0, w1), w2)), F);
    double r0 = dsub(q0, q1), r1 = dsub(q2, q0);
    double v1 = fp_reduce(dadd(mn, dadd(dmul(2.0, r0), r1)), F);
    double v3 = fp_reduce(dsub(dadd(r0, dmul(2.0, r1)), mn), F);
    double v2 = fp_reduce(dadd(dsub(mn, r0), r1), F);
    double a1 = dadd(x0, u1), a2 = dadd(x0, u2), a3 = dadd(x0, u3);
    y[0] = y0;
    y[1] = dadd(a1, v1); y[2] = dadd(a2, v2); y[3] = dadd(a3, v3);
    y[4] = dsub(a3, v3); y[5] = dsub(a2, v2); y[6] = dsub(a1, v1);
}

template <int M, bool REV>
__device__ __forceinline__ void combine(double* y, const double* rot, Fp F) {
    if constexpr (M == 3) dft3(y[0], y[1], y[2], rot[0], F);
    else if constexpr (M == 4) dft4(y[0], y[1], y[2], y[3], rot[0], F);
    else if constexpr (M == 5) dft5(y, rot, F);
    else if constexpr (M == 7) dft7<REV>(y, rot, F);
}

// One butterfly of an odd or radix-4 stage.  w[t] (t >= 1) is the lane-t twiddle.
template <int M, bool FWD>
__device__ __forceinline__ void butterfly(double* y, const double* w, const double* rot, Fp F) {
    if (FWD) combine<M, false>(y, rot, F);
    y[0] = fp_reduce(y[0], F);
#pragma unroll
    for (int t = 1; t < M; t++) y[t] = fp_mulmod(y[t], w[t], F);
    if (!FWD) {
        combine<M, true>(y, rot, F);
        if (M == 5 || M == 7) y[0] = fp_reduce(y[0], F);
    }
}

// Twiddle-free radix-2, both directions (fp_radix2! :630-638)
__device__ __forceinline__ void butterfly2(double& u, double& v, Fp F) {
    double s = fp_reduce(dadd(u, v), F);
    double d = fp_reduce(dsub(u, v), F);
    u = s; v = d;
}

}  // namespace nbg
