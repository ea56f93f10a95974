// fp.cuh — exact Float64 residue arithmetic on the FP64 CUDA cores.
//
// Device restatement of the field layer of NativeBigInt.jl src/fpntt.jl:81-121.
// Every operation is written with the IEEE round-to-nearest intrinsics
// (__dadd_rn, __dmul_rn, __fma_rn) so nvcc can neither contract a*b+c into an
// FMA nor reassociate: the reference's exactness argument (fpntt.jl:8-45) needs
// each product split h + l by an explicit fma and each round done by the
// magic-constant add/sub pair.  The library is also compiled with -fmad=false.
#pragma once
#include <cstdint>

#include "consts.h"

namespace nbg {

struct Fp {
    double p;     // the prime, exact in a double
    double pinv;  // fl(1/p)
};

__device__ __forceinline__ double fp_round(double v) {
    return __dsub_rn(__dadd_rn(v, FP_MAGIC), FP_MAGIC);
}

// r == x (mod p), |r| < p for |x| <= 2^51 p (fpntt.jl:88-91)
__device__ __forceinline__ double fp_reduce(double x, Fp F) {
    double q = fp_round(__dmul_rn(x, F.pinv));
    return __fma_rn(q, -F.p, x);
}

// 3-argument (value/stage) mulmod (fpntt.jl:101-105): 7 FP64 instructions
__device__ __forceinline__ double fp_mulmod(double x, double y, Fp F) {
    double h = __dmul_rn(x, y);
    double l = __fma_rn(x, y, -h);
    return __dadd_rn(fp_reduce(h, F), l);
}

// 4-argument Shoup form with precomputed wpinv = fl(w/p) (fpntt.jl:106-111)
__device__ __forceinline__ double fp_mulmod4(double x, double w, double wpinv, Fp F) {
    double h = __dmul_rn(x, w);
    double l = __fma_rn(x, w, -h);
    double q = fp_round(__dmul_rn(x, wpinv));
    return __dadd_rn(__fma_rn(q, -F.p, h), l);
}

// minimal balanced representative |x| <= p/2 of |x| < ~p (fpntt.jl:118-119)
__device__ __forceinline__ double fp_minbal(double x, Fp F) {
    double h = F.p * 0.5;
    return x > h ? __dsub_rn(x, F.p) : (x < -h ? __dadd_rn(x, F.p) : x);
}

__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }

}  // namespace nbg
