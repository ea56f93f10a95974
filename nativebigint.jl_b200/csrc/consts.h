// consts.h — the two NTT primes and the rounding constant (host and device).
#pragma once
#include <cstdint>

namespace nbg {

// 1.5 * 2^52: (v + M) - M rounds v to the nearest integer for |v| <= 2^51 (src/fpntt.jl:81-83)
constexpr double FP_MAGIC = 6755399441055744.0;

// p1 = 65205*2^34 + 1, p2 = 4095*2^38 + 1 = 2^50 - 2^38 + 1 (src/fpntt.jl:78-79)
constexpr uint64_t P1_U = 65205ULL * (1ULL << 34) + 1ULL;
constexpr uint64_t P2_U = 4095ULL * (1ULL << 38) + 1ULL;

}  // namespace nbg
