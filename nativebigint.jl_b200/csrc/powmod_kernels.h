// powmod_kernels.h — device state of the Barrett powermod chains and the
// launchers of their per-step kernels (powmod_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include "types.h"

namespace nbg {

constexpr int PM_NOP = 0;       // chain finished: its step product is ignored
constexpr int PM_MUL = 1;       // dst = src1 * src2 mod m
constexpr int PM_COPYOP = 2;    // dst = src1
constexpr uint8_t PM_COPY = 255;  // src2 value that marks a copy in a step list

struct PmChains {
    int32_t count;              // chains
    int32_t nslot;              // slots per chain (k limbs each)
    int32_t acc_slot, one_slot, base_slot, pad_;
    int64_t k;                  // modulus limbs
    int64_t max_steps;          // row length of ops
    const uint8_t* ops;         // [count][max_steps][3] step lists
    const int64_t* nsteps;      // steps of each chain
    uint64_t* slots;            // [count][nslot][k]
    DProd* prods;               // descriptors of the step product batch (one per chain)
    int4* cur;                  // per chain (mode, dst, src1, src2) of the current step
    uint64_t* prod;             // T = x*y, prod_stride limbs per chain (2k + 1 used)
    int64_t prod_stride;
    uint64_t* r2;               // m*q3, r2_stride limbs per chain
    int64_t r2_stride;
    const uint64_t* mod;        // [count][k] moduli
};

cudaError_t pm_launch_select(const PmChains& C, const int64_t* ctr, cudaStream_t st);
cudaError_t pm_launch_finish(const PmChains& C, cudaStream_t st);
cudaError_t pm_launch_advance(int64_t* ctr, cudaStream_t st);
cudaError_t pm_launch_init(const PmChains& C, const uint64_t* const* bases, const int64_t* lbs, cudaStream_t st);
cudaError_t pm_launch_output(const PmChains& C, uint64_t* const* outs, cudaStream_t st);

}  // namespace nbg
