// powmod_kernels.cu — per-step kernels of the Barrett powermod chains.
//
// State of chain c lives in device memory: `nslot` slots of k limbs each
// (odd-power table, b^2, accumulator, raw base, constant 1), the product
// buffer T (2k+1 limbs, the top one always zero), q2 = q1·μ and r2 = m·q3.
// One exponent step is
//   k_pm_select   points chain c's product descriptor at its step's operands
//   (three fp-NTT batches: T = x·y, q2 = q1·μ, r2 = m·q3)
//   k_pm_finish   r = (T − r2) mod β^(k+1), r −= m while r ≥ m, into the
//                 step's destination slot
//   k_pm_advance  step counter + 1
// so a run of steps is a fixed launch sequence that a CUDA graph replays.
#include <cuda_runtime.h>
#include <stdint.h>

#include "powmod_kernels.h"

namespace nbg {

// Step op of chain c: (dst, src1, src2); src2 == PM_COPY copies src1 to dst.
__global__ void k_pm_select(const PmChains C, const int64_t* __restrict__ ctr) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C.count) return;
    const int64_t s = *ctr;
    const int64_t k = C.k;
    uint64_t* base = C.slots + (int64_t)c * C.nslot * k;
    int mode = PM_NOP, dst = 0, a = C.acc_slot, b = C.one_slot;
    if (s < C.nsteps[c]) {
        const uint8_t* op = C.ops + ((int64_t)c * C.max_steps + s) * 3;
        dst = op[0];
        if (op[2] == PM_COPY) {
            mode = PM_COPYOP;
            a = op[1];
        } else {
            mode = PM_MUL;
            a = op[1];
            b = op[2];
        }
    }
    C.prods[c].a = base + (int64_t)a * k;
    C.prods[c].b = base + (int64_t)b * k;
    C.cur[c] = make_int4(mode, dst, a, b);
}

// Borrow out of a lane's block given borrow in 0 (g) and 1 (p), composed
// across lanes by an inclusive scan (borrow-lookahead).
__device__ __forceinline__ void scan_borrow(uint32_t& g, uint32_t& p, int lane) {
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t go = __shfl_up_sync(0xffffffffu, g, off);
        const uint32_t po = __shfl_up_sync(0xffffffffu, p, off);
        if (lane >= off) {  // this block after the lower one: borrow-in is the lower one's output
            const uint32_t ng = go ? p : g;
            const uint32_t np = po ? p : g;
            g = ng;
            p = np;
        }
    }
}

// x[0..n) = u[0..n) − v[0..n) (v limbs at index >= nv read as zero) by one
// warp; returns the top limb of the result in every lane.  x may alias u.
__device__ uint64_t warp_sub(uint64_t* x, const uint64_t* u, const uint64_t* v, int64_t n, int64_t nv, int lane) {
    const int64_t per = (n + 31) / 32;
    const int64_t j0 = (int64_t)lane * per, j1 = min(j0 + per, n);
    uint32_t g = 0, p = 1;  // borrow-out with borrow-in 0 / 1; an empty block passes the borrow on
    for (int64_t j = j0; j < j1; j++) {
        const uint64_t a = u[j], b = j < nv ? v[j] : 0;
        const uint64_t d = a - b;
        const uint32_t bo0 = a < b;                // borrow-in 0
        const uint32_t bo1 = (a < b) || (d == 0);  // borrow-in 1: a − b − 1 underflows
        const uint32_t ng = g ? bo1 : bo0, np = p ? bo1 : bo0;
        g = ng;
        p = np;
    }
    scan_borrow(g, p, lane);
    uint32_t bin = __shfl_up_sync(0xffffffffu, g, 1);  // exclusive: lanes before, borrow-in 0 at lane 0
    if (lane == 0) bin = 0;
    for (int64_t j = j0; j < j1; j++) {
        const uint64_t a = u[j], b = j < nv ? v[j] : 0;
        const uint64_t d = a - b - bin;
        bin = (a < b) || (a - b < (uint64_t)bin);
        x[j] = d;
    }
    __syncwarp();
    return x[n - 1];
}

// 1 if x[0..n) >= v[0..nv) (nv <= n; missing v limbs are zero), by one warp.
__device__ int warp_geq(const uint64_t* x, const uint64_t* v, int64_t n, int64_t nv, int lane) {
    const int64_t per = (n + 31) / 32;
    const int64_t j0 = (int64_t)lane * per, j1 = min(j0 + per, n);
    int cmp = 0;  // this lane's answer from its highest differing limb
    for (int64_t j = j1 - 1; j >= j0; j--) {
        const uint64_t a = x[j], b = j < nv ? v[j] : 0;
        if (a != b) {
            cmp = a > b ? 1 : -1;
            break;
        }
    }
    const unsigned diff = __ballot_sync(0xffffffffu, cmp != 0);
    if (!diff) return 1;  // equal
    const int top = 31 - __clz(diff);
    return __shfl_sync(0xffffffffu, cmp, top) > 0;
}

// One warp per chain.  r (k+1 limbs) is built in the chain's r2 buffer
// (limbs it no longer needs), then copied to the destination slot.
__global__ void __launch_bounds__(128) k_pm_finish(const PmChains C) {
    const int lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (c >= C.count) return;
    const int64_t k = C.k;
    const int4 cur = C.cur[c];
    if (cur.x == PM_NOP) return;
    uint64_t* base = C.slots + (int64_t)c * C.nslot * k;
    uint64_t* dst = base + (int64_t)cur.y * k;
    if (cur.x == PM_COPYOP) {
        const uint64_t* src = base + (int64_t)cur.z * k;
        for (int64_t j = lane; j < k; j += 32) dst[j] = src[j];
        return;
    }
    const uint64_t* T = C.prod + (int64_t)c * C.prod_stride;
    uint64_t* r = C.r2 + (int64_t)c * C.r2_stride;
    const uint64_t* m = C.mod + (int64_t)c * k;
    // r = (T − q3·m) mod β^(k+1); the true value is < 3m, so the borrow out is dropped
    warp_sub(r, T, r, k + 1, k + 1, lane);
    for (int it = 0; it < 4 && warp_geq(r, m, k + 1, k, lane); it++) warp_sub(r, r, m, k + 1, k, lane);
    for (int64_t j = lane; j < k; j += 32) dst[j] = r[j];
}

__global__ void k_pm_advance(int64_t* ctr) { *ctr += 1; }

// Slots: raw base (lb limbs, zero-padded to k), the constant 1; T's top limb 0.
__global__ void k_pm_init(const PmChains C, const uint64_t* const* __restrict__ bases,
                          const int64_t* __restrict__ lbs) {
    const int c = blockIdx.x;
    if (c >= C.count) return;
    const int64_t k = C.k;
    uint64_t* base = C.slots + (int64_t)c * C.nslot * k;
    uint64_t* braw = base + (int64_t)C.base_slot * k;
    uint64_t* one = base + (int64_t)C.one_slot * k;
    const uint64_t* b = bases[c];
    const int64_t lb = lbs[c];
    for (int64_t j = threadIdx.x; j < k; j += blockDim.x) {
        braw[j] = j < lb ? b[j] : 0;
        one[j] = j == 0 ? 1 : 0;
    }
    if (threadIdx.x == 0) C.prod[(int64_t)c * C.prod_stride + 2 * k] = 0;
}

__global__ void k_pm_output(const PmChains C, uint64_t* const* __restrict__ outs) {
    const int c = blockIdx.x;
    if (c >= C.count) return;
    const int64_t k = C.k;
    const uint64_t* acc = C.slots + ((int64_t)c * C.nslot + C.acc_slot) * k;
    uint64_t* r = outs[c];
    for (int64_t j = threadIdx.x; j < k; j += blockDim.x) r[j] = acc[j];
}

cudaError_t pm_launch_select(const PmChains& C, const int64_t* ctr, cudaStream_t st) {
    k_pm_select<<<(unsigned)((C.count + 127) / 128), 128, 0, st>>>(C, ctr);
    return cudaGetLastError();
}
cudaError_t pm_launch_finish(const PmChains& C, cudaStream_t st) {
    k_pm_finish<<<(unsigned)((C.count + 3) / 4), 128, 0, st>>>(C);
    return cudaGetLastError();
}
cudaError_t pm_launch_advance(int64_t* ctr, cudaStream_t st) {
    k_pm_advance<<<1, 1, 0, st>>>(ctr);
    return cudaGetLastError();
}
cudaError_t pm_launch_init(const PmChains& C, const uint64_t* const* bases, const int64_t* lbs, cudaStream_t st) {
    k_pm_init<<<(unsigned)C.count, 256, 0, st>>>(C, bases, lbs);
    return cudaGetLastError();
}
cudaError_t pm_launch_output(const PmChains& C, uint64_t* const* outs, cudaStream_t st) {
    k_pm_output<<<(unsigned)C.count, 256, 0, st>>>(C, outs);
    return cudaGetLastError();
}

}  // namespace nbg
