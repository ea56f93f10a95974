// peak.cu — FP64 issue-rate probe for the roofline denominator (libnbgpu_peak.so).
//
// The driver-measured peaks cover HBM copy and bf16 GEMM only; the fp-NTT
// kernels run on the FP64 CUDA cores, so their ceiling is measured here:
// every thread runs 8 independent DFMA (or DADD) chains, grid = SMs x 8
// blocks of 256 threads, timed with CUDA events.  Rates are FP64
// instructions per second (DFMA, DADD and DMUL each count once).
#include <cuda_runtime.h>

#include <cstdint>

namespace {

template <bool FMA>
__global__ void __launch_bounds__(256) k_chains(double* out, int iters, double a, double b) {
    double x[8];
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = 1.0 + 1e-3 * (threadIdx.x + k);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) x[k] = FMA ? __fma_rn(x[k], a, b) : __dadd_rn(x[k], b);
    }
    double s = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) s += x[k];
    if (s == 12345.678) out[blockIdx.x] = s;  // keeps the chains live
}

template <bool FMA>
double rate(int sms, double* out) {
    const int blocks = sms * 8, threads = 256, iters = 1 << 15;
    k_chains<FMA><<<blocks, threads>>>(out, 64, 0.5, 1.0);  // warm-up
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 5; rep++) {
        cudaEventRecord(e0);
        k_chains<FMA><<<blocks, threads>>>(out, iters, 0.5, 1e-9);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return (double)blocks * threads * iters * 8.0 / (best * 1e-3);
}

}  // namespace

extern "C" int nbgpeak_fp64(int device, double* dfma_per_s, double* dadd_per_s) {
    if (cudaSetDevice(device) != cudaSuccess) return 1;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    double* out = nullptr;
    if (cudaMalloc(&out, sizeof(double) * (size_t)sms * 8) != cudaSuccess) return 2;
    *dfma_per_s = rate<true>(sms, out);
    *dadd_per_s = rate<false>(sms, out);
    cudaError_t e = cudaGetLastError();
    cudaFree(out);
    return e == cudaSuccess ? 0 : 3;
}
