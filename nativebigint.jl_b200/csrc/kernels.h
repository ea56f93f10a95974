// kernels.h — host-side entry points of kernels.cu.
#pragma once
#include <cuda_runtime.h>

#include "types.h"

namespace nbg {

// Uploads the prime constants and raises the kernels' dynamic shared-memory cap.
cudaError_t kernels_init(double p1, double p2);
int kernels_smem_optin();
// reads and clears the count of bounded waits that gave up (current device)
cudaError_t kernels_take_faults(unsigned int* n);
// binaryVersion of the pass kernels as loaded on the current device
cudaError_t kernels_binary_version(int* version);

// An explicit job list as a launch's job source.
inline JobSrc job_list(const Job* l) {
    JobSrc s{};
    s.list = l;
    s.mode = JM_LIST;
    return s;
}

// One work-queue launch of `kind` (JobKind) over jobs 0..njobs-1 of `jobs`.
// odd = false: no pass of the launch holds a radix-3/5/7 stage (a leaner kernel build).
cudaError_t launch_jobs(int kind, const DProd* prods, const DPlan* plans, const JobSrc& jobs, int64_t njobs,
                        size_t smem, int grid_cap, cudaStream_t st, bool odd = true);

// Work-queue execution of a batch (k_queue): need[prod * QSTEPS + step] +=
// the jobs of every step (need zeroed first), the persistent grid for a
// dynamic shared-memory size, and the launch (qs and done zeroed first) whose
// CTAs claim `chunk` consecutive jobs at a time.
cudaError_t launch_qcount(const DProd* prods, const Job* jobs, const QLaunch* ql, int nl, int64_t total,
                          uint32_t* need, cudaStream_t st);
cudaError_t queue_grid(size_t smem, int* grid);
cudaError_t launch_queue(const DProd* prods, const DPlan* plans, const Job* jobs, const QLaunch* ql, int nl,
                         QState* qs, uint32_t* done, const uint32_t* need, size_t smem, int grid, int chunk,
                         cudaStream_t st);

// Writes a batch's explicit job list from its compact description: out[g] for
// every g < total, entry e covering [e.begin, e.begin + e.n).
cudaError_t launch_expand(const ExpandEntry* entries, int nentries, Job* out, int64_t total, cudaStream_t st);

// Expands one stage's twiddle table (see k_twiddle).
cudaError_t launch_twiddle(double* out, int m, int64_t Q, int64_t step, const double* hi, const double* lo, int f,
                           cudaStream_t st);

cudaError_t launch_pack(double* x, int64_t N, const uint64_t* limbs, int64_t n, int b, int64_t nch, cudaStream_t st);
cudaError_t launch_pointwise(double* xa, const double* xb, int64_t N, int f, cudaStream_t st);
cudaError_t launch_topbits(const DProd* prods, int64_t count, int64_t* bits, cudaStream_t st);

}  // namespace nbg
