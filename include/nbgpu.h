/*
 * nbgpu.h — C ABI of the B200 fp-NTT multiplication engine (libnbgpu.so).
 *
 * Drop-in for the two-prime Float64 NTT branch of NativeBigInt.jl's mpn
 * multiply: every product is bit-identical to the reference's
 * mul_fpntt2!/sqr_fpntt2! (src/fpntt.jl:982-1037).  Plain pointers and sizes
 * only; limbs are little-endian uint64_t.  All entry points return an int
 * status (NBG_OK = 0) and never abort; nbg_last_error() describes the last
 * failure on the calling thread.  The library is thread-safe: calls on one
 * device are serialized by an internal lock.  It keeps device state (plans,
 * twiddle tables, workspace, kernel settings) for the life of the process, so
 * it must not outlive a cudaDeviceReset of a device it has used.
 */
#ifndef NBGPU_H
#define NBGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define NBG_OK 0
#define NBG_EINVAL 1   /* bad argument (null pointer, n < 1, aliasing, ...) */
#define NBG_ERANGE 2   /* transform length beyond 315*2^34: the reference's ArgumentError (fpntt.jl:948-949) */
#define NBG_ENOMEM 3   /* device or host allocation failed / over the HBM budget */
#define NBG_ECUDA 4    /* CUDA runtime error */
#define NBG_ETIMEOUT 5 /* a bounded wait expired */
#define NBG_EBUSY 6    /* queue full (serving back-pressure) */
#define NBG_ENODEV 7   /* no CUDA device */

/* ---- products, host buffers (synchronous) ------------------------------ */

/* r[0..m+n) = a[0..m) * b[0..n), m, n >= 1.  Replaces mul_fpntt2!
 * (src/fpntt.jl:982) and the NTT branch of mul!/mul_bal!
 * (src/mul.jl:388-390, :161).  r must not alias a or b (fpntt.jl:979-981). */
int nbg_mul(uint64_t *r, const uint64_t *a, int64_t m, const uint64_t *b, int64_t n);

/* r[0..2n) = a[0..n)^2.  Replaces sqr_fpntt2! (src/fpntt.jl:1016) and the NTT
 * branch of sqr! (src/mul.jl:141-147, :134). */
int nbg_sqr(uint64_t *r, const uint64_t *a, int64_t n);

/* r[0..k) = a[0..la) * b[0..lb) mod 2^(64k) (a^2 for nbg_sqrlo), la, lb, k >= 1;
 * r holds exactly k limbs and must not alias an input.  Replaces the
 * full-product branches of mullo!/sqrlo! (src/mul.jl:316-319, :361-364),
 * which keep the low k limbs of mul!/sqr!, and extends them below the
 * reference's MULLO_FULL_THRESHOLD / SQRLO_FULL_THRESHOLD (src/mul.jl:183-184). */
int nbg_mullo(uint64_t *r, const uint64_t *a, int64_t la, const uint64_t *b, int64_t lb, int64_t k);
int nbg_sqrlo(uint64_t *r, const uint64_t *a, int64_t la, int64_t k);

/* ---- products, device buffers (asynchronous on `stream`, a cudaStream_t; ----
 * ---- NULL is the legacy default stream)                                  - */

int nbg_mul_dev(uint64_t *r, const uint64_t *a, int64_t m, const uint64_t *b, int64_t n, void *stream);
int nbg_sqr_dev(uint64_t *r, const uint64_t *a, int64_t n, void *stream);

/* No counterpart in the reference (Julia allocates freely).  The same product
 * as nbg_mul_dev (device buffers, b == NULL for a square, asynchronous on
 * `stream` after reading the two top limbs), for callers that cannot allocate
 * GPU memory: code running inside a memory arena or pool that owns the whole
 * device, under an allocator hook that must not recurse, or in a foreign
 * runtime that lends only the input and output buffers.  It calls no
 * cudaMalloc/cudaFree and no allocating library routine; its workspace is a
 * fixed 16 MiB device array inside the library (held on every GPU that loads
 * the library until exit), located once per device with cudaGetSymbolAddress
 * on the first call there — make that first call before any stream capture.
 * Every call synchronizes `stream`: it reads the operands' top limbs to the
 * host to size the transform (twice more when it builds twiddle tables for a
 * new transform length).  Products that do not fit return NBG_ENOMEM: transform lengths above about
 * 3.4e5 points for products (balanced operands above about 2^16 limbs) or
 * 5.2e5 points for squares.  All calls
 * share the array: calls that overlap on the GPU race; order them on one
 * stream. */
int nbg_mul_dev_noalloc(uint64_t *r, const uint64_t *a, int64_t m, const uint64_t *b, int64_t n, void *stream);

/* ---- batches ------------------------------------------------------------- */

/* One product of a batch.  b == NULL (or b == a with n == m) requests the
 * square of a.  bits_a / bits_b are the operands' magnitude bits
 * (64(n-1) + bit length of the top limb, kernels/addsub.jl:150); 0 asks the
 * library to read the top limbs itself (one device-to-host copy for device
 * batches). */
typedef struct nbg_desc {
    uint64_t *r;
    const uint64_t *a;
    const uint64_t *b;
    int64_t m;
    int64_t n;
    int64_t bits_a;
    int64_t bits_b;
} nbg_desc;

/* Whole batch in one call, host buffers, synchronous.  Products of any size
 * run together in one launch per pipeline step; the batch is cut into chunks
 * whose copies overlap the neighbouring chunks' products.  Results must not
 * overlap any operand of the batch.  Pinned (page-locked) buffers get
 * asynchronous DMA; contiguous operands are copied together. */
int nbg_mul_batch(const nbg_desc *descs, int64_t count);

/* Same with device buffers, asynchronous on `stream`. */
int nbg_mul_batch_dev(const nbg_desc *descs, int64_t count, void *stream);

/* Reusable batch over device buffers: plans, work queues and workspace are
 * built once and the launch sequence is captured in a CUDA graph; each run
 * replays it (operands may change between runs as long as their magnitude
 * bits do not). */
typedef struct nbg_batch nbg_batch;
int nbg_batch_create(const nbg_desc *descs, int64_t count, nbg_batch **out);
int nbg_batch_run(nbg_batch *bt, void *stream);
/* number of kernel launches one nbg_batch_run issues */
int nbg_batch_launches(const nbg_batch *bt);
int nbg_batch_destroy(nbg_batch *bt);
/* Per launch of a batch (up to cap): kernel kind (0 forward pass, 1 last pass
 * with pointwise product, 2 reverse pass, 3 unpack, 4 carry, 5 carries through
 * runs of all-ones limbs, 6 the last pass with one CTA per prime, 7 the last
 * pass of products with a kept operand spectrum, 8 and 9 the forward and
 * reverse column passes with tiles staged by TMA), jobs, and the
 * algorithmic FP64 instruction count and compulsory bytes of the reference
 * schedule for that launch.  Any output pointer may be NULL. */
int nbg_batch_stats(const nbg_batch *bt, int32_t *kinds, int64_t *njobs, double *alg_ops, double *alg_bytes,
                    int32_t cap);
/* Runs the batch's launches one by one (not as a graph) on `stream` with a
 * CUDA event between launches; ms[i] = duration of launch i. */
int nbg_batch_profile(nbg_batch *bt, void *stream, float *ms, int32_t cap);

/* ---- serving: continuous batching ------------------------------------------ */

/* A server owns a worker thread and an HBM arena of hbm_budget_bytes.
 * Requests submitted from any thread are batched as they arrive: while earlier
 * batches run (up to three in flight, each on its own stream) the worker forms
 * the next one from everything pending that fits in the free arena.
 * A new batch starts at once while fewer than two batches are in flight;
 * with two or more it starts when the pending requests hold at least
 * batch_points transform points (0: 2^23), or when the oldest pending request
 * has waited max_hold_us (0: 2000 us), so that under load batches stay
 * large enough to fill the GPU while an idle GPU still takes a lone request
 * immediately and no request waits on the point threshold for long.
 * max_batch bounds a batch (0: no bound); max_queue bounds
 * pending requests (0: no bound; past it nbg_submit returns NBG_EBUSY).
 * Requests whose result overlaps an operand fail with NBG_EINVAL. */
typedef struct nbg_server_opts {
    int64_t hbm_budget_bytes;
    int64_t max_batch;
    int64_t max_queue;
    int64_t batch_points;
    int64_t max_hold_us;
} nbg_server_opts;

typedef struct nbg_server_stats_t {
    int64_t completed;
    int64_t failed;
    int64_t pending;
    int32_t in_flight_batches;
    int32_t reserved;
    double p50_ms;             /* submit-to-completion latency percentiles */
    double p99_ms;
    double output_limbs_per_s; /* completed output limbs / (last completion - first submit) */
    int64_t batches;           /* batches launched */
    double mean_batch_requests;
} nbg_server_stats_t;

typedef struct nbg_server nbg_server;
int nbg_server_create(const nbg_server_opts *opts, nbg_server **out);
/* Host request: operands read (and the result written) through host pointers;
 * the buffers must stay valid until the request completes.  Returns a ticket. */
int nbg_submit(nbg_server *s, const nbg_desc *d, int64_t *ticket);
/* Device-resident request: device pointers, bits_a/bits_b required. */
int nbg_submit_dev(nbg_server *s, const nbg_desc *d, int64_t *ticket);
/* *done = 1 once the request finished; returns its status. */
int nbg_poll(nbg_server *s, int64_t ticket, int32_t *done);
/* Waits at most timeout_us for the request (NBG_ETIMEOUT after that). */
int nbg_wait(nbg_server *s, int64_t ticket, int64_t timeout_us);
/* Forgets a finished request's record. */
int nbg_release(nbg_server *s, int64_t ticket);
int nbg_server_stats(nbg_server *s, nbg_server_stats_t *st);
/* Drains the queue, stops the worker, frees the arena. */
int nbg_server_destroy(nbg_server *s);

/* ---- Barrett powermod chains ------------------------------------------------ */

/* One chain: r[0..k) = b^e mod m.  m has k limbs with m[k-1] != 0 and m > 1;
 * b has lb <= k limbs (any value, reduced mod m first); e has le limbs and is
 * nonzero.  The schedule is the reference's powermod_limbs
 * (src/algorithms.jl:17-107) on its Barrett branch (src/barrett.jl:33-81):
 * sliding window of width w(bits of e), a table of the odd powers b^1..b^(2^w-1),
 * and every multiply or square followed by barrett_reduce!. */
typedef struct nbg_powmod_desc {
    uint64_t *r;
    const uint64_t *b;
    const uint64_t *e;
    const uint64_t *m;
    int64_t lb, le;
} nbg_powmod_desc;

/* count chains sharing one modulus size k, run side by side on the GPU: each
 * exponent step is one square or multiply per chain plus the two Barrett
 * products, all three as batched fp-NTT products, the step captured in a CUDA
 * graph, the chains' state resident on the device.  Host buffers. */
int nbg_powermod_batch(const nbg_powmod_desc *d, int64_t count, int64_t k);
/* Same with device buffers (r, b, e, m device pointers), on `stream`; returns
 * after the work is queued (μ is computed on the host from a copy of m). */
int nbg_powermod_batch_dev(const nbg_powmod_desc *d, int64_t count, int64_t k, void *stream);
/* μ = floor(β^(2k) / m), β = 2^64, into mu[0..k+2); returns its normalized
 * length (k+1, or k+2 iff m = β^(k-1)), or -NBG_EINVAL when m[k-1] = 0.
 * Host only (barrett_mu!, src/barrett.jl:22-31). */
int64_t nbg_barrett_mu(const uint64_t *m, int64_t k, uint64_t *mu);
/* The chain's step list: ops[3*i .. 3*i+2] = (dst, src1, src2) slot indices,
 * slots 0..T-1 the odd-power table (T = 2^(w-1)), T = b^2, T+1 = accumulator,
 * T+2 = the raw base, T+3 = the constant 1; src2 = 255 marks a copy of src1.
 * Returns the number of steps, writing the first min(steps, cap) of them,
 * or -NBG_EINVAL for a zero exponent; the table size goes to *tsize.
 * Host only. */
int64_t nbg_powmod_schedule(const uint64_t *e, int64_t le, uint8_t *ops, int64_t cap, int32_t *tsize);

/* ---- sums of products (HGCD callers) --------------------------------------- */

/* M <- M * M1 for 2x2 matrices of nonnegative integers, device buffers, entry
 * order (m00, m01, m10, m11).  M's entries hold n limbs (zero-padded) and
 * have room for n + n1 + 1, which they receive; M1's hold n1.  The eight
 * products run as one GPU batch (zero entries drop out), the four sums on the
 * GPU.  Replaces hgcd_matrix_mul! (src/gcd.jl:371-389).  Returns when done. */
int nbg_matrix22_mul_dev(uint64_t *const *m, int64_t n, const uint64_t *const *m1, int64_t n1, void *stream);
/* r[0..rn) = a*x + b*y, nonnegative, device buffers, rn >= max(la+lx, lb+ly)+1
 * (cof_mul2!, src/gcd.jl:571-598).  Returns when done. */
int nbg_mul2add_dev(uint64_t *r, int64_t rn, const uint64_t *a, int64_t la, const uint64_t *x, int64_t lx,
                    const uint64_t *b, int64_t lb, const uint64_t *y, int64_t ly, void *stream);

/* Value of the little-endian base-bb chunks chunks[0..n) (each < bb, 2 <= bb)
 * as binary limbs: out[0..*out_len) normalized, cap >= n.  The reference's
 * subquadratic radix_combine (src/nbig.jl:410-417) with its power table by
 * repeated squaring (:396-399); every level's products run as one GPU batch.
 * Host buffers. */
int nbg_radix_combine(uint64_t *out, int64_t cap, const uint64_t *chunks, int64_t n, uint64_t bb, int64_t *out_len);

/* The power table of radix_chunks_dc (src/nbig.jl:394-399): entry 1 is bb,
 * entry i+1 the square of entry i, continued while the last entry is <= x
 * (x[0..xn), host buffer).  Entry i (0-based) is out[offsets[i] ..
 * offsets[i+1]), normalized; *entries gets the count (offsets needs
 * max_entries + 1 slots, out `cap` limbs; about 4*xn suffice).  Every square
 * runs on the GPU, the chain staying on the device. */
int nbg_radix_powtab(uint64_t *out, int64_t cap, int64_t *offsets, int32_t max_entries, uint64_t bb,
                     const uint64_t *x, int64_t xn, int32_t *entries);

/* ---- admission (host-side restatement of the reference's sizing) -------- */

/* fp_ntt_params (src/fpntt.jl:964-977): chunk width b and transform length N. */
int nbg_ntt_params(int64_t bits_a, int64_t bits_b, int32_t *b, int64_t *N);
/* ntt_len (src/fpntt.jl:936-951); NBG_ERANGE past 315*2^34. */
int nbg_ntt_len(int64_t T, int64_t *N);
/* magnitude_bits (src/kernels/addsub.jl:150) of a host operand. */
int64_t nbg_magnitude_bits(const uint64_t *a, int64_t n);

/* ---- transform-level entry points (device buffers; parity tests) --------- */

/* fp_ntt_pack! (src/fpntt.jl:744-768): x[0..N) = b-bit chunks of limbs, zero filled. */
int nbg_pack_dev(double *x, int64_t N, const uint64_t *limbs, int64_t n, int32_t b, int64_t nch, void *stream);
/* fp_ntt_fwd! / fp_ntt_rev! (src/fpntt.jl:715-733) in place, prime 0 or 1. */
int nbg_ntt_fwd_dev(double *x, int64_t N, int32_t prime, void *stream);
int nbg_ntt_rev_dev(double *x, int64_t N, int32_t prime, void *stream);
/* fp_ntt_pointwise! (src/fpntt.jl:770-785): xa[i] = mulmod(xa[i], xb[i]). */
int nbg_pointwise_dev(double *xa, const double *xb, int64_t N, int32_t prime, void *stream);
/* fp_ntt_unpack2! (src/fpntt.jl:869-925): r[0..rn) from the two reversed
 * transforms of length N (both primes), nconv coefficients of b bits. */
int nbg_unpack_dev(uint64_t *r, int64_t rn, const double *x1, const double *x2, int64_t N, int64_t nconv,
                   int32_t b, void *stream);

/* ---- plans and tuning ----------------------------------------------------- */

/* Pass structure chosen for length N: fills up to `cap` entries of
 * stage_m[] (radix per stage, forward order) and pass_end[] (last stage of each
 * pass); returns via *nst, *npass. */
int nbg_plan_info(int64_t N, int32_t *nst, int32_t *npass, int32_t *stage_m, int32_t *pass_end, int32_t cap);
/* Host-only view of the plan for length N under the current tuning (no
 * device needed): stages[3*i..] = (radix, span L, stride Q) in forward order,
 * passes[7*j..] = (first stage, last stage, rows G, columns C, column stride
 * Qb, tiles, rounds), rounds[j*cap + r] = (round kind << 8) | first stage
 * (rounds may be NULL).  `cap` bounds the entry counts. */
int nbg_plan_layout(int64_t N, int32_t sqr, int64_t *stages, int32_t *nst, int64_t *passes, int32_t *npass,
                    int32_t *rounds, int32_t cap);
/* Tuning knobs (JSON object, keys: full_max_mul, full_max_sqr, last_max,
 * last_max_sqr, early_gmax, tile_target, cmax, tma (1: column tiles staged by
 * TMA), queue (0: an nbg_batch replays one launch per pipeline step and
 * kernel kind; k in 1..64: one persistent work-queue launch whose CTAs claim
 * k jobs at a time and wait per product for the previous step), and
 * "overrides": a list of
 * {"N", "sqr", "pass_ends": [last stage of each pass], "tile_target", "cmax"}
 * giving an explicit pass split per transform class).  Changing them drops
 * cached plans. */
int nbg_set_tuning(const char *json);
/* Current tuning as a JSON object into buf (NUL-terminated). */
int nbg_get_tuning(char *buf, int64_t cap);
/* Applies a tuning file written by the autotuner ({"gpu", "version",
 * "tuning": {...}}) if it matches this GPU model and library version;
 * otherwise NBG_EINVAL and the current tuning stays.  On first use the
 * library loads $NBGPU_TUNING, else <lib dir>/../tuning/<GPU name>.json, when
 * present and matching. */
int nbg_load_tuning(const char *path);
/* Frees the twiddle tables of every cached plan (including those dropped by
 * a tuning change).  Only call it when no nbg_batch exists and no call is in
 * flight; plans are rebuilt on demand. */
int nbg_trim_plans(void);
/* Library version string (tuning files are keyed by it). */
const char *nbg_version(void);

/* ---- device / errors ------------------------------------------------------ */

int nbg_init(int32_t device);
const char *nbg_last_error(void);
/* the stream the synchronous host-buffer calls run on (a cudaStream_t) */
void *nbg_default_stream(void);
/* counters: kernel launches issued by this library since load */
int64_t nbg_launch_count(void);
/* Diagnostic, no counterpart in the reference: the number of bounded waits in
 * the library's kernels (the TMA tile loads of the column passes wait on an
 * mbarrier for at most about two seconds) that gave up on the current device
 * since the last call, after which the kernel returned early and its results
 * are invalid; reading clears the count.  Synchronizes the device. */
int nbg_device_faults(int64_t *count);
/* Diagnostic, no counterpart in the reference: the binary version (major * 10
 * + minor, cudaFuncGetAttributes) of the transform kernels as the CUDA runtime
 * loaded them on the current device, 100 for the sm_100a build; NBG_ECUDA
 * when the device cannot run them. */
int nbg_kernel_arch(int32_t *version);

#ifdef __cplusplus
}
#endif

#endif /* NBGPU_H */
