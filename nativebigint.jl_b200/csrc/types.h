// types.h — plan, product and job descriptors shared by host and device code.
//
// A transform of length N = m*2^k is the reference's flat stage list
// (src/fpntt.jl:236-271): odd Winograd stages 7,5,3,3 (those dividing m), the
// radix-4 tower, and a twiddle-free radix-2 stage when k is odd.  Stage s has
// span L_s (its butterflies run inside L_s-blocks) and stride Q_s = L_s/m_s;
// its twiddle for lane t, column j is omega^((N/L_s)*t*j) in minimal balanced
// form, stored t-major: tw[(t-1)*Q_s + j].
//
// On the GPU a contiguous run of stages [sa, sb] is one *pass*: every pass
// tile is G = L_sa/Q_sb rows by C adjacent columns of stride Qb = Q_sb, held in
// shared memory while all the pass's butterflies run.  The last pass always has
// Qb = 1 (a contiguous G-block), so the pointwise product and the reverse's
// first pass run on the same tile.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define NBG_HD __host__ __device__
#else
#define NBG_HD
#endif

namespace nbg {

constexpr int MAXST = 24;    // 4 odd + 17 radix-4 + radix-2 at N = 315*2^34
constexpr int MAXPASS = MAXST;

struct DStage {
    int32_t m;           // radix 2, 3, 4, 5, 7
    int32_t pad_;
    int64_t L;           // span
    int64_t Q;           // L / m
    const double* tw[2]; // per prime, (m-1)*Q doubles (null for radix-2)
    double rot[2][8];    // per prime combine constants (radix-4: rot[0] = wi)
};

// Round kinds: how a pass's stages are executed in shared memory.
enum RoundKind : int8_t {
    RK_ODD = 0,  // one radix-3/5/7 stage, one butterfly per work unit
    RK_R4 = 1,   // one radix-4 stage
    RK_R16 = 2,  // radix-4 stages s (span L) and s+1 (span L/4) on 16 registers per unit
    RK_R8 = 3,   // radix-4 stage s (span 8) and the radix-2 stage s+1 on 8 registers per unit
    RK_R2 = 4,   // a lone radix-2 stage
};

struct DPass {
    int32_t sa, sb;      // stage range, inclusive
    int32_t G;           // rows per tile = L_sa / Q_sb
    int32_t C;           // columns per tile (power of two dividing Qb)
    int64_t Qb;          // column stride = Q_sb
    int64_t ntiles;      // (N / L_sa) * (Qb / C)
    int32_t nrounds;
    int8_t rkind[MAXST]; // forward order; the reverse runs them backwards
    int8_t rstage[MAXST];// first stage of each round
};

struct DPlan {
    int64_t N;
    int32_t nst, npass;
    double ninv[2], ninvp[2]; // 1/N mod p (minimal balanced) and ninv/p
    DStage st[MAXST];
    DPass pass[MAXPASS];
};

// One product r[0..rn) = a[0..m) * b[0..n) (b == a for a square).
struct DProd {
    const uint64_t* a;
    const uint64_t* b;
    uint64_t* r;
    int64_t m, n, rn;
    int64_t nca, ncb, nconv;
    int32_t bch;         // chunk width in bits
    int32_t sqr;         // 1: square (one operand transform per prime)
    int32_t plan;        // index into the device plan array
    int32_t npass;
    int32_t flags;       // PF_* bits
    int32_t tslot;       // TMA column passes: index of the product in its class's buffers (z = 2 * tslot + prime)
    const void* tmap;    // TMA column passes: the class's tensor maps, 128 B each, [pass][operand]
    double* xa[2];       // per-prime transform buffers of operand a (and the result)
    double* xb[2];       // per-prime buffers of operand b (multi-pass products only)
    uint32_t* agg;       // per limb-tile carry aggregates (bit0 generate, bit1 propagate)
    int64_t ntl;         // number of limb tiles
};

// Work item of one launch.  kind-specific meaning of `sub`:
//   k_fwd: bit 1 operand (0 = a, 1 = b), pass index in bits 8..15
//   k_rev: pass index in bits 8..15
//   (pass kernels process both primes of a tile; unpack/carry ignore `sub`).
struct Job {
    int32_t prod;
    int32_t sub;
    int64_t tile;
};

// Work-queue execution of a batch (one persistent launch): the batch's
// launches, in pipeline-step order, as consecutive ranges of queue positions.
// Queue position g lies in entry k when qstart[k] <= g < qstart[k + 1]; its
// job is jobs[off + g - qstart].  A last entry holds the total in qstart.
struct QLaunch {
    int64_t qstart;
    int64_t off;
    int32_t kind;  // JobKind (no JK_CARRYFIX: the carry job fixes its own tiles)
    int32_t odd;
};
// Queue state, zeroed before every run.
struct QState {
    unsigned long long head;  // next queue position to claim
    unsigned int abort;       // a bounded wait gave up: every CTA leaves
    unsigned int pad_;
};
// Per product, the jobs of each of its pipeline steps: forward passes
// 0..npass-2, the last pass (npass-1), reverse passes (npass..2 npass-2),
// unpack (2 npass-1) and carry (2 npass).
constexpr int QSTEPS = 2 * MAXPASS + 2;

// A run of jobs of one plan class inside a launch: jobs [begin, begin +
// ntiles * nop * nprod), ordered tile-major, then operand, then product, so
// CTAs that run together read the same twiddle slice.  The class's products
// are plist[first .. first + nprod).
struct JobSeg {
    int64_t begin;
    int64_t ntiles;
    int32_t nop, nprod;
    int32_t first, sub_base;
    // column passes: tiles are visited column-major, so consecutive jobs (and
    // the jobs one CTA runs in a row) read the same twiddle columns: the
    // t-th visited tile is (t % nblk) * per + t / nblk, per = tiles per block
    // row (Qb / C), nblk = ntiles / per.  per = 0: tiles in index order.
    int32_t per, nblk;
};

// Where a launch's jobs come from.  Batches describe them implicitly, so the
// host writes a few bytes per plan class or product instead of one Job per CTA.
enum JobMode : int32_t {
    JM_LIST = 0,     // list[ji]
    JM_SEGS = 1,     // segs[nseg] over plist
    JM_TILES = 2,    // product k owns jobs [tstart[k], tstart[k+1]): tile = ji - tstart[k]
    JM_PERPROD = 3,  // job ji is product ji, tile 0
};
struct JobSrc {
    const Job* list;
    const JobSeg* segs;
    const int32_t* plist;
    const int64_t* tstart;
    int32_t mode, nseg;
    int64_t nprod;  // JM_TILES: products in tstart (tstart has nprod + 1 entries)
};

// One launch of a batch for the job-expansion kernel: jobs [begin, begin + n)
// of the batch's job list are jobs 0..n-1 of src.
struct ExpandEntry {
    JobSrc src;
    int64_t begin, n;
};

// Job ji of a launch described by s (ji < the launch's job count).
NBG_HD inline Job job_at(const JobSrc& s, int64_t ji) {
    Job j;
    if (s.mode == JM_LIST) return s.list[ji];
    if (s.mode == JM_PERPROD) {
        j.prod = (int32_t)ji;
        j.sub = 0;
        j.tile = 0;
        return j;
    }
    if (s.mode == JM_TILES) {  // last k with tstart[k] <= ji
        int64_t lo = 0, hi = s.nprod - 1;
        while (lo < hi) {
            const int64_t mid = (lo + hi + 1) >> 1;
            if (s.tstart[mid] <= ji) lo = mid;
            else hi = mid - 1;
        }
        j.prod = (int32_t)lo;
        j.sub = 0;
        j.tile = ji - s.tstart[lo];
        return j;
    }
    int lo = 0, hi = s.nseg - 1;  // last segment with begin <= ji
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (s.segs[mid].begin <= ji) lo = mid;
        else hi = mid - 1;
    }
    const JobSeg g = s.segs[lo];
    const int64_t local = ji - g.begin;
    const int64_t per_tile = (int64_t)g.nop * g.nprod;
    const int64_t t = local / per_tile;
    const int64_t r = local - t * per_tile;
    const int32_t op = (int32_t)(r / g.nprod);
    j.prod = s.plist[g.first + (int32_t)(r - (int64_t)op * g.nprod)];
    j.sub = g.sub_base | (op << 1);
    j.tile = g.per ? (t % g.nblk) * g.per + t / g.nblk : t;
    return j;
}

enum JobKind : int32_t {
    JK_FWD = 0,   // forward pass (pass 0 packs limbs on load)
    JK_PWR = 1,   // last pass: forward, pointwise, reverse (packs when npass == 1)
    JK_REV = 2,   // reverse pass
    JK_UNPACK = 3,// Garner + limb assembly + in-tile carries
    JK_CARRY = 4, // cross-tile carry scan and fix-up (one job per product)
    JK_CARRYFIX = 5, // carries through runs of all-ones limbs (one job per unpack tile)
    JK_PWR_SPLIT = 6,// JK_PWR with one job per prime (sub bit 1) for small batches
    JK_PWR_KEEP = 7, // JK_PWR for products with a kept operand spectrum (PF_BSAVE / PF_BSPEC)
    JK_FWD_TMA = 8,  // JK_FWD with tiles staged by TMA (DProd.tmap; at least 16 columns per tile)
    JK_REV_TMA = 9,  // JK_REV with tiles staged by TMA
};

constexpr int UNPACK_TL = 1024;  // output limbs per unpack tile
// Residues staged per prime for one unpack tile of chunk width b: the
// coefficients that start in bits [64 (w0 - 4), 64 (w0 + UNPACK_TL)), plus one
// double at each end for the 16-byte alignment of the bulk copy (kept even).
NBG_HD inline int64_t unpack_stage_doubles(int b) {
    const int64_t ncoef = (64 * (int64_t)(UNPACK_TL + 4)) / b + 2;
    return (ncoef + 3) & ~(int64_t)1;
}
// Dynamic shared memory of the unpack kernel: 128 bytes of mbarriers, then two
// stages (the tile being assembled and the next one in flight) of both primes'
// staged residues.  For the chunk widths of transforms up to 2^32 points
// (b >= 33) this is at most 64 KB.
NBG_HD inline size_t unpack_smem_bytes(int b) { return 128 + 2 * 2 * 8 * (size_t)unpack_stage_doubles(b); }
constexpr int PASS_THREADS = 256;

// Shared-memory tiles are padded by one double every 16 so that strided
// accesses of the radix-16/8 rounds fall in distinct banks.
NBG_HD inline int tile_pad_index(int i) { return i + (i >> 4); }
NBG_HD inline int tile_stride_doubles(int n) { return ((n + (n >> 4) + 1) + 1) & ~1; }

// DProd.flags
constexpr int32_t PF_PRELOADED = 1;  // pass 0 loads xa/xb as-is instead of packing limbs
// One-pass products whose operand b is the same on every run (a modulus or a
// reciprocal in the powermod chains): a run with PF_BSAVE stores b's forward
// transform (both primes) in xb; runs with PF_BSPEC load it from there instead
// of packing and transforming b again.
constexpr int32_t PF_BSAVE = 2;
constexpr int32_t PF_BSPEC = 4;

}  // namespace nbg
