// engine.h — host engine internals shared by engine.cpp, api.cpp and serve.cpp.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "types.h"

namespace nbg {

int fail(int code, const char* fmt, ...);
const char* last_error();
extern std::atomic<int64_t> g_launches;

int64_t magnitude_bits(const uint64_t* a, int64_t n);
int64_t ntt_len(int64_t T);
int ntt_params(int64_t bits_a, int64_t bits_b, int* b_out, int64_t* N_out);

// An explicit pass split for one (transform length, square) class, chosen by
// the autotuner: the last stage of each pass, and the column-tile knobs.
struct SplitOverride {
    std::vector<int> pass_ends;
    int tile_target = 0;  // 0: the global value
    int cmax = 0;
};

// Pass-split knobs (the autotuner's search space).
struct Tuning {
    int full_max_mul = 2048;  // one-pass (whole transform in shared memory) up to this N, products
    int full_max_sqr = 4096;  // same for squares (one operand tile per prime)
    int last_max = 2048;      // largest contiguous block of the last pass, products
    int last_max_sqr = 4096;  // same for squares
    int early_gmax = 256;     // largest row count of an early (column) pass
    int tile_target = 4096;   // target doubles per column-pass tile (>= 16 G: TMA-eligible columns)
    int cmax = 128;           // most adjacent columns per column-pass tile
    int tma = 1;              // stage column tiles of at least 16 columns by TMA (0: cp.async for all)
    int queue = 0;            // > 0: reusable batches run as one persistent work-queue launch (k_queue)
                              // whose CTAs claim this many consecutive jobs at a time (at most 64)
    std::map<int64_t, SplitOverride> overrides;  // key: N * 2 + square
    std::string to_json() const;
    int from_json(const char* js);
};

// shared memory the pass kernels may use per CTA (B200 opt-in is 227 KB)
constexpr size_t PASS_SMEM_LIMIT = 220 * 1024;

int plan_structure(int64_t N, int for_sqr, const Tuning& tun, DPlan& d);
int plan_rounds(DPlan& d);

struct PlanRec {
    DPlan d;
    double* dtab = nullptr;
    size_t table_bytes = 0;
    int slot = -1;
};

struct Engine {
    bool ready = false;
    int dev = -1;
    int num_sms = 0;
    int smem_optin = 0;
    cudaStream_t stream = nullptr;   // compute
    cudaStream_t copy_in = nullptr;  // host-to-device copies of the pipelined host calls
    cudaStream_t copy_out = nullptr; // device-to-host copies
    cudaStream_t side[4] = {};       // parallel branches of one pipeline step (host-buffer batches)
    cudaEvent_t hb_ev[3][4] = {};    // host-buffer batches: per slot, operands in / computed / results out
    std::recursive_mutex mu;
    Tuning tun;
    std::map<int64_t, PlanRec> plans;
    std::vector<double*> graveyard;
    DPlan* d_plans = nullptr;
    int plan_cap = 4096;
    int plan_used = 0;
    void* pool = nullptr;
    size_t pool_bytes = 0;
    // pinned staging for the descriptor/job-table head of each pipelined chunk
    char* stage[4] = {};
    size_t stage_bytes[4] = {};
    // pinned staging of operands and results that live in pageable host
    // memory (host-buffer batches), per pipeline slot; allocated on first need
    char* pg_in[4] = {};
    size_t pg_in_bytes[4] = {};
    char* pg_out[4] = {};
    size_t pg_out_bytes[4] = {};

    int init(int device);
    int ensure();
    int build_plan(int64_t N, PlanRec& pr, int for_sqr);
    int get_plan(int64_t N, int for_sqr, PlanRec** out);
    void drop_plans();
    void trim_plans();  // frees every plan's tables: no batch may exist or be running
    int ensure_pool(size_t bytes);
    int ensure_stage(int i, size_t bytes);
};
extern Engine g_eng;

// One product as the batch builder sees it (device pointers).
struct ProdIn {
    const uint64_t* a;
    const uint64_t* b;
    uint64_t* r;
    int64_t m, n;
    int64_t bits_a, bits_b;
    int sqr;
    // one-pass products only: keep operand b's spectrum in workspace (PF_BSAVE)
    int keep_b = 0;
};

struct Launch {
    int kind;
    int64_t off, n;        // explicit lists: first job and count; batches: n = job count
    size_t smem;
    // batches: where the launch's jobs are described (JobMode), as byte
    // offsets into the batch's job table
    int mode = JM_LIST;
    int nseg = 0;
    size_t seg_off = 0, plist_off = 0;
    int step = 0;          // pipeline step: launches of one step are independent
    bool odd = true;       // some pass of the launch holds a radix-3/5/7 stage
    double alg_ops = 0;    // FP64 instructions of the reference schedule done by this launch
    double alg_bytes = 0;  // compulsory global bytes (operand/limb reads, tile loads and stores)
};

struct BatchBuild {
    std::vector<DProd> prods;
    std::vector<PlanRec*> plan_of;
    std::vector<char> table;  // job table: per launch segments and product lists, then tile starts
    size_t tstart_off = 0;    // per-product first unpack tile (count + 1 int64), in the table
    size_t expand_off = 0;    // ExpandEntry per launch, in the table (written by bind_batch)
    int64_t total_jobs = 0;   // explicit jobs, written on the device by the expansion kernel
    size_t off_joblist = 0;   // region offset of that job list
    size_t head_bytes = 0;    // [0, head_bytes): descriptors and table, the host-written head
    std::vector<Launch> launches;
    std::vector<size_t> xa_off, xb_off, agg_off;
    // product classes (one plan, one kept-spectrum flag): contiguous transform
    // buffers, and the tensor maps of their TMA column passes
    struct ClassRec {
        size_t xa0 = 0, xb0 = 0;  // first buffers (doubles into the workspace); xb0 SIZE_MAX: none
        int32_t nprod = 0;
        int32_t map0 = -1;        // first of 2 * (passes - 1) tensor maps ([pass][operand]); -1: none
        uint32_t tma_mask = 0;    // column passes staged by TMA
        const PlanRec* plan = nullptr;
    };
    std::vector<ClassRec> classes;
    std::vector<int32_t> class_of;  // per product
    size_t tmap_off = 0;            // tensor maps in the table (128 B each)
    int ntmaps = 0;
    size_t work_doubles = 0, agg_words = 0;
    size_t off_prods = 0, off_jobs = 0, off_work = 0, off_agg = 0, dev_bytes = 0;
};

int build_batch(Engine& E, const ProdIn* in, int64_t count, BatchBuild& bb);
int upload_batch(Engine& E, BatchBuild& bb, char* dbase, cudaStream_t st);
// Points each product's workspace and carry words into the batch's device
// region at dbase and encodes the TMA tensor maps over it (what upload_batch
// does before copying).
int bind_batch(BatchBuild& bb, char* dbase);
// Writes the bound descriptors and job table into `host` in their device
// layout: head_bytes that one copy to dbase makes the region's head.
void stage_batch(const BatchBuild& bb, char* host);
// Writes the batch's explicit job list on the device (one kernel); the
// run_launches functions do this before the batch's first launch.
cudaError_t expand_jobs(const BatchBuild& bb, char* dbase, cudaStream_t st);
// The job source of launch L of a batch whose region starts at dbase.
JobSrc launch_src(const BatchBuild& bb, const Launch& L, const char* dbase);
// expand = false reuses the job list a previous run wrote (same region).
int run_launches(Engine& E, const BatchBuild& bb, char* dbase, cudaStream_t st, bool expand = true);
// Work-queue execution of a batch: one persistent launch (k_queue) walks the
// batch's jobs in pipeline-step order.  d: [QState | done | need | table],
// the first zero_bytes cleared before every run.
struct QueueRun {
    char* d = nullptr;
    size_t bytes = 0, zero_bytes = 0;
    size_t off_done = 0, off_need = 0, off_ql = 0;
    int nl = 0;
    int64_t total = 0;
    size_t smem = 0;
    int grid = 0;
    int chunk = 1;  // consecutive jobs per claim
};
// Allocates and fills q for a bound, uploaded batch (expands its job list and
// counts each product's jobs per step); NBG_EINVAL when a tile set and an
// unpack stage do not fit one CTA's shared memory.
int queue_prepare(Engine& E, const BatchBuild& bb, char* dbase, QueueRun& q, cudaStream_t st);
// One run: clears the queue state, expands the job list, launches k_queue.
int queue_run(Engine& E, const BatchBuild& bb, char* dbase, const QueueRun& q, cudaStream_t st);
void queue_free(QueueRun& q);
// run_launches with the independent launches of each step forked onto `side`
// streams (used while capturing a CUDA graph, where they become parallel branches).
int run_launches_branched(Engine& E, const BatchBuild& bb, char* dbase, cudaStream_t st, cudaStream_t* side,
                          int nside);

}  // namespace nbg
