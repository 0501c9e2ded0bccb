// Internal engine interfaces: device layout of the graph, the move levels and
// the module state, and the launchers of every hot-path kernel.
//
// HBM layout (structure of arrays; N nodes, E kept links):
//   node CSR  out_off[N+1] i64 | out_dst[E] i32 | out_w0[E] f64 (summed input
//             weight) | out_f[E] f64 (normalised weight, then flow) | out_fx[E]
//   node CSC  in_off[N+1] i64 | in_src[E] i32 | in_w[E] f64 (normalised) | in_fx[E]
//   nodes     tw[N] f64 teleport weight | dangling[N] u8 | p[N] f64 flow
//   units     attr[n] Stat4 (fixed-point P, TW, D, OUT) | mod[n] | inst[n] | nnodes[n]
//   modules   stat[M] Stat4 | count[M] i32 | inst[M] i32        (M = N ids)
// A "level" is the set of moving units: nodes, super-nodes (modules of the
// previous stage) or sub-module super-nodes (coarse-tune), each with its own
// CSR/CSC of aggregated fixed-point flows.
#pragma once
#include <vector>

#include "rmx_common.cuh"
#include "rmx_prims.cuh"

namespace rmx {

struct Level {
    int32_t n = 0;      // units
    int64_t m = 0;      // links
    int64_t *out_off = nullptr, *in_off = nullptr;
    int32_t *out_dst = nullptr, *in_src = nullptr;
    int32_t *out_src = nullptr;  // row of every out-link (levels that are coarsened again)
    fx_t *out_fx = nullptr, *in_fx = nullptr;
    Stat4 *attr = nullptr;
    int32_t *mod = nullptr;     // module id of each unit
    int32_t *inst = nullptr;    // instance (independent sub-problem) of each unit
    int32_t *nnodes = nullptr;  // original nodes inside each unit
};

// A module's statistics and cached terms in one 64-byte record (two sectors
// of one 128-byte line): what the move evaluation reads per candidate, so a
// candidate costs one random line instead of one in each of two arrays.
struct __align__(64) ModRec {
    Stat4 s;
    double2 t;
    double2 pad;
};

struct ModState {
    int32_t cap = 0;
    Stat4 *stat = nullptr;
    double2 *term = nullptr;    // cached {plogp(exit), plogp(exit + P)} of each module
    ModRec *rec = nullptr;      // stat and term together, written with term (read by the evaluation)
    int32_t *count = nullptr;   // units of the current level in the module
    int32_t *inst = nullptr;
};

// Per-instance code-length bookkeeping (one instance = the whole graph, or
// one sub-problem of the coarse-tune / batched engine).
struct InstState {
    int32_t n = 0;
    double *sum_exit = nullptr;   // sum of module exits
    double *L = nullptr;          // code length (nats)
    double *L_prev = nullptr;     // at the start of the current stage step
    fx_t *s0 = nullptr;           // sum p log p of member nodes (fixed 2^-58)
    fx_t *acc = nullptr;          // 3 per instance: sum exit, sum plogp(q), sum plogp(q+P)
    uint8_t *active = nullptr;    // still iterating
};

// Sweep parameters passed to the move kernels.
struct SweepArgs {
    double vthresh;          // accept when best change < vthresh (<= 0)
    int allow_new;           // empty-module candidate enabled for this stage
};

// ---------------------------------------------------------------- graph build
struct CsrBuild {
    int64_t n_links = 0, n_self = 0;
};
// Sort + sum duplicate pairs, drop self-loops and non-positive sums, build CSR
// and CSC. src/dst/w are device arrays of n_edges entries (consumed).
CsrBuild build_csr(int32_t n, int64_t n_edges, int32_t *d_src, int32_t *d_dst, double *d_w, int64_t *out_off,
                   int32_t *out_dst, double *out_w0, int64_t *in_off, int32_t *in_src, double *in_w, Arena &ar,
                   cudaStream_t s, int64_t *self_count_dev);

// ---------------------------------------------------------------- flows
// Row-normalise (CSR and CSC), power iteration, edge flows, unit attributes.
struct FlowOut {
    int iters = 0;
};
// alpha: teleportation probability (the reference's 0.15 unless a caller varies it).
int power_iteration(int32_t n, const int64_t *in_off, const int32_t *in_src, const double *in_w, const double *tw,
                    const uint8_t *dangling, double *p, Arena &ar, cudaStream_t s, int vec, double alpha = kAlpha);
// The same solve writing into caller-provided scratch (y[n], parts[3*max_blocks],
// iters on the device); asynchronous, allocates nothing.
void power_iteration_into(int32_t n, const int64_t *in_off, const int32_t *in_src, const double *in_w,
                          const double *tw, const uint8_t *dangling, double *p, double *y, double *parts,
                          int max_blocks, int *iters, cudaStream_t s, int vec);
// The stationary flow of every component of a disjoint union: one block per
// canonical component (comp: [lo, hi) node ranges, device), then every other
// instance copies its canonical instance's flow. Returns the largest
// iteration count.
int power_iteration_components(int32_t n, int32_t n_comp, const int64_t *comp, const int32_t *node_inst,
                               const int64_t *inst_noff, const int32_t *inst_canon, const int64_t *in_off,
                               const int32_t *in_src, const double *in_w, const double *tw, const uint8_t *dangling,
                               double *p, Arena &ar, cudaStream_t s, int vec);
// Sub-warp width of the pull SpMV for a mean in-degree.
int spmv_width(double mean_in_degree);
// cols: also normalise the CSC weights (in place when in_w_raw == in_w: once).
void normalise(int32_t n, const int64_t *out_off, const double *out_w0, double *out_f, const int64_t *in_off,
               const int32_t *in_src, const double *in_w_raw, double *in_w, uint8_t *dangling, Arena &ar,
               cudaStream_t s, bool cols = true);
void edge_flows(int32_t n, int64_t m, const int64_t *out_off, double *out_f, fx_t *out_fx, const int32_t *in_src,
                const double *in_w, fx_t *in_fx, const double *p, const double *tw, const uint8_t *dangling,
                Stat4 *attr, fx_t *s0_acc, cudaStream_t s);
void singleton_exits(int32_t n, const int64_t *out_off, const double *out_f, const double *p, const double *tw,
                     const uint8_t *dangling, double *exitpr, cudaStream_t s);

// ---------------------------------------------------------------- moves
void init_singletons(const Level &L, ModState &M, cudaStream_t s);
void module_stats_from_units(const Level &L, ModState &M, cudaStream_t s);
void count_units(const Level &L, ModState &M, cudaStream_t s);
// Refresh the cached log terms of every module from its statistics.
void refresh_terms(ModState &M, cudaStream_t s);
// Code length per instance from the module statistics.
void instance_codelength(const ModState &M, InstState &I, cudaStream_t s);

// Counter slots in SweepWork::counters (device int64). kCntMods: non-empty
// modules at the start of the current sweep (counted only while profiling).
// kCntBins: per degree bin of the move evaluation (register, warp, mid,
// block, large, hub), links read, units evaluated and candidates evaluated
// (cumulative).
enum {
    kCntActive = 0, kCntFree = 1, kCntMoved = 3, kCntMods = 7, kCntBins = 8, kEvalBins = 6,
    kCntSlots = kCntBins + 3 * kEvalBins
};

// Device time per kernel class, recorded with CUDA events on the stream.
enum {
    kTimerSpmv = 0, kTimerEval, kTimerCommit, kTimerCoarsen, kTimerCodelen, kTimerOther, kTimerAdjoint,
    // whole sweep loops by level (they contain the kernel classes above)
    kTimerLvNode, kTimerLvSN, kTimerLvSub,
    // each degree bin of the move evaluation (register, warp, mid, block, large, hub)
    kTimerBinReg, kTimerBinWarp, kTimerBinMid, kTimerBinBlock, kTimerBinLarge, kTimerBinHub, kTimerCount
};
struct Timers {
    bool on = false;
    std::vector<cudaEvent_t> pool;
    size_t used = 0;
    struct Pending {
        int k;
        cudaEvent_t a, b;
    };
    std::vector<Pending> pending;
    cudaEvent_t open[kTimerCount] = {};
    double ms[kTimerCount] = {};
    int64_t launches[kTimerCount] = {};
    // Compulsory bytes of the move evaluation, per launch group (one
    // sub-batch's bins): 16 B per link read (neighbour id 4, fixed-point flow
    // 8, neighbour's module 4), 40 B per unit (module id 4, statistics 32,
    // proposal written 4), and the module statistics (40 B) once per launch,
    // at most one per candidate: 40 * min(candidates, non-empty modules).
    // The same per degree bin (each bin's kernel reads its own statistics).
    // Each launch group appends the running counters to a device log
    // (log_eval); resolve() turns consecutive entries into per-launch counts.
    static constexpr int kLogWords = 1 + 3 * kEvalBins;  // non-empty modules, then the bin counters
    int64_t *dlog = nullptr;
    int64_t nlog = 0, logcap = 0;
    cudaStream_t log_stream = nullptr;  // the stream the log entries were written on
    int64_t last[3 * kEvalBins] = {};
    double eval_bytes = 0.0;
    double eval_bin_bytes[kEvalBins] = {};
    void begin(int k, cudaStream_t s);
    void end(int k, cudaStream_t s);
    void log_eval(const int64_t *counters, cudaStream_t s);
    void resolve();  // synchronises on the recorded events
    void reset();
    void destroy();
};


// Per-level sweep workspace (sized for the largest level: N units, N modules).
struct SweepWork {
    int32_t *list = nullptr, *list2 = nullptr;  // active units; active units grouped by bucket
    uint16_t *bucket = nullptr;
    int64_t *bucket_off = nullptr;              // nsub * 3 + 1 bucket boundaries (device)
    int64_t *ranges = nullptr;                  // [beg,end) of each sub-batch (device)
    int32_t *prop = nullptr;                    // proposed module (-1 none, -2 empty module)
    double *pdelta = nullptr;
    int32_t *ptarget = nullptr;                 // claimed empty module
    int32_t *prevmod = nullptr;
    uint32_t *stamp = nullptr;                  // sub-batch stamp of the last move of a unit
    uint8_t *next_active = nullptr;
    int32_t *free_list = nullptr;
    unsigned long long *claim = nullptr;        // per module id
    int64_t *counters = nullptr;
    // hub units (above the large bin's bound), each split over many blocks:
    // the plan arrays (per unit), the partition arrays (per partition) and
    // the buckets of partitioned links (hub_links entries), sized for every
    // hub unit of the current level
    int64_t hub_units = 0, hub_parts = 0, hub_links = 0, hub_chunks = 0;  // capacities
    int64_t hub_gen = 0;                                   // allocations so far
    int64_t *hub_coff = nullptr, *hub_poff = nullptr, *hub_loff = nullptr, *hub_pstart = nullptr;
    int32_t *hub_nparts = nullptr, *hub_cunit = nullptr, *hub_punit = nullptr;
    fx_t *hub_own = nullptr;
    uint8_t *hub_act = nullptr;
    unsigned long long *hub_pcnt = nullptr;
    double *hub_best = nullptr;
    int32_t *hub_bmod = nullptr;
    int32_t *hub_bkey = nullptr;
    int32_t *hub_lkey = nullptr;   // per hub link: its neighbour's module (count pass -> scatter pass)
    fx_t *hub_bfx = nullptr;
    int64_t *hub_tot = nullptr;
    std::vector<int64_t> bucket_host;  // host copy of bucket_off after bucket_units
    uint32_t *dparams = nullptr;       // device {stamp, hseed} per sub-batch of the current sweep
    uint32_t hparams[64] = {};         // host staging of dparams
    cudaStream_t aux[5] = {};  // concurrent degree bins
    cudaEvent_t fork = nullptr, join[5] = {};
};

void configure_eval_kernels();
// What the hub pipeline needs for a level: hub units (above
// block_bin_max_degree), their partitions, their links and their link chunks
// (out[0..3]); one device reduction, then a sync.
void hub_level_needs(const Level &L, int64_t *out, int64_t *dev_tmp, cudaStream_t s);

// Launch shape of move evaluation, process-wide and read at every launch:
// the grid cap of each bin in blocks per SM, and the degree bounds that
// assign units to the warp, mid, block and large bins (units above large_max
// go to the hub bin). Results do not depend on them (each bin's kernel loops
// over its units by grid stride, every bin computes the same exact integer
// sums and the same change per candidate), only the time does. The hub bin's
// grid is not tuned: its global table slices are indexed by block.
struct EvalTuning {
    int mid, block, large, warp, reg;              // grid caps
    int warp_max, mid_max, block_max, large_max;   // degree bounds (at most 128, 512, 1024, 4096)
    int hub_part;                                  // mean links per partition of a hub unit / huge group
};
EvalTuning eval_tuning();
// Throws std::invalid_argument unless every grid cap lies in [1, 64] and
// 32 <= warp_max <= mid_max <= block_max <= large_max, each within its bin's
// table limit, and 64 <= hub_part <= 2^30.
void set_eval_tuning(const EvalTuning &t);
// Changes with every set_eval_tuning (part of the sweep graph cache key).
int eval_tuning_generation();
// Units above this degree need the hub bin's global tables.
int64_t block_bin_max_degree();
void all_units(int32_t n, SweepWork &W, cudaStream_t s);
// host_counts: also copy the bin offsets to W.bucket_host (one stream sync).
void bucket_units(const Level &L, SweepWork &W, int64_t n_active, uint32_t seed, int nsub, Arena &ar, cudaStream_t s,
                  bool host_counts = true);
// bucket_units for a captured sweep: the active count (counters[kCntActive])
// and the seed are read on the device; grids are sized for n_max units.
void bucket_units_dev(const Level &L, SweepWork &W, int64_t n_max, const uint32_t *seed_dev, int nsub, Arena &ar,
                      cudaStream_t s);
// all_units for *n_dev units (device), grids sized for n_max.
void all_units_dev(const int64_t *n_dev, int64_t n_max, SweepWork &W, cudaStream_t s);
void free_modules(const ModState &M, SweepWork &W, Arena &ar, cudaStream_t s);
// Evaluate, claim, commit and apply link deltas for sub-batch sb.
// sp: device {stamp, hseed} of the sub-batch. stamp: unique per sub-batch over
// the handle's life (marks this sub-batch's movers); hseed: a function of
// (attempt seed, sweep, sub-batch) only, so runs with the same seed make the
// same choices. fitted: use the host bin sizes (see bucket_units).
void sweep_subbatch(const Level &L, ModState &M, const InstState &I, SweepWork &W, const SweepArgs &a, int sb,
                    const uint32_t *sp, bool mark_active, bool fitted, cudaStream_t s, Timers *tm);
// Move evaluation only, for the parity hook (no commit).
void evaluate_all(const Level &L, const ModState &M, const InstState &I, SweepWork &W, const uint8_t *allow_new,
                  double vthresh, Arena &ar, cudaStream_t s);

// ---------------------------------------------------------------- coarsening
// Group nodes by group[v] (0..ng-1) and aggregate the node CSR into a group
// CSR/CSC: FP64 sums in node/link order (bit-exact to the reference) and
// fixed-point sums for the engine. Returns the number of group links.
int64_t coarsen_links(int32_t n, const int64_t *out_off, const int32_t *out_dst, const double *out_f,
                      const fx_t *out_fx, const int32_t *group, int32_t ng, int64_t *g_out_off, int32_t *g_out_dst,
                      double *g_out_f, fx_t *g_out_fx, int64_t *g_in_off, int32_t *g_in_src, double *g_in_f,
                      fx_t *g_in_fx, Arena &ar, cudaStream_t s);

// Engine aggregation of rows (nodes or super-nodes) into groups by hashing:
// fixed-point sums only, rows and columns in no particular order. src: the
// row of every input link (CSR order); g_out_src receives the row (group) of
// every output link. rowsum (may be NULL) receives each group's total
// out-flow. gtab / gtab_cap: a global table in gtab_arena, grown on demand for
// groups too large for shared memory. W (may be NULL): auxiliary streams and
// events on which the size bins run concurrently.
int64_t aggregate_links(int32_t n, const int64_t *off, const int32_t *dst, const fx_t *fx, const int32_t *src,
                        const int32_t *group, int32_t ng, int64_t *g_out_off, int32_t *g_out_dst, fx_t *g_out_fx,
                        int32_t *g_out_src, int64_t *g_in_off, int32_t *g_in_src, fx_t *g_in_fx, fx_t *rowsum,
                        Arena &gtab_arena, fx_t *&gtab, int64_t &gtab_cap, Arena &ar, cudaStream_t s,
                        const SweepWork *W);
// src[e] = the row of link e for the CSR offsets off[0..n] (a warp per row).
void rows_of_links(int32_t n, const int64_t *off, int32_t *src, cudaStream_t s);

}  // namespace rmx
