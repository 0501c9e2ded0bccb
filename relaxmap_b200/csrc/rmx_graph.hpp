// The opaque handle behind the C ABI: one graph resident on one device, its
// CUDA stream, the device arenas, and the engine state of the optimiser.
#pragma once
#include <functional>
#include <string>
#include <vector>

#include "../../include/relaxmap_b200.h"
#include "rmx_engine.cuh"

// A disjoint union of K instances (host arrays): node_inst[N] the instance of
// every node, inst_noff[K+1] their node ranges, inst_canon[K] the first copy
// of the same graph (whose flow the instance shares; k itself if first).
// With n_canon > 0 the edge arrays describe only the canonical copies, their
// nodes numbered 0..n_canon-1 in instance order, and every other copy is
// written on the device from its canonical copy's CSR/CSC; full_edges bounds
// the input edges of the whole union (sizes the link arrays).
struct UnionSpec {
    int32_t K;
    const int32_t *node_inst;
    const int64_t *inst_noff;
    const int32_t *inst_canon;
    int32_t n_canon = 0;
    int64_t full_edges = 0;
};

// The captured sub-batch pipeline of one sweep configuration.
struct SweepGraphKey {
    const rmx::Level *lv;
    const rmx::ModState *M;
    const rmx::InstState *I;
    int allow_new, mark;
    double vthresh;
    int nsub;
    int64_t hub_gen;  // the hub arrays' allocation: graphs hold their addresses
    int tuning_gen;  // eval_tuning_generation() at capture: grid sizes are part of the graph
    bool operator==(const SweepGraphKey &o) const {
        return lv == o.lv && M == o.M && I == o.I && allow_new == o.allow_new && mark == o.mark &&
               vthresh == o.vthresh && nsub == o.nsub && hub_gen == o.hub_gen &&
               tuning_gen == o.tuning_gen;
    }
};
struct SweepGraph {
    SweepGraphKey key;
    cudaGraphExec_t exec;
    unsigned long long kernels;  // kernel nodes, counted as launches per replay
};

// A whole stage loop of sweeps (stage_sweeps) as one CUDA graph: a while
// node whose body is one sweep plus the stop rule evaluated on the device.
// Sizes are read on the device, so one graph serves every level held in the
// same buffers.
struct StageGraphKey {
    const rmx::Level *lv;
    const rmx::ModState *M;
    const rmx::InstState *I;
    int allow_new, prior, max_iter, nsub;
    double vthresh, threshold;
    int64_t hub_gen;  // the hub arrays' allocation: graphs hold their addresses
    int tuning_gen;
    size_t scratch_mark;  // the scratch the body's primitives use starts here
    bool operator==(const StageGraphKey &o) const {
        return lv == o.lv && M == o.M && I == o.I && allow_new == o.allow_new && prior == o.prior &&
               max_iter == o.max_iter && nsub == o.nsub && vthresh == o.vthresh && threshold == o.threshold &&
               hub_gen == o.hub_gen && tuning_gen == o.tuning_gen && scratch_mark == o.scratch_mark;
    }
};
struct StageGraph {
    StageGraphKey key;
    cudaGraphExec_t exec;
    unsigned long long kernels;  // kernel nodes of one sweep of the body
};

struct rmx_graph {
    // ---- host-side description
    int32_t N = 0;
    int64_t E = 0;       // kept links
    int64_t n_self = 0;  // dropped self-links with positive weight
    std::vector<std::string> names;
    std::vector<double> node_w;
    double tot_w = 0.0;

    // ---- device
    cudaStream_t stream = nullptr;
    rmx::Arena perm, scratch;
    int64_t *out_off = nullptr, *in_off = nullptr;
    int32_t *out_dst = nullptr, *in_src = nullptr;
    double *out_w0 = nullptr, *out_f = nullptr, *in_w = nullptr;
    rmx::fx_t *out_fx = nullptr, *in_fx = nullptr;
    double *tw = nullptr, *p = nullptr;
    uint8_t *dangling = nullptr;
    rmx::Stat4 *nattr = nullptr;
    int32_t *nmod = nullptr, *zeros = nullptr, *node_sn = nullptr, *submod = nullptr;
    int32_t *best_part = nullptr;  // the best attempt's partition while later attempts run
    rmx::fx_t *s0 = nullptr;
    int64_t *dtmp = nullptr;  // small device scratch (counters)

    rmx::Level node_lv, sub_lv;
    rmx::Level sn_buf[2];  // super-node levels: the current one and the next conversion's target
    int sn_cur = 0;
    rmx::Level &sn() { return sn_buf[sn_cur]; }
    rmx::ModState mods, submods;
    rmx::InstState inst1, instsub;
    rmx::SweepWork work;
    rmx::Timers timers;
    // Arrays grown on demand for the largest units / groups of a level: the
    // hub pipeline's buckets and plan arrays (work.hub_*) and the global hash
    // tables of the link aggregation. Both are arenas, so their blocks
    // come from and return to the process-wide block cache like the
    // handle's other device memory (no cudaMalloc / cudaFree of their own).
    rmx::Arena hub_arena, agg_arena;
    rmx::fx_t *agg_tab = nullptr;
    int64_t agg_cap = 0;

    // ---- instances: 1 for a single graph; a batch is a disjoint union of
    // graph-attempt copies, node ranges inst_noff[k]..inst_noff[k+1]
    int32_t K = 1;
    int32_t *node_inst = nullptr;       // device: instance of every node (zeros when K == 1)
    std::vector<int64_t> inst_noff;     // host, K + 1
    std::vector<int32_t> inst_canon;    // host: the copy whose flow instance k shares (itself if first)
    std::vector<double> L0v;            // initial code length per instance

    // ---- CUDA graphs of the sweep pipeline (off: every kernel launched directly)
#ifndef RMX_USE_GRAPHS
#define RMX_USE_GRAPHS 1
#endif
    bool use_graphs = RMX_USE_GRAPHS != 0;
    int64_t runs_done = 0;  // completed optimiser runs (attempts) on this handle
    std::vector<SweepGraph> sweep_graphs;
    std::vector<StageGraph> stage_graphs;
    // device state of a captured stage loop: [0] sweep number, [1] sub-batch
    // stamp, [2] attempt seed, [3] sweeps run, [4] instances still sweeping,
    // [5] units of the level
    int64_t *stage_ctl = nullptr;
    uint32_t *stage_seed = nullptr;      // the current sweep's seed
    uint8_t *stage_sweeping = nullptr;   // per instance: still sweeping
    double *stage_oldL = nullptr;        // per instance: code length before the current sweep

    // ---- state
    bool initiated = false;
    bool cols_normalised = false;  // in_w holds the normalised weights
    int power_iters = 0;
    int spmv_vec = 32;
    double L0 = 0.0;
    uint32_t stamp = 0;
    uint64_t sweep_no = 0;
    std::vector<double> step_bits;
    rmx_profile prof{};

    // current run settings
    rmx_opts opt{};
    uint32_t run_seed = 0;
    int nsub = 4;
    int superstep = 0;

    ~rmx_graph();
    void create(const int32_t *src, const int32_t *dst, const double *w, int64_t n_edges, int32_t n,
                const double *node_weights, const UnionSpec *u = nullptr);
    // One run over every instance of a union (seed for all); per-instance code lengths (nats).
    std::vector<double> run_union(const rmx_opts &o);
    void initiate();
    double codelength_fp64(const int32_t *part_host);
    void coarsen_hook(const int32_t *part, int32_t *n_sn, int64_t *n_links, int32_t *sn_of_mod, int64_t *o_off,
                      int32_t *o_dst, double *o_f, int64_t *i_off, int32_t *i_src, double *i_f);
    void evaluate_hook(const int32_t *part, const uint8_t *allow_new, int32_t *best_mod, double *best_delta);
    // The optimiser's own coarsening (convert_to_supernodes, aggregate_links)
    // on a given partition, optionally followed by a second conversion of the
    // super-nodes (part2: module of every first-level module id); outputs the
    // last level as the engine holds it (fixed-point flows, rows unordered).
    void coarsen_engine_hook(const int32_t *part, const int32_t *part2, int32_t *n_sn, int64_t *n_links,
                             int32_t *sn_of_mod, int64_t *o_off, int32_t *o_dst, rmx::fx_t *o_fx, int64_t *i_off,
                             int32_t *i_src, rmx::fx_t *i_fx, rmx::fx_t *sn_stat);
    // Move decisions of every super-node of the level built from part, with
    // the super-nodes assigned to modules sn_part[n_sn].
    void evaluate_sn_hook(const int32_t *part, int32_t n_sn, const int32_t *sn_part, const uint8_t *allow_new,
                          int32_t *best_mod, double *best_delta);
    double optimize(const rmx_opts &o, int32_t *part_out, int32_t *n_modules);
    // Code length of a fixed partition at teleportation probability tau, and
    // optionally its gradient (rmx_adjoint.cu).
    void adjoint(const int32_t *part, double tau, double *L, double *p, double *grad, double *dL_dtau,
                 int *solve_iters);

  private:
    void alloc_engine();
    void ensure_hub_table(const rmx::Level &lv);
    std::vector<double> run_attempt(uint32_t seed);
    void stage(bool fine, std::vector<double> &L, const std::vector<uint8_t> &run);
    void stage_sweeps(rmx::Level &lv, bool allow_new, std::vector<double> &L, const std::vector<uint8_t> &act);
    void sweep_single(rmx::Level &lv, bool prior, bool allow_new, double vthresh, int64_t &n_active,
                      std::vector<double> &L);
    bool stage_graph_ok(const rmx::Level &lv) const;
    void stage_sweeps_graph(rmx::Level &lv, bool allow_new, std::vector<double> &L, const std::vector<uint8_t> &act);
    void stage_body(rmx::Level &lv, bool allow_new, bool prior, double vthresh, int ns, unsigned long long cond);
    void subtune_body(int ns, unsigned long long cond);
    void loop_graph(const StageGraphKey &key, int64_t n_level, const std::function<void(unsigned long long)> &body);
    void set_active(const std::vector<uint8_t> &m);
    void run_subbatches(rmx::Level &lv, int64_t n_active, rmx::ModState &M, rmx::InstState &I,
                        const rmx::SweepArgs &sa, int ns, bool mark, uint32_t seed);
    int union_flows();
    void convert_to_supernodes(bool from_sn);
    void generate_sub_modules();
    void project_sn_to_nodes();
    int32_t count_modules();
    int sub_batches_for(int64_t n_active) const;
    int64_t max_degree(const rmx::Level &lv);
    void check_partition(const int32_t *part_host) const;
    int32_t supernodes_of(const int32_t *part_host);
};
