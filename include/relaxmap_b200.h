/*
 * relaxmap_b200: C ABI of the B200 map-equation optimiser (RelaxMap drop-in).
 *
 * The reference (uwescience/RelaxMap) is a monolithic OpenMP executable with no
 * plugin or FFI layer. Its internal driver API is class Network (Module.h:99-200)
 * called from OmpRelaxmap.cpp; each entry point below replaces one of those
 * calls, cited per function. Conventions:
 *   - Ownership: the caller owns every host array; inputs are copied in,
 *     outputs are written to caller-sized host buffers. The library owns all
 *     device memory through the opaque handle, freed by rmx_graph_destroy.
 *   - Errors: every call returns rmx_status; no C++ exception crosses the ABI.
 *     rmx_last_error() gives a thread-local message for the last failure.
 *   - Threading: a handle is bound to one CUDA stream and is not thread-safe;
 *     distinct handles may be used concurrently from different threads.
 *   - Node ids are int32 (0..N-1), link offsets int64, flows/weights FP64.
 *   - Code lengths are returned in nats unless the name says bits.
 * There is no CPU fallback: without a usable CUDA device, calls that compute
 * return RMX_ERR_CUDA.
 */
#ifndef RELAXMAP_B200_H
#define RELAXMAP_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    RMX_OK = 0,
    RMX_ERR_INVALID = 1,        /* bad argument (null pointer, id out of range, ...) */
    RMX_ERR_IO = 2,             /* file could not be opened / written */
    RMX_ERR_FORMAT = 3,         /* malformed Pajek header (the reference exits -1) */
    RMX_ERR_CUDA = 4,           /* CUDA runtime error or no device */
    RMX_ERR_OOM = 5,            /* device allocation failed */
    RMX_ERR_NO_CONVERGENCE = 6, /* iteration cap reached where convergence is required */
    RMX_ERR_TIMEOUT = 7,        /* a device-side watchdog budget ran out */
    RMX_ERR_STATE = 8           /* call out of order (e.g. no result yet) */
} rmx_status;

typedef struct rmx_graph rmx_graph;

/* Solver options: the reference CLI arguments (OmpRelaxmap.cpp:43-79) plus
 * engine knobs. */
typedef struct {
    uint32_t seed;        /* argv[1]: random seed (OmpRelaxmap.cpp:55) */
    int32_t threads;      /* argv[3]: host threads for parsing (device work ignores it) */
    int32_t attempts;     /* argv[4]: independent attempts, best code length kept */
    double threshold;     /* argv[5]: stop threshold in bits (OmpRelaxmap.cpp:62) */
    double vthresh;       /* argv[6]: per-move threshold, negated internally (:63-66) */
    int32_t max_iter;     /* argv[7]: sweeps per stage (OmpRelaxmap.cpp:49) */
    int32_t prior;        /* argv[9] == "prior": active-set sweeps (OmpRelaxmap.cpp:70-72) */
    int32_t sub_batches;  /* engine: relaxation sub-batches per sweep (0 = automatic) */
    int32_t verbose;      /* 1: print the reference's progress lines to stdout */
} rmx_opts;

/* Per-kernel-class device time recorded with CUDA events while profiling is on. */
typedef struct {
    int64_t launches;
    double ms;          /* summed event time */
    double bytes;       /* algorithmic bytes moved (compulsory traffic model): move evaluation,
                           per launch group, 16 B per link + 40 B per unit + 40 B per module
                           (at most one per candidate, at most the non-empty modules); the
                           adjoint solve, per sweep, 20 B per link + 65 B per node */
} rmx_kernel_stat;

enum {
    RMX_K_SPMV = 0,     /* power-iteration launch (one cooperative launch per solve) */
    RMX_K_EVAL,         /* move evaluation, all degree bins */
    RMX_K_COMMIT,       /* move commit + module statistic updates */
    RMX_K_COARSEN,      /* modules -> super-nodes (sort + segmented reduce) */
    RMX_K_CODELEN,      /* code length reductions */
    RMX_K_OTHER,
    RMX_K_ADJOINT,      /* transposed flow solve of rmx_adjoint_backward (one cooperative launch per call) */
    RMX_K_COUNT
};

typedef struct {
    rmx_kernel_stat k[RMX_K_COUNT];
    int64_t sweeps;          /* move sweeps run (node + super-node + coarse-tune) */
    int64_t supersteps;
    int64_t power_iters;
    double total_ms;         /* last rmx_optimize, device time on the handle's stream */
    int64_t kernel_launches; /* kernels this library launched (all handles) since it was loaded */
    int64_t links_evaluated; /* unit links read by move evaluation since profiling was enabled */
    int64_t units_evaluated; /* units evaluated since profiling was enabled */
    int64_t adjoint_iters;   /* sweeps of the transposed solve since profiling was enabled */
    double level_ms[3];      /* device time of the sweep loops on nodes, super-nodes, coarse-tune sub-problems */
    int64_t candidates_evaluated; /* (unit, candidate module) pairs evaluated since profiling was enabled */
    double eval_bin_ms[6];   /* move evaluation per degree bin (register, warp, mid, block, large, hub): summed
                                kernel time; the bins of one sub-batch run concurrently on separate streams */
    int64_t eval_bin_launches[6];
    int64_t eval_bin_links[6]; /* links read per degree bin since profiling was enabled */
    double eval_bin_bytes[6];  /* compulsory bytes per degree bin (links, units, module statistics) while profiling */
} rmx_profile;

const char *rmx_last_error(void);
const char *rmx_version(void);
void rmx_opts_default(rmx_opts *o);

/* Graph from an edge list held in host memory. Replaces the loaders' edge map
 * plus the edge preparation of main: duplicate (src,dst) pairs are summed in
 * input order (FileIO.cpp:157, :220), then self-loops and pairs whose summed
 * weight is <= 0 are dropped (OmpRelaxmap.cpp:117-135). w may be NULL (weight
 * 1); node_w may be NULL (uniform teleportation, FileIO.cpp:229), otherwise
 * the Pajek node weights (FileIO.cpp:114-120: values <= 0 already mapped to 1
 * by the caller). Builds CSR (out-links) and CSC (in-links) on the device. */
rmx_status rmx_graph_create(const int32_t *src, const int32_t *dst, const double *w, int64_t n_edges,
                            int32_t n_nodes, const double *node_w, rmx_graph **out);

/* Load a .net (Pajek) or any other extension (edge list) file with the
 * reference's parsing rules (FileIO.cpp:32-171, :177-265; format chosen by
 * extension as at OmpRelaxmap.cpp:60, :93-98) and build the device graph.
 * Node names are kept for rmx_write_outputs. */
rmx_status rmx_graph_load_file(const char *path, int32_t threads, rmx_graph **out);

/* Parse a file with the loader rules of rmx_graph_load_file on the host only
 * (no device work). Raw links in file order with duplicates kept (their sum is
 * formed by rmx_graph_create) and self-links removed (their count in
 * *n_self). Call with NULL buffers to get *n_nodes / *n_edges, then again with
 * src/dst/w of *n_edges entries and node_w of *n_nodes entries (node_w gets
 * the Pajek node weights, 1 for edge lists). The size query keeps its parse
 * for the next call on the same thread with the same path and thread count if
 * the file is unchanged (device, inode, size and modification time), so the
 * pair of calls parses once; any other call drops it. */
rmx_status rmx_parse_file(const char *path, int32_t threads, int32_t *n_nodes, int64_t *n_edges, int64_t *n_self,
                          int32_t *src, int32_t *dst, double *w, double *node_w);

rmx_status rmx_graph_destroy(rmx_graph *g);

/* N, kept links, and self-links that were dropped (OmpRelaxmap.cpp:117-142). */
rmx_status rmx_graph_info(const rmx_graph *g, int32_t *n_nodes, int64_t *n_links, int64_t *n_self_links);

/* Kept links as CSR (off[N+1], dst[E], w[E]: the summed input weights) and
 * the teleport weight per node (OmpRelaxmap.cpp:113-115). Any pointer may be NULL. */
rmx_status rmx_graph_links(const rmx_graph *g, int64_t *off, int32_t *dst, double *w, double *teleport);

/* Network::initiate (Module.cpp:210-333): dangling detection, row
 * normalisation, stationary flow by power iteration (calculateSteadyState,
 * Module.cpp:340-469: tau = 0.15, at most 200 iterations, stop when the L1
 * change is <= 1e-15 after at least 50), edge flows. Idempotent. Outputs may
 * be NULL: p[N] node flow, f[E] edge flow in CSR order, exit[N] singleton exit
 * (Module.cpp:67-99), dangling[N]; *iters = power iterations; *L0 = initial
 * code length in nats (calibrate, Module.cpp:474-501). */
rmx_status rmx_initiate(rmx_graph *g, double *p, double *f, double *exitpr, uint8_t *dangling, int32_t *iters,
                        double *L0);

/* Drop the handle's stationary flow and edge flows: the next rmx_initiate,
 * rmx_optimize or rmx_codelength recomputes them (OmpRelaxmap.cpp:113-155,
 * the part of the reference's timed region before the partitioning). */
rmx_status rmx_reset_flow(rmx_graph *g);

/* From-scratch code length of a partition (module id per node, any int32
 * labels in [0,N)), in nats: Network::calculateCodeLength (Module.cpp:2966-3002),
 * FP64 throughout. Runs rmx_initiate first if needed. */
rmx_status rmx_codelength(rmx_graph *g, const int32_t *part, double *L);

/* convertModulesToSuperNodes (Module.cpp:3008-3077) for partition part:
 * modules renumbered in ascending id order (sn_of_mod[N], -1 for unused ids),
 * inter-super-node links summed in member-node then link order (bit-identical
 * FP64 sums), CSR sorted by destination and CSC by source. Buffers are sized N
 * (+1 for offsets) and E by the caller. Outputs may be NULL individually. */
rmx_status rmx_coarsen(rmx_graph *g, const int32_t *part, int32_t *n_sn, int64_t *n_sn_links, int32_t *sn_of_mod,
                       int64_t *out_off, int32_t *out_dst, double *out_f, int64_t *in_off, int32_t *in_src,
                       double *in_f);

/* The move decision of every node against a fixed snapshot (the evaluation
 * phase of Network::parallelMove, Module.cpp:1004-1123): candidates are the
 * modules of out/in neighbours plus, where allow_new[u] != 0 (may be NULL),
 * an empty module; best_mod[u] is the module with the most negative change
 * (ties to the lowest id), -2 for a new module, -1 when none is negative;
 * best_delta[u] is that change in nats. Module statistics are formed from
 * part. The handle's partition state is overwritten (the next rmx_optimize
 * starts from singletons as always). */
rmx_status rmx_evaluate_moves(rmx_graph *g, const int32_t *part, const uint8_t *allow_new, int32_t *best_mod,
                              double *best_delta);

/* convertModulesToSuperNodes (Module.cpp:3008-3077) as the optimiser itself
 * performs it (rmx_coarsen above is a separate sort-based path): module
 * statistics from the nodes of part, super-nodes numbered by ascending module
 * id (sn_of_mod[N], -1 for unused ids), and the super-node links aggregated by
 * the engine's hash kernels into fixed-point flow sums. With part2 non-NULL a
 * second conversion follows, as after a super-node stage (the super-node loop
 * of OmpRelaxmap.cpp:379-411 calling convertModulesToSuperNodes again): every
 * first-level module m joins module part2[m] (part2 has N entries) and the
 * new super-nodes aggregate the first level's links; the outputs then
 * describe that second level, sn_of_mod indexed by part2's module ids.
 * Flows are fixed point, value * 2^62 rounded to nearest, each link sum
 * exact: out_fx/in_fx[E] per link, sn_stat[4 * n_sn] the super-node's
 * {flow, teleport weight, dangling flow, out-flow} (SuperNode(Module, int),
 * Node.cpp:76-106). Rows of the CSR and CSC come in no particular order.
 * Buffers are sized N (+1 for offsets) and E by the caller; outputs may be
 * NULL individually. The handle's partition state is overwritten. */
rmx_status rmx_coarsen_engine(rmx_graph *g, const int32_t *part, const int32_t *part2, int32_t *n_sn,
                              int64_t *n_sn_links, int32_t *sn_of_mod, int64_t *out_off, int32_t *out_dst,
                              int64_t *out_fx, int64_t *in_off, int32_t *in_src, int64_t *in_fx, int64_t *sn_stat);

/* The move decision of every super-node against a fixed snapshot (the
 * evaluation phase of Network::parallelMoveSuperNodes, Module.cpp:2198-2313,
 * and prioritize_parallelMoveSPnodes, :2555-2670): the super-node level of
 * part is built as rmx_coarsen_engine builds it, super-node s is placed in
 * module sn_part[s] (n_sn entries, ids in [0,N)), module statistics are
 * formed from the super-nodes, and every super-node is evaluated as
 * rmx_evaluate_moves evaluates nodes (allow_new[n_sn] may be NULL). n_sn must
 * equal the number of distinct modules of part. The handle's partition state
 * is overwritten. */
rmx_status rmx_evaluate_sn_moves(rmx_graph *g, const int32_t *part, int32_t n_sn, const int32_t *sn_part,
                                 const uint8_t *allow_new, int32_t *best_mod, double *best_delta);

/* The whole optimiser (OmpRelaxmap.cpp:155-233): initiate, superstep 1
 * (fine-tune), then alternating fine/coarse supersteps until a superstep gains
 * less than opts->threshold bits; attempts > 1 repeats with seeds seed+k and
 * keeps the lowest code length. part_out[N] (may be NULL) receives the module
 * index per node (the .clu labels minus one); *L_out the code length in nats;
 * *n_modules the number of non-empty modules. */
rmx_status rmx_optimize(rmx_graph *g, const rmx_opts *opts, int32_t *part_out, double *L_out, int32_t *n_modules);

/* Per-superstep code lengths (bits) of the last rmx_optimize; returns the count. */
int32_t rmx_superstep_codelengths(const rmx_graph *g, double *bits, int32_t cap);

/* Write <outdir>/<name>.tree and <outdir>/<name>.clu exactly as the reference
 * (print_twoLevel_Cluster OmpRelaxmap.cpp:790-812, .clu writer :240-249) for
 * the partition part and code length L (nats). name keeps its leading '/'. */
rmx_status rmx_write_outputs(rmx_graph *g, const int32_t *part, double L, const char *outdir, const char *name);

/* Read a .clu file as rmx_write_outputs writes it (a "*Vertices N" line, then
 * one label per node, module index + 1; CRLF or LF) into part_out[n_nodes]:
 * the partition a run saved, to resume from (rmx_codelength, the adjoint,
 * rmx_write_outputs). A vertex count other than n_nodes or a label that is
 * not an integer in 1..n_nodes is RMX_ERR_FORMAT, an unreadable file
 * RMX_ERR_IO. The reference writes .clu files but never reads them. */
rmx_status rmx_read_clu(const char *path, int32_t n_nodes, int32_t *part_out);

/* ---- Batched multi-graph x multi-attempt optimisation.
 * The reference optimises one network per run and its attempts one after
 * another (OmpRelaxmap.cpp:181-219); a batch optimises many graphs, each
 * `attempts` times, together. rmx_batch_create copies the graphs to host
 * memory: graph k has n_nodes[k] nodes and n_edges[k] edges, stored one graph
 * after another in src/dst (ids local to the graph, 0..n_nodes[k]-1) and w (may
 * be NULL: weight 1); node_w (may be NULL) the Pajek-style node weights, one
 * graph after another. Edge preparation per graph is rmx_graph_create's. */
typedef struct rmx_batch rmx_batch;
rmx_status rmx_batch_create(int32_t n_graphs, const int32_t *n_nodes, const int64_t *n_edges, const int32_t *src,
                            const int32_t *dst, const double *w, const double *node_w, rmx_batch **out);
/* Device budget of one wave: graph-attempt copies are packed into one
 * disjoint-union graph of at most max_links links and max_nodes nodes (a
 * single graph's attempts always form one wave). Defaults 2^27 and 2^25. */
rmx_status rmx_batch_set_wave(rmx_batch *b, int64_t max_links, int64_t max_nodes);
/* Runs every graph opts->attempts times (stop rules per graph-attempt as in
 * rmx_optimize, opts->seed for all; copies differ in their random choices) and
 * keeps each graph's lowest code length. Outputs (each may be NULL):
 * part_out[sum n_nodes] module per node, graph by graph, renumbered 0.. in
 * order of first appearance; L_out[n_graphs] nats; n_modules[n_graphs];
 * best_attempt[n_graphs] the attempt index kept. */
rmx_status rmx_batch_optimize(rmx_batch *b, const rmx_opts *opts, int32_t *part_out, double *L_out,
                              int32_t *n_modules, int32_t *best_attempt);
/* The last rmx_batch_optimize: waves, graph-attempt instances and the device
 * time of the optimiser runs (ms, CUDA events; host packing excluded). */
rmx_status rmx_batch_info(const rmx_batch *b, int32_t *n_graphs, int32_t *waves, int64_t *instances,
                          double *device_ms);
rmx_status rmx_batch_destroy(rmx_batch *b);

/* Code length of a FIXED partition as a function of the link weights and the
 * teleportation probability tau (fixed at 0.15 in the reference,
 * Module.cpp:340-469 and :2966-3002). The reference has no gradient: these two
 * calls are new API built on its forward model (row normalisation
 * Module.cpp:237-247, stationary flow with dangling mass redistributed by
 * teleport weight, module exit flows, calculateCodeLength).
 * rmx_adjoint_forward: *L (nats) at tau; p[N] (may be NULL) the stationary flow
 * at tau (power iteration with the reference's stop rule).
 * rmx_adjoint_backward: the same L (may be NULL), dL_dw[E] (may be NULL) the
 * derivative with respect to every kept link weight in the graph's CSR order
 * (the order of rmx_graph_links; input duplicates share their summed link's
 * value, dropped self-loops have none), *dL_dtau (may be NULL). The stationary
 * flow is recomputed, then one transposed solve (pull over the out-links)
 * gives the adjoint of the flow. part: module id per node in [0,N); tau in
 * (0,1). The solve stops when its L1 change is at most 1e-15 of the norm; if
 * 4000 sweeps do not get there (a small tau on a slowly mixing graph: the
 * error falls by about (1-tau)|lambda_2| per sweep) the call returns
 * RMX_ERR_NO_CONVERGENCE and writes neither dL_dw nor dL_dtau. */
rmx_status rmx_adjoint_forward(rmx_graph *g, const int32_t *part, double tau, double *L, double *p);
rmx_status rmx_adjoint_backward(rmx_graph *g, const int32_t *part, double tau, double *dL_dw, double *dL_dtau,
                                double *L);

/* Launch shape of move evaluation, process-wide: the grid cap of each degree
 * bin in blocks per SM, and the degree bounds (out + in links of a unit at
 * its level) that assign units to the bins: up to 8, 16 and 32 links the
 * register bins (fixed), then the warp bin up to warp_max_degree, the mid bin
 * up to mid_max_degree, the block bin up to block_max_degree, the large bin
 * up to large_max_degree, and the hub bin above; each hub unit's links are
 * partitioned by module into ceil(links / hub_partition_links) parts, each
 * aggregated by one block (so are the links of a super-node of more than
 * 16384 member links when the coarsening sums them). Results do not depend on
 * these values (every bin's kernel loops over its units by grid stride,
 * module statistics are exact integer sums, and every bin computes the same
 * change per candidate), only the time does. rmx_set_tuning takes effect at
 * the next launch; sweep pipelines captured as CUDA graphs under other values
 * are captured again. Each grid cap must lie in [1, 64], and
 * 32 <= warp_max <= 128, warp_max <= mid_max <= 512, mid_max <= block_max <=
 * 1024, block_max <= large_max <= 4096 (the bins' table limits; an equal
 * bound leaves a bin empty), and 64 <= hub_partition_links <= 2^30, else
 * RMX_ERR_INVALID. The Python module
 * relaxmap_b200.autotune picks the values by timing. No reference
 * counterpart. */
typedef struct rmx_tuning {
    int32_t eval_mid_grid;    /* mid bin (default 8) */
    int32_t eval_block_grid;  /* block bin (default 4) */
    int32_t eval_large_grid;  /* large bin (default 2) */
    int32_t eval_warp_grid;   /* warp bin (default 3) */
    int32_t eval_reg_grid;    /* register bins (default 8) */
    int32_t warp_max_degree;  /* default 128 */
    int32_t mid_max_degree;   /* default 512 */
    int32_t block_max_degree; /* default 1024 */
    int32_t large_max_degree; /* default 4096 */
    int32_t hub_partition_links; /* default 1024 */
} rmx_tuning;

rmx_status rmx_get_tuning(rmx_tuning *out);
rmx_status rmx_set_tuning(const rmx_tuning *t);

/* Device-time profiling of the handle's kernels (CUDA events on its stream). */
rmx_status rmx_set_profiling(rmx_graph *g, int32_t on);
rmx_status rmx_get_profile(const rmx_graph *g, rmx_profile *out);

/* The CUDA stream (cudaStream_t) all work of this handle is issued on. */
void *rmx_graph_stream(const rmx_graph *g);

/* Block until the handle's stream is idle. */
rmx_status rmx_sync(rmx_graph *g);

/* The device memory of a graph handle (and the scratch of an adjoint call)
 * is kept in a process-wide cache when the handle closes, up to half of each
 * device's memory: the next handle or call of similar size (a cached
 * block is reused for requests of at least half its size) takes it without a
 * cudaMalloc / cudaFree pair, and an allocation that fails empties the cache
 * and retries. This frees every cached block (all devices); handles still open
 * are untouched. No reference counterpart (the reference holds no device
 * memory). */
rmx_status rmx_release_device_cache(void);

/* Largest graph rmx_steady_state_noalloc accepts. */
#define RMX_NOALLOC_MAX_NODES (1 << 20)

/* The stationary flow of rmx_initiate for callers that cannot allocate device
 * memory: a framework whose memory pool owns the whole device under a fixed
 * budget, or a latency-bound path that must not pay for the device-wide
 * synchronisation an allocation implies. This entry point has no counterpart
 * in the reference (it computes calculateSteadyState only as part of
 * Network::initiate).
 * Every pointer is device memory owned by the caller: the in-links as CSC
 * (in_off[n_nodes+1], in_src[n_links], in_w[n_links] = row-normalised link
 * weights w_ab / sum_b w_ab), teleport[n_nodes], dangling[n_nodes] (1 for nodes
 * without out-links), p_out[n_nodes] (result); iters_out (device int, may be
 * NULL) receives the number of power iterations. n_nodes must not exceed
 * RMX_NOALLOC_MAX_NODES (larger graphs: RMX_ERR_INVALID). The work is queued
 * on `stream` (a cudaStream_t, NULL for the legacy default stream) and the call
 * returns without waiting for it.
 * It runs rmx_initiate's power iteration and stop rule, except that rows with
 * very many in-links (more than 64 steps of their lanes) are summed in one
 * pass instead of in chunks: on graphs with such in-degree hubs p agrees with
 * rmx_initiate's to rounding (1e-12 relative L1) and the iteration count can
 * differ by one; on other graphs both are identical.
 * Temporary storage is one array of about 8 MB inside this library, present on
 * every device that loads it until the process exits; it calls no cudaMalloc
 * or cudaFree. The first call on each device looks up that array's device
 * address (cudaGetSymbolAddress) with the device current and keeps it for the
 * life of the process: make that first call before any stream capture, and do
 * not call again after a cudaDeviceReset of that device. All calls on a device
 * share the array: calls whose work overlaps on the GPU (other streams, other
 * host threads) race and give wrong results; order them on one stream or with
 * events. Error text: rmx_noalloc_last_error(). */
rmx_status rmx_steady_state_noalloc(int32_t n_nodes, int64_t n_links, const int64_t *in_off, const int32_t *in_src,
                                    const double *in_w, const double *teleport, const uint8_t *dangling,
                                    double *p_out, int32_t *iters_out, void *stream);
const char *rmx_noalloc_last_error(void);

/* The reference command line (OmpRelaxmap.cpp:41-252), same positional
 * arguments and output files; returns the process exit code. */
int rmx_cli_main(int argc, char **argv);

#ifdef __cplusplus
}
#endif
#endif
