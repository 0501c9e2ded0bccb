/* Oracle: plain-C restatement of the reference RelaxMap algorithm for the hot
 * path. TEST INFRASTRUCTURE ONLY -- tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may call it as the checker; the product never
 * links it. Each function cites the reference file:line it restates.
 *
 * Conventions: nodes 0..N-1; out-links as CSR (off[N+1], dst[], value[]),
 * destinations ascending per row (the order the reference's sorted edge map
 * gives, OmpRelaxmap.cpp:118-134); in-links as CSC with sources ascending
 * (OmpRelaxmap.cpp:158-162). All flows FP64. tau = teleportation 0.15.
 *
 * Parity pin: every routine is checked against the reference compiled from its
 * own sources (oracle/_ref/librmxref.so, driven by ref_harness.cpp) in
 * tests/test_oracle_pin.py, and against golden vectors in tests/golden/.
 */
#ifndef RMX_ORACLE_H
#define RMX_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* MT19937 as bundled with the reference (MersenneTwister.h:54-347): one-word
 * seeding by the 69069 linear congruence (MersenneTwister.h:172-183), randInt(n)
 * by mask rejection (MersenneTwister.h:156-169). */
typedef struct {
    uint32_t state[624];
    int left;
    int next;
} rmxo_mt;
void rmxo_mt_seed(rmxo_mt *r, uint32_t seed);
uint32_t rmxo_mt_rand(rmxo_mt *r);
uint32_t rmxo_mt_randint(rmxo_mt *r, uint32_t n);

/* Network::initiate (Module.cpp:210-333) with calculateSteadyState
 * (Module.cpp:340-469) at one thread. Input w = positive edge weights (CSR),
 * tw = teleport weights. Outputs: p (node flow), f (edge flow, CSR order),
 * dsize (dangling size), exitpr (singleton exit, Module.cpp:67-99), dangling
 * flags; returns power iterations; *L0 = initial code length (nats, calibrate
 * Module.cpp:474-501), *all_log_all = sum plogp(p) (Module.cpp:295-307). */
int rmxo_initiate(int N, const int64_t *off, const int32_t *dst, const double *w, const double *tw, double *p,
                  double *f, double *dsize, double *exitpr, uint8_t *dangling, double *L0, double *all_log_all);

/* Network::calculateCodeLength (Module.cpp:2966-3002) for partition part[]
 * (module ids in [0,N)); module sums P/TW/D formed in node order. Returns L in
 * nats; *sum_exit = sum of module exits. */
double rmxo_codelength(int N, const int64_t *off, const int32_t *dst, const double *f, const double *p,
                       const double *tw, const double *dsize, const int32_t *part, double all_log_all,
                       double *sum_exit);

/* convertModulesToSuperNodes (Module.cpp:3008-3077): renumber non-empty modules
 * in ascending index order (part ids in [0,N)), aggregate inter-super-node
 * out-links summed in member-node / link order, sorted by destination; in-links
 * by ascending source. sn_of_mod[N] receives the renumbering (-1 if empty).
 * Returns the number of super-nodes; *n_links the number of SN out-links.
 * Output arrays must hold N (+1 for offsets) and E entries. */
int rmxo_convert(int N, const int64_t *off, const int32_t *dst, const double *f, const int32_t *part,
                 int32_t *sn_of_mod, int64_t *sn_out_off, int32_t *sn_out_dst, double *sn_out_f,
                 int64_t *sn_in_off, int32_t *sn_in_src, double *sn_in_f, int64_t *n_links);

/* Snapshot move evaluation for every unit (the decision phase of
 * Network::parallelMove, Module.cpp:1004-1123, identical in
 * prioritize_parallelMove :1366-1485 and the super-node variants
 * :2198-2313, :2555-2670). Units carry p, tw, dsize, exitpr and a module
 * mod[]; module stats (exit, P, TW, D) are indexed by module id; sum_exit is
 * the network's sumAllExitPr. Candidates are visited in ascending module id,
 * strict improvement keeps the first (lowest id) of equal gains; if
 * allow_new[u] the empty-module option (exit e_u, flows 0) is visited last.
 * best_mod[u] = chosen module, -2 for a new empty module, -1 if no candidate
 * beats 0; best_delta[u] = its code-length change (nats). */
void rmxo_evaluate(int nunits, const int64_t *out_off, const int32_t *out_dst, const double *out_f,
                   const int64_t *in_off, const int32_t *in_src, const double *in_f, const double *p,
                   const double *tw, const double *dsize, const double *exitpr, const int32_t *mod,
                   const double *mexit, const double *mP, const double *mTW, const double *mD, double sum_exit,
                   const uint8_t *allow_new, int32_t *best_mod, double *best_delta);

/* One-thread node sweeps of the reference: Network::move (Module.cpp:511-715)
 * when prior==0 or Network::prioritize_move (Module.cpp:727-950), repeated as in
 * stochastic_greedy_partition's first loop (OmpRelaxmap.cpp:291-339), starting
 * from singleton modules after initiate, with the bundled MT19937 seeded by
 * seed (OmpRelaxmap.cpp:55). vthresh is the CLI value (negated as at
 * OmpRelaxmap.cpp:66). Writes the module per node; returns the incremental code
 * length (nats); *n_sweeps = sweeps run. Needs the CSC too. */
double rmxo_node_sweeps(int N, const int64_t *off, const int32_t *dst, const double *f, const int64_t *in_off,
                        const int32_t *in_src, const double *in_f, const double *p, const double *tw,
                        const double *dsize, const double *exitpr, const uint8_t *dangling, double L0,
                        uint32_t seed, int prior, double vthresh, double threshold, int max_iter, int32_t *part,
                        int *n_sweeps);

#ifdef __cplusplus
}
#endif
#endif
