// Move sweeps: the relaxed parallel node / super-node moves of RelaxMap
// (Network::parallelMove Module.cpp:962-1307, prioritize_parallelMove
// :1317-1685, parallelMoveSuperNodes :2154-2497, prioritize_parallelMoveSPnodes
// :2506-2869) as bulk-synchronous GPU sub-batches.
//
// A sweep splits its active units into `nsub` pseudo-random sub-batches. Each
// sub-batch is evaluated against the module statistics left by the previous
// one (the reference evaluates against a snapshot that other threads keep
// changing), then committed at once:
//   evaluate  per unit, flow to/from every neighbouring module is aggregated
//             in a hash table (registers+shared memory for a warp, shared memory
//             for a block, global memory for hubs), the teleportation terms of
//             Module.cpp:1047-1061 are added and the code-length change of
//             Module.cpp:1088-1123 is evaluated for every candidate; the lowest
//             change wins, ties to the lowest module id.
//   commit    module P/TW/D and unit counts move with exact fixed-point atomics;
//             units proposing an empty module claim one deterministically.
//   delta     every link of a mover updates the out-flow OUT of the modules it
//             leaves / joins, exactly (old vs new membership of both ends).
// Module statistics are therefore always the exact fixed-point sums of the
// current partition, and the code length is recomputed from them per sweep.
#include <algorithm>
#include <climits>
#include <mutex>
#include <stdexcept>
#include <vector>

#include "rmx_engine.cuh"

// links each thread of a shared-table bin gathers ahead of its table inserts
#ifndef RMX_EVAL_ILP
#define RMX_EVAL_ILP 4
#endif
// the total-exit term of every candidate through log1p of a per-unit log (1) or a log each (0)
#ifndef RMX_LOG1P
#define RMX_LOG1P 1
#endif

namespace rmx {

constexpr unsigned kFull = 0xffffffffu;
constexpr int32_t kEmpty = -1;
constexpr int32_t kNewMod = -2;

// ---------------------------------------------------------------- helpers

__device__ __forceinline__ uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

__device__ __forceinline__ int tab_slot(int32_t key, int mask) { return (int)(mix32((uint32_t)key) & (uint32_t)mask); }

__device__ __forceinline__ bool better(double d1, int32_t m1, double d2, int32_t m2) {
    return d1 < d2 || (d1 == d2 && m1 < m2);
}

// Everything about the moving unit that every candidate needs. The terms of
// the code-length change that depend only on the unit and its old module
// (Module.cpp:1109-1112: sumAllExitPr, exit and stay of the old module before
// and after) are folded into K once per unit.
struct UnitCtx {
    double pu, tu, eu, cu;  // flow, teleport weight, exit, tau*p + (1-tau)*d
    double eA, nexA;        // old module exit before / after the unit leaves
    double sum_exit;
    double K;               // -plogp(se) - 2 (plogp(nexA) - plogp(eA)) + plogp(nexA + nPA) - plogp(eA + PA)
    double S0, logS0, rS0;  // the new total exit without the target's change, its log and reciprocal
    int32_t A;
};

// plogp of the new total exit flow S0 + dm, where dm = (new - old exit of the
// target module) is tiny next to S0 for almost every candidate: then
// log(S0 + dm) = log(S0) + log1p(dm / S0) with log(S0) computed once per unit
// and log1p by its Mercator series through t^6 (|t| < 2^-10: truncation below
// 2^-70 / 7 of the value, far under FP64 rounding); otherwise the direct log.
__device__ __forceinline__ double plogp_total(const UnitCtx &c, double dm) {
#if RMX_LOG1P
    const double t = dm * c.rS0;
    if (c.rS0 > 0.0 && fabs(t) < 0x1p-10) {
        const double l1p = t * (1.0 - t * (0.5 - t * (1.0 / 3.0 - t * (0.25 - t * (0.2 - t * (1.0 / 6.0))))));
        return (c.S0 + dm) * (c.logS0 + l1p);
    }
#endif
    return plogp(c.S0 + dm);
}

// Change of moving the unit into module with statistics st, given the unit's
// link flow to and from it (fixed point, out-links plus in-links, before the
// 1-tau factor): d_all - 2 d_exit + d_stay of Module.cpp:1109-1115 with the
// unit terms in K. The out- and in-flows (Module.cpp:1058, :1059) enter the
// change only through their sum (the new exit, :1104), so the tables keep one
// sum per module. t = the module's cached {plogp(exit), plogp(exit + P)}.
__device__ __forceinline__ double candidate_delta(const UnitCtx &c, const ModRec &r, fx_t sfx) {
    const Stat4 &st = r.s;
    const double2 t = r.t;
    const double P = from_fx(st.P), TW = from_fx(st.TW), D = from_fx(st.D), OUT = from_fx(st.OUT);
    const double em = exit_flow(P, TW, D, OUT);
    const double om_im = kBeta * from_fx(sfx) + c.cu * TW + (kAlpha * P + kBeta * D) * c.tu;  // :1058 + :1059
    const double nexm = em + c.eu - om_im;                                                    // Module.cpp:1104
    // new total exit sumAllExitPr + (nexA - eA) + (nexm - em), Module.cpp:1106
    return plogp_total(c, nexm - em) + c.K - 2.0 * (plogp(nexm) - t.x) + (plogp(nexm + P + c.pu) - t.y);
}

// The empty-module option: exit e_u, no shared flow (Module.cpp:1072-1077).
__device__ __forceinline__ double newmod_delta(const UnitCtx &c) {
    const double nexm = c.eu;
    return plogp_total(c, nexm) + c.K - 2.0 * plogp(nexm) + plogp(nexm + c.pu);
}

__device__ __forceinline__ UnitCtx make_ctx(const Stat4 &ua, const ModRec &mA, double sum_exit, int32_t A,
                                            fx_t sA) {
    const Stat4 &ma = mA.s;
    const double2 tA = mA.t;
    UnitCtx c;
    c.pu = from_fx(ua.P);
    c.tu = from_fx(ua.TW);
    const double du = from_fx(ua.D);
    c.eu = exit_flow(c.pu, c.tu, du, from_fx(ua.OUT));
    c.cu = kAlpha * c.pu + kBeta * du;
    const double PA = from_fx(ma.P), TWA = from_fx(ma.TW), DA = from_fx(ma.D);
    c.eA = exit_flow(PA, TWA, DA, from_fx(ma.OUT));
    // outFlow + inFlow to the old module (Module.cpp:1047, :1048), sA = their link flows' sum
    const double outA_inA = kBeta * from_fx(sA) + c.cu * (TWA - c.tu) +
                            (kAlpha * (PA - c.pu) + kBeta * (DA - du)) * c.tu;
    c.nexA = c.eA - c.eu + outA_inA;  // :1084
    c.sum_exit = sum_exit;
    c.K = -plogp(sum_exit) - 2.0 * (plogp(c.nexA) - tA.x) + (plogp(c.nexA + (PA - c.pu)) - tA.y);
    c.S0 = sum_exit + c.nexA - c.eA;
#if RMX_LOG1P
    const bool pos = c.S0 > 0.0;
    c.logS0 = pos ? log(c.S0) : 0.0;
    c.rS0 = pos ? 1.0 / c.S0 : 0.0;
#else
    c.logS0 = c.rS0 = 0.0;
#endif
    c.A = A;
    return c;
}

struct EvalArgs {
    // level
    const int64_t *out_off, *in_off;
    const int32_t *out_dst, *in_src;
    const fx_t *out_fx, *in_fx;
    const Stat4 *attr;
    const int32_t *mod, *uinst;
    // modules / instances
    const ModRec *mrec;     // per module: statistics and cached terms
    const int32_t *mcount;
    const double *inst_sum_exit;
    const uint8_t *inst_active;
    // work
    const int32_t *list;
    const int64_t *range;  // [beg, end) at range[0], range[1]
    int32_t *prop;
    double *pdelta;
    unsigned long long *stats;  // [0] links read [1] units evaluated [2] candidates evaluated
    double vthresh;
    int allow_new;             // stage-level switch
    const uint8_t *allow_new_unit;  // optional per-unit override (parity hook)
    int swap_guard;            // singleton min-label rule
    uint8_t *next_active;      // prioritised mode: neighbours of units that propose a move
    int mark;
};

// Decide and write the proposal for unit u given the argmin over candidates.
__device__ __forceinline__ int32_t finish_unit(const EvalArgs &a, int32_t u, const UnitCtx &c, double best,
                                               int32_t bm) {
    bool allow = a.allow_new_unit ? a.allow_new_unit[u] != 0 : (a.allow_new && a.mcount[c.A] > 1);
    if (allow) {
        double dn = newmod_delta(c);
        if (better(dn, INT_MAX, best, bm)) {
            best = dn;
            bm = kNewMod;
        }
    }
    int32_t out = -1;
    if (bm != INT_MAX && best < a.vthresh) {
        out = bm;
        // A singleton never moves into another singleton with a larger id: the
        // pair then merges in one direction instead of swapping.
        if (a.swap_guard && bm >= 0 && a.mcount[c.A] == 1 && a.mcount[bm] == 1 && bm > c.A) out = -1;
    }
    a.prop[u] = out;
    a.pdelta[u] = best;
    // a unit that found a move below the threshold activates its neighbours
    // for the next prioritised sweep, whether or not the move is then taken
    // (Module.cpp:1661-1668)
    return (bm != INT_MAX && best < a.vthresh) ? 1 : 0;
}

// Mark every out/in neighbour of u active (a group of NT threads, rank r).
template <int NT>
__device__ __forceinline__ void mark_neighbours(const EvalArgs &a, int32_t u, int r) {
    const int64_t ob = a.out_off[u], oe = a.out_off[u + 1], ib = a.in_off[u], ie = a.in_off[u + 1];
    for (int64_t e = ob + r; e < oe; e += NT) a.next_active[a.out_dst[e]] = 1;
    for (int64_t e = ib + r; e < ie; e += NT) a.next_active[a.in_src[e]] = 1;
}

// ---------------------------------------------------------------- evaluation
// Degree bins (out+in degree d of the unit at this level):
//   reg    d <= 32    8, 16 or 32 lanes per unit, one link per lane: the
//                     group sorts (module, flows) by module with a bitonic
//                     network and sums equal runs with a segmented scan, all
//                     in registers; each run's last lane is one candidate
//   warp   d <= 128   one warp per unit, table of <= 256 slots per warp in
//                     shared memory, candidates compacted in place
//   block  d <= 1024  256 threads per unit, table of <= 2048 slots in shared memory
//   large  d <= 4096  512 threads per unit, table of <= 8192 slots in shared memory
//   hub    d > 4096   512 threads per unit, table in a per-block slice of a
//                     global table (one block per SM)
// Each unit: clear the table, insert every link's neighbour module with its
// fixed-point flow (integer atomics, so the sums do not depend on the order),
// look up the own module, compact the other occupied slots in place into a
// dense candidate list, and evaluate the candidates with all lanes.

constexpr int kWarpMaxDeg = 128, kWarpCap = 256, kEvalWarps = 8;
// degree bins: 8 / 16 / 32 lanes in registers, warp (shared table), block
// (shared table), hub (global table)
constexpr int kBins = 8;
constexpr int kBinReg8 = 0, kBinReg16 = 1, kBinReg32 = 2, kBinWarp = 3, kBinMid = 4, kBinBlock = 5, kBinLarge = 6,
              kBinHub = 7;
// units of 129..512 links: four warps each (eight teams per SM), a 1024-slot table
#ifndef RMX_MID_CAP
#define RMX_MID_CAP 1024
#endif
constexpr int kMidT = 128, kMidCap = RMX_MID_CAP, kMidMaxDeg = kMidCap / 2, kMidDefault = 512;
constexpr int kBlkT = 256, kBlkMaxDeg = 1024, kBlkCap = 2048;
// resident blocks per SM of the block bin; default grid caps of the block, warp and register bins
#ifndef RMX_BLK_MINB
#define RMX_BLK_MINB 4
#endif
#ifndef RMX_BLK_GRID
#define RMX_BLK_GRID 4
#endif
#ifndef RMX_WARP_GRID
#define RMX_WARP_GRID 3
#endif
#ifndef RMX_REG_GRID
#define RMX_REG_GRID 8
#endif
// resident blocks per SM the register bin, warp bin and out-flow update are compiled for
#ifndef RMX_REG_MINB
#define RMX_REG_MINB 4
#endif
#ifndef RMX_WARP_MINB
#define RMX_WARP_MINB 3
#endif
#ifndef RMX_DELTA_MINB
#define RMX_DELTA_MINB 6
#endif
// the large bin's shared table (slots; units of up to half as many links) and
// its resident blocks per SM
#ifndef RMX_LRG_CAP
#define RMX_LRG_CAP 8192
#endif
#ifndef RMX_LRG_MINB
#define RMX_LRG_MINB 2
#endif
constexpr int kLrgT = 512, kLrgCap = RMX_LRG_CAP, kLrgMaxDeg = kLrgCap / 2;

// Slot of key, or -1 (linear probing); keys[s * KS] is slot s's key.
template <int KS = 1>
__device__ __forceinline__ int tab_find(const int32_t *keys, int mask, int32_t key) {
    int s = tab_slot(key, mask);
    for (int probe = 0; probe <= mask; probe++) {
        const int32_t k = keys[(int64_t)s * KS];
        if (k == key) return s;
        if (k == kEmpty) return -1;
        s = (s + 1) & mask;
    }
    return -1;
}

template <int NT>
__device__ __forceinline__ void gsync() {
    if (NT == 32)
        __syncwarp();
    else
        __syncthreads();
}

template <int NT>
struct GroupShared {  // reductions across the warps of a block group
    double best[NT / 32];
    int32_t mod[NT / 32];
    int ncand;
};

// Inserts the unit's links j = first, first + NT, ... below end (out-links
// first, then in-links; dout of them out) into the table keys/vals keyed by
// the neighbour's module, adding each link's fixed-point flow to the slot's
// sum. RMX_EVAL_ILP links at a time have their neighbour ids, flows and then
// neighbour modules loaded before any is inserted, so that many gathers are in
// flight per thread. Capacity >= 2 x the unit's links, so probing always
// finds a slot.
template <int NT>
__device__ __forceinline__ void insert_links(const EvalArgs &a, int64_t ob, int64_t ib, int64_t dout, int64_t first,
                                             int64_t d, int32_t *keys, fx_t *vals, int mask) {
    for (int64_t j0 = first; j0 < d; j0 += (int64_t)RMX_EVAL_ILP * NT) {
        int32_t key[RMX_EVAL_ILP];
        fx_t q[RMX_EVAL_ILP];
#pragma unroll
        for (int k = 0; k < RMX_EVAL_ILP; k++) {
            const int64_t j = j0 + (int64_t)k * NT;
            key[k] = -1;
            q[k] = 0;
            if (j < d) {
                const bool isout = j < dout;
                const int64_t e = isout ? ob + j : ib + (j - dout);
                // links are streamed (evict-first) so that the module ids they point to stay in L2
                key[k] = __ldcs(isout ? a.out_dst + e : a.in_src + e);
                q[k] = __ldcs(isout ? a.out_fx + e : a.in_fx + e);
            }
        }
#pragma unroll
        for (int k = 0; k < RMX_EVAL_ILP; k++)
            if (key[k] >= 0) key[k] = __ldg(a.mod + key[k]);
        // first probes of all keys issued together, then each key's collisions
        int slot[RMX_EVAL_ILP];
        int32_t prev[RMX_EVAL_ILP];
#pragma unroll
        for (int k = 0; k < RMX_EVAL_ILP; k++)
            if (key[k] >= 0) {
                slot[k] = tab_slot(key[k], mask);
                prev[k] = atomicCAS(keys + slot[k], kEmpty, key[k]);
            }
#pragma unroll
        for (int k = 0; k < RMX_EVAL_ILP; k++)
            if (key[k] >= 0) {
                // capacity >= 2 x the unit's links: a free slot exists, probing stays below mask steps
                for (int probe = 0; prev[k] != kEmpty && prev[k] != key[k] && probe < mask; probe++) {
                    slot[k] = (slot[k] + 1) & mask;
                    prev[k] = atomicCAS(keys + slot[k], kEmpty, key[k]);
                }
                atomic_add_fx(vals + slot[k], q[k]);
            }
    }
}

// One unit evaluated by a group of NT threads (a warp or a block); r = rank.
// The candidate list overwrites the table in place.
template <int NT>
__device__ __forceinline__ void eval_unit(const EvalArgs &a, const int32_t u, const int r, int32_t *keys, fx_t *vals,
                                          GroupShared<NT> *sh, unsigned long long &seen, unsigned long long &cands) {
    const int lane = r & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int64_t ob = a.out_off[u], ib = a.in_off[u];
    const int64_t dout = a.out_off[u + 1] - ob, d = dout + (a.in_off[u + 1] - ib);
    int64_t cap = 32;
    while (cap < 2 * d) cap <<= 1;
    const int mask = (int)(cap - 1);
    // The table is empty on entry: cleared once when the kernel starts (shared
    // tables) or when it is allocated (global slices), and every unit leaves
    // it empty again (below), so no clearing pass runs per unit.
    insert_links<NT>(a, ob, ib, dout, r, d, keys, vals, mask);
    gsync<NT>();
    const int32_t A = a.mod[u];
    const int sA = tab_find(keys, mask, A);
    const UnitCtx c = make_ctx(a.attr[u], a.mrec[A], a.inst_sum_exit[a.uinst[u]], A,
                               sA >= 0 ? vals[sA] : 0);
    if (NT > 32) __syncthreads();  // every lookup is done before slots are overwritten
    // Each warp compacts its own contiguous slice of the table in place (the
    // dense position never passes the slot being read) and evaluates it. A
    // slot left beyond the dense prefix is emptied at once; the prefix is
    // emptied as its candidates are evaluated.
    const int64_t seg = cap / (NT / 32), lo = (int64_t)(r >> 5) * seg, hi = lo + seg;
    int nc = 0;
    for (int64_t base = lo; base < hi; base += 32) {
        const int64_t s = base + lane;
        int32_t k = kEmpty;
        fx_t v = 0;
        if (s < hi) {
            k = keys[s];
            v = vals[s];
        }
        const bool occ = k != kEmpty && k != A;
        const unsigned bal = __ballot_sync(kFull, occ);
        __syncwarp();
        if (occ) {
            const int64_t p = lo + nc + __popc(bal & lt);
            keys[p] = k;
            vals[p] = v;
        }
        nc += __popc(bal);
        if (k != kEmpty && s >= lo + nc) {  // not overwritten by the dense prefix
            keys[s] = kEmpty;
            vals[s] = 0;
        }
    }
    __syncwarp();
    double best = 0.0;
    int32_t bm = INT_MAX;
    for (int q = lane; q < nc; q += 32) {
        const int32_t m = keys[lo + q];
        const fx_t v = vals[lo + q];
        keys[lo + q] = kEmpty;
        vals[lo + q] = 0;
        const double dl = candidate_delta(c, a.mrec[m], v);
        if (better(dl, m, best, bm)) {
            best = dl;
            bm = m;
        }
    }
    // lanes without a candidate hold (0, INT_MAX), which no real candidate loses to
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ob2 = __shfl_xor_sync(kFull, best, o);
        const int32_t om = __shfl_xor_sync(kFull, bm, o);
        if (better(ob2, om, best, bm)) {
            best = ob2;
            bm = om;
        }
    }
    if (NT > 32) {
        if (lane == 0) {
            sh->best[r >> 5] = best;
            sh->mod[r >> 5] = bm;
        }
        __syncthreads();
        if (r == 0)
            for (int q = 1; q < NT / 32; q++)
                if (better(sh->best[q], sh->mod[q], best, bm)) {
                    best = sh->best[q];
                    bm = sh->mod[q];
                }
    }
    int act = 0;
    if (lane == 0) cands += nc;
    if (r == 0) {
        act = finish_unit(a, u, c, best, bm);
        seen += d;
    }
    if (a.mark) {
        if (NT == 32) {
            act = __shfl_sync(kFull, act, 0);
        } else {
            if (r == 0) sh->ncand = act;
            __syncthreads();
            act = sh->ncand;
        }
        if (act) mark_neighbours<NT>(a, u, r);
    }
    gsync<NT>();
}

// Group of W lanes per unit (d <= W), everything in registers.
template <int W>
__device__ __forceinline__ void eval_unit_reg(const EvalArgs &a, const int32_t u, const bool valid, const int gl,
                                              const unsigned gmask, unsigned long long &seen,
                                              unsigned long long &cands) {
    int32_t key = INT_MAX, nbr = -1;
    fx_t v = 0;
    int64_t d = 0;
    int32_t A = -1;
    if (valid) {
        const int64_t ob = a.out_off[u], ib = a.in_off[u];
        const int64_t dout = a.out_off[u + 1] - ob;
        d = dout + (a.in_off[u + 1] - ib);
        A = a.mod[u];
        if (gl < d) {
            const bool isout = gl < dout;
            const int64_t e = isout ? ob + gl : ib + (gl - dout);
            nbr = __ldcs(isout ? a.out_dst + e : a.in_src + e);  // links streamed, module ids kept
            key = __ldg(a.mod + nbr);
            v = __ldcs(isout ? a.out_fx + e : a.in_fx + e);
        }
    }
    // bitonic sort of (key, flow) by key within the group
#pragma unroll
    for (int k = 2; k <= W; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const int32_t pk = __shfl_xor_sync(kFull, key, j, W);
            const fx_t pv = __shfl_xor_sync(kFull, v, j, W);
            const bool up = (gl & k) == 0, lower = (gl & j) == 0;
            const bool take = lower == up ? pk < key : pk > key;
            if (take) {
                key = pk;
                v = pv;
            }
        }
    }
    // sums over runs of equal keys (segmented inclusive scan)
#pragma unroll
    for (int off = 1; off < W; off <<= 1) {
        const int32_t k2 = __shfl_up_sync(kFull, key, off, W);
        const fx_t v2 = __shfl_up_sync(kFull, v, off, W);
        if (gl >= off && k2 == key) v += v2;
    }
    const int32_t nk = __shfl_down_sync(kFull, key, 1, W);
    const bool tail = key != INT_MAX && (gl == W - 1 || nk != key);
    // the flow to and from the unit's own module from the lane ending A's run
    const unsigned own = __ballot_sync(kFull, tail && key == A) & gmask;
    const int src = own ? __ffs(own) - 1 : (threadIdx.x & 31);
    fx_t sA = __shfl_sync(kFull, v, src);
    if (!own) sA = 0;
    double best = 0.0;
    int32_t bm = INT_MAX;
    UnitCtx c;
    if (valid) {
        c = make_ctx(a.attr[u], a.mrec[A], a.inst_sum_exit[a.uinst[u]], A, sA);
        if (tail && key != A) {
            best = candidate_delta(c, a.mrec[key], v);
            bm = key;
        }
    }
    const unsigned ncand = __popc(__ballot_sync(kFull, tail && key != A) & gmask);
#pragma unroll
    for (int o = W / 2; o > 0; o >>= 1) {
        const double ob2 = __shfl_xor_sync(kFull, best, o, W);
        const int32_t om = __shfl_xor_sync(kFull, bm, o, W);
        if (better(ob2, om, best, bm)) {
            best = ob2;
            bm = om;
        }
    }
    int act = 0;
    if (valid && gl == 0) {
        act = finish_unit(a, u, c, best, bm);
        seen += d;
        cands += ncand;
    }
    if (a.mark) {
        act = __shfl_sync(kFull, act, (threadIdx.x & 31) & ~(W - 1));
        if (act && nbr >= 0) a.next_active[nbr] = 1;
    }
}

// Bins reg8, reg16, reg32: ranges range[0..3) of consecutive buckets.
__global__ void __launch_bounds__(256, RMX_REG_MINB) k_eval_reg(EvalArgs a) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long seen = 0, units = 0, cands = 0;
#define RMX_REG_BIN(W, b)                                                                       \
    {                                                                                           \
        const int64_t beg = a.range[b], end = a.range[b + 1];                                   \
        const int g = lane / W, gl = lane % W;                                                  \
        const unsigned gmask = (W == 32 ? kFull : ((1u << W) - 1u)) << (g * W);                 \
        for (int64_t base = beg + gw * (32 / W); base < end; base += nw * (32 / W)) {           \
            const int64_t i = base + g;                                                         \
            bool valid = i < end;                                                               \
            const int32_t u = valid ? a.list[i] : 0;                                            \
            if (valid && !a.inst_active[a.uinst[u]]) {                                          \
                if (gl == 0) a.prop[u] = -1;                                                    \
                valid = false;                                                                  \
            }                                                                                   \
            eval_unit_reg<W>(a, u, valid, gl, gmask, seen, cands);                              \
            if (valid && gl == 0) units++;                                                      \
        }                                                                                       \
    }
    RMX_REG_BIN(8, 0)
    RMX_REG_BIN(16, 1)
    RMX_REG_BIN(32, 2)
#undef RMX_REG_BIN
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        seen += __shfl_xor_sync(kFull, seen, o);
        units += __shfl_xor_sync(kFull, units, o);
        cands += __shfl_xor_sync(kFull, cands, o);
    }
    if (lane == 0 && units) {
        atomicAdd(a.stats + 0, seen);
        atomicAdd(a.stats + 1, units);
        atomicAdd(a.stats + 2, cands);
    }
}

__device__ __forceinline__ void flush_stats(const EvalArgs &a, unsigned long long seen, unsigned long long units,
                                            unsigned long long cands) {
    if (units) {
        atomicAdd(a.stats + 0, seen);
        atomicAdd(a.stats + 1, units);
        atomicAdd(a.stats + 2, cands);
    }
}

__device__ __forceinline__ void flush_stats_split(const EvalArgs &a, unsigned long long seen, unsigned long long units,
                                                  unsigned long long cands) {
    if (seen) atomicAdd(a.stats + 0, seen);
    if (units) atomicAdd(a.stats + 1, units);
    if (cands) atomicAdd(a.stats + 2, cands);
}

__global__ void __launch_bounds__(kEvalWarps * 32, RMX_WARP_MINB) k_eval_warp(EvalArgs a) {
    __shared__ int32_t skey[kEvalWarps][kWarpCap];
    __shared__ fx_t sval[kEvalWarps][kWarpCap];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t beg = a.range[0], end = a.range[1];
    const int64_t gw = (int64_t)blockIdx.x * kEvalWarps + w, nw = (int64_t)gridDim.x * kEvalWarps;
    unsigned long long seen = 0, units = 0, cands = 0;
    for (int s = lane; s < kWarpCap; s += 32) {  // every unit leaves its table empty again
        skey[w][s] = kEmpty;
        sval[w][s] = 0;
    }
    __syncwarp();
    for (int64_t i = beg + gw; i < end; i += nw) {
        const int32_t u = a.list[i];
        if (!a.inst_active[a.uinst[u]]) {
            if (lane == 0) a.prop[u] = -1;
            continue;
        }
        eval_unit<32>(a, u, lane, skey[w], sval[w], nullptr, seen, cands);
        units++;
    }
    if (lane == 0) flush_stats(a, seen, units, cands);
}

// One unit per block of NT threads, its table of CAP slots in shared memory
// (the mid, block and large bins; the large bin's residency is RMX_LRG_MINB).
template <int NT, int CAP>
__global__ void __launch_bounds__(NT, NT >= 512 ? RMX_LRG_MINB : (NT == 128 ? 8 : RMX_BLK_MINB))
    k_eval_block(EvalArgs a) {
    extern __shared__ __align__(16) unsigned char dsm[];
    __shared__ GroupShared<NT> sh;
    fx_t *vals = reinterpret_cast<fx_t *>(dsm);
    int32_t *keys = reinterpret_cast<int32_t *>(vals + CAP);
    for (int s = threadIdx.x; s < CAP; s += NT) {  // every unit leaves its table empty again
        keys[s] = kEmpty;
        vals[s] = 0;
    }
    __syncthreads();
    const int64_t beg = a.range[0], end = a.range[1];
    unsigned long long seen = 0, units = 0, cands = 0;
    for (int64_t i = beg + blockIdx.x; i < end; i += gridDim.x) {
        const int32_t u = a.list[i];
        if (!a.inst_active[a.uinst[u]]) {
            if (threadIdx.x == 0) a.prop[u] = -1;
            continue;
        }
        eval_unit<NT>(a, u, threadIdx.x, keys, vals, &sh, seen, cands);
        units++;
    }
    // every warp found its own share of the candidates; thread 0 alone counted the links
    if ((threadIdx.x & 31) == 0) flush_stats_split(a, threadIdx.x == 0 ? seen : 0, threadIdx.x == 0 ? units : 0, cands);
}

// ---------------------------------------------------------------- hub units
// Units above the large bin's bound (R-MAT hubs and the heaviest super-nodes,
// 10^4 to 10^6 links) are not left to one block's long chain of dependent
// gathers and atomics. Every hub unit's links are radix-partitioned by a hash
// of their neighbour's module into partitions of about part_links links, so
// that each partition's distinct modules fit one block's shared table:
//   plan     one block lays out, by prefix sums, every hub unit's link chunks
//            (kHubCh links), partitions and bucket region;
//   count    blocks take link chunks: each link's partition is counted, and the
//            flow to and from the unit's own module is summed;
//   offsets  one block turns the partition counts into bucket offsets;
//   scatter  blocks take link chunks again and write (module, flow) into
//            their partition's bucket;
//   evaluate a block per partition aggregates its bucket in a shared table,
//            evaluates the candidates and keeps the partition's best change;
//   finish   a warp per unit reduces its partitions' bests and decides;
//   mark     in prioritised sweeps, link chunks of units that found a move
//            mark their neighbours.
// Counters are taken with one atomic per group of lanes that share a
// partition (__match_any_sync), not one per link.
constexpr int kHubCh = 2048;     // links per chunk item
constexpr int kHubPT = 256;      // threads per block of the pipeline
constexpr int kPartLinks = 1024; // mean links per partition (default of the run-time setting)
// shared table slots of a partition block (at most half filled per round) and
// its resident blocks per SM
#ifndef RMX_HUB_CAP
#define RMX_HUB_CAP 2048
#endif
#ifndef RMX_HUB_MINB
#define RMX_HUB_MINB 4
#endif
constexpr int kPartCap = RMX_HUB_CAP;
constexpr int kMaxParts = 1 << 20;
constexpr size_t kHubEvalSmem = (size_t)kPartCap * (sizeof(fx_t) + sizeof(int32_t));

struct HubPlan {
    int64_t *coff, *poff, *loff;   // per unit (+1): first chunk, first partition, first bucket element
    int32_t *nparts;               // per unit: partitions
    fx_t *own;                     // per unit: the link flow to and from the unit's own module
    uint8_t *act;                  // per unit: found a move below the threshold
    unsigned long long *pcnt;      // per partition: links (counted), then the fill position
    int64_t *pstart;               // per partition (+1): first bucket element
    double *best;                  // per partition: best change found
    int32_t *bmod;                 // per partition: its module
    int32_t *bkey;                 // bucket elements: module
    int32_t *lkey;                 // per link (at loff + link): the neighbour's module, from the count pass
    fx_t *bfx;                     //   and flow
    int32_t *cunit, *punit;        // unit (index in the sub-batch) of every chunk item and partition
    int64_t *tot;                  // [0] chunks, [1] partitions, [2] units, [3] over capacity, [4] links
    int64_t max_units, max_parts, max_links, max_chunks;  // capacities
    int64_t part_links;                       // mean links per partition
};

__device__ __forceinline__ uint32_t part_hash(int32_t key) { return mix32((uint32_t)key * 0x9E3779B1u + 0x7F4A7C15u); }

// Largest j < n with off[j] <= x (off ascending, off[0] <= x).
__device__ __forceinline__ int32_t hub_find(const int64_t *off, int32_t n, int64_t x) {
    int32_t lo = 0, hi = n - 1;
    while (lo < hi) {
        const int32_t mid = lo + ((hi - lo + 1) >> 1);
        if (off[mid] <= x)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Exclusive scan over the block (blockDim.x == 1024) of one value per thread.
__device__ __forceinline__ long long hub_block_scan(long long v, long long *ws, long long *total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    if (w == 0) {
        long long t = ws[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long y = __shfl_up_sync(kFull, t, o);
            if (lane >= o) t += y;
        }
        ws[lane] = t;
    }
    __syncthreads();
    const long long pre = (w > 0 ? ws[w - 1] : 0) + x - v;
    *total = ws[31];
    __syncthreads();
    return pre;
}

__device__ __forceinline__ int64_t unit_links(const EvalArgs &a, int32_t u) {
    return (a.out_off[u + 1] - a.out_off[u]) + (a.in_off[u + 1] - a.in_off[u]);
}

// The capacities are sized for every hub unit of the level, so they hold any
// sub-batch; should they not (the bin bounds changed since they were sized),
// nothing of the sub-batch is laid out and its hub units propose no move.
__global__ void __launch_bounds__(1024) k_hub_plan(EvalArgs a, HubPlan p) {
    __shared__ long long ws[32];
    const int64_t h0 = a.range[0], nu = a.range[1] - h0;
    if (nu > p.max_units) {
        if (threadIdx.x == 0) {
            p.tot[0] = p.tot[1] = p.tot[2] = p.tot[4] = 0;
            p.tot[3] = 1;
        }
        return;
    }
    long long r0 = 0, r1 = 0, r2 = 0;
    for (int64_t base = 0; base < nu; base += 1024) {
        const int64_t j = base + threadIdx.x;
        long long d = 0, nch = 0, np = 0;
        if (j < nu) {
            const int32_t u = a.list[h0 + j];
            if (a.inst_active[a.uinst[u]]) {  // inactive units take no chunk and no partition
                d = unit_links(a, u);
                nch = (d + kHubCh - 1) / kHubCh;
                np = min((long long)kMaxParts, max(1ll, (d + p.part_links - 1) / p.part_links));
            }
        }
        long long t0, t1, t2;
        const long long e0 = hub_block_scan(nch, ws, &t0);
        const long long e1 = hub_block_scan(np, ws, &t1);
        const long long e2 = hub_block_scan(d, ws, &t2);
        if (j < nu) {
            p.coff[j] = r0 + e0;
            p.poff[j] = r1 + e1;
            p.loff[j] = r2 + e2;
            p.nparts[j] = (int32_t)np;
            p.own[j] = 0;
        }
        r0 += t0;
        r1 += t1;
        r2 += t2;
    }
    __shared__ int over;
    if (threadIdx.x == 0) {
        over = r1 > p.max_parts || r2 > p.max_links || r0 > p.max_chunks;
        p.coff[nu] = r0;
        p.poff[nu] = r1;
        p.loff[nu] = r2;
        p.tot[0] = over ? 0 : r0;
        p.tot[1] = over ? 0 : r1;
        p.tot[2] = over ? 0 : nu;
        p.tot[3] = over;
        p.tot[4] = over ? 0 : r2;
    }
    __syncthreads();
    if (!over)
        for (int64_t q = threadIdx.x; q < r1; q += 1024) p.pcnt[q] = 0;
}

// Link l of unit u (out-links first): neighbour module and flow.
__device__ __forceinline__ void hub_link(const EvalArgs &a, int64_t ob, int64_t ib, int64_t dout, int64_t l,
                                         int32_t &key, fx_t &q) {
    const bool in = l >= dout;
    const int64_t e = in ? ib + (l - dout) : ob + l;
    key = __ldg(a.mod + __ldcs(in ? a.in_src + e : a.out_dst + e));  // links streamed, module ids kept
    q = __ldcs(in ? a.in_fx + e : a.out_fx + e);
}

// Count (scatter = false) or place (scatter = true) the links of the chunks.
// Links to the unit's own module are only summed (into own); the others are
// combined per warp step by module with __match_any_sync, so a
// module that many of a hub's links reach takes one bucket element per warp
// step instead of one per link (integer sums: exact in any order). Both
// passes form the same groups (the same lanes read the same links), so the
// counts hold the scatter exactly. The count pass stores each link's module,
// which the scatter pass reads back in order instead of gathering it again.
template <bool SCATTER>
__global__ void __launch_bounds__(kHubPT) k_hub_links(EvalArgs a, HubPlan p) {
    constexpr int ILP = 4;  // links gathered per thread before any is combined
    __shared__ fx_t wq[kHubPT];
    const int lane = threadIdx.x & 31;
    const int64_t h0 = a.range[0], total = p.tot[0];
    const int32_t nu = (int32_t)p.tot[2];
    for (int64_t item = blockIdx.x; item < total; item += gridDim.x) {
        // the count pass finds each chunk's unit and lists it (and the unit's
        // partitions, from its first chunk) for the later kernels
        const int32_t j = SCATTER ? p.cunit[item] : hub_find(p.coff, nu, item);
        const int32_t u = a.list[h0 + j];
        const int32_t A = a.mod[u], np = p.nparts[j];
        const int64_t ob = a.out_off[u], ib = a.in_off[u];
        const int64_t dout = a.out_off[u + 1] - ob, d = dout + (a.in_off[u + 1] - ib);
        const int64_t c0 = (item - p.coff[j]) * kHubCh, c1 = min(d, c0 + kHubCh);
        int32_t *const lk = p.lkey + p.loff[j];  // the unit's links' modules
        if (!SCATTER) {
            if (threadIdx.x == 0) p.cunit[item] = j;
            if (c0 == 0)
                for (int q = threadIdx.x; q < np; q += kHubPT) p.punit[p.poff[j] + q] = j;
        }
        fx_t sA = 0;
        for (int64_t b0 = c0; b0 < c1; b0 += kHubPT * ILP) {  // uniform over the block
            int32_t keys[ILP];
            fx_t qs[ILP];
#pragma unroll
            for (int k = 0; k < ILP; k++) {
                const int64_t l = b0 + k * kHubPT + threadIdx.x;
                keys[k] = A;  // lanes past the chunk: flow 0 to the own module
                qs[k] = 0;
                if (l < c1) {
                    if (!SCATTER) {
                        hub_link(a, ob, ib, dout, l, keys[k], qs[k]);
                        lk[l] = keys[k];
                    } else {  // the module the count pass found: no second gather
                        const bool in = l >= dout;
                        keys[k] = __ldcs(lk + l);
                        qs[k] = __ldcs(in ? a.in_fx + ib + (l - dout) : a.out_fx + ob + l);
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < ILP; k++) {
                const int32_t key = keys[k];
                const fx_t q = qs[k];
                if (key == A) sA += q;
                const bool valid = key != A;
                const unsigned kpeers = __match_any_sync(kFull, valid ? key : -1);
                const bool head = valid && lane == __ffs(kpeers) - 1;  // one lane per module
                const int32_t part = head ? (int32_t)(part_hash(key) % (uint32_t)np) : -1;
                const unsigned peers = __match_any_sync(kFull, part);
                const int leader = __ffs(peers) - 1;
                if (!SCATTER) {
                    if (head && lane == leader)
                        atomicAdd(p.pcnt + p.poff[j] + part, (unsigned long long)__popc(peers));
                } else {
                    wq[threadIdx.x] = q;
                    __syncwarp();
                    fx_t sum = 0;
                    if (head)
                        for (unsigned m = kpeers; m; m &= m - 1) sum += wq[(threadIdx.x & ~31) + __ffs(m) - 1];
                    unsigned long long base = 0;
                    const int64_t pidx = p.poff[j] + part;
                    if (head && lane == leader) base = atomicAdd(p.pcnt + pidx, (unsigned long long)__popc(peers));
                    base = __shfl_sync(kFull, base, leader);
                    if (head) {
                        const int64_t pos = p.pstart[pidx] + (int64_t)base + __popc(peers & ((1u << lane) - 1u));
                        p.bkey[pos] = key;
                        p.bfx[pos] = sum;
                    }
                    __syncwarp();
                }
            }
        }
        if (!SCATTER) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) sA += __shfl_xor_sync(kFull, sA, o);
            if (lane == 0 && sA) atomic_add_fx(p.own + j, sA);
        }
    }
}

// Partition counts -> bucket offsets (each unit's buckets inside its region,
// in partition order); the counters restart at zero as fill positions.
__global__ void __launch_bounds__(1024) k_hub_offsets(HubPlan p) {
    __shared__ long long ws[32];
    const int64_t np = p.tot[1];
    long long r = 0;
    for (int64_t base = 0; base < np; base += 1024) {
        const int64_t q = base + threadIdx.x;
        const long long c = q < np ? (long long)p.pcnt[q] : 0;
        long long t;
        const long long e = hub_block_scan(c, ws, &t);
        if (q < np) {
            p.pstart[q] = r + e;
            p.pcnt[q] = 0;
        }
        r += t;
    }
    if (threadIdx.x == 0) p.pstart[np] = r;
}

// A block per partition: its bucket aggregated in a shared table, in R rounds
// if it holds more distinct modules than half the table (which the
// partitioning makes rare): round r takes the keys whose second hash h2 (a
// bijection of the key) has h2 mod R == r, and R doubles until no round
// overfills (at R = 2^31 a round holds at most two keys).
__global__ void __launch_bounds__(kHubPT, RMX_HUB_MINB) k_hub_eval(EvalArgs a, HubPlan p) {
    extern __shared__ __align__(16) unsigned char hub_smem[];  // kHubEvalSmem bytes
    fx_t *vals = reinterpret_cast<fx_t *>(hub_smem);
    int32_t *keys = reinterpret_cast<int32_t *>(vals + kPartCap);
    __shared__ double sb[kHubPT / 32];
    __shared__ int32_t sm[kHubPT / 32];
    __shared__ int16_t taken[kPartCap / 2 + kHubPT];  // slots taken in this round, in the order taken
    __shared__ int nfresh;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t h0 = a.range[0], total = p.tot[1];
    const int32_t nu = (int32_t)p.tot[2];
    const int mask = kPartCap - 1;
    unsigned long long cands = 0;
    for (int s = threadIdx.x; s < kPartCap; s += kHubPT) {
        keys[s] = kEmpty;
        vals[s] = 0;
    }
    for (int64_t pidx = blockIdx.x; pidx < total; pidx += gridDim.x) {
        const int32_t j = p.punit[pidx];
        const int32_t u = a.list[h0 + j];
        const int64_t b0 = p.pstart[pidx], b1 = p.pstart[pidx + 1];
        const int32_t A = a.mod[u];
        const UnitCtx c = make_ctx(a.attr[u], a.mrec[A], a.inst_sum_exit[a.uinst[u]], A, p.own[j]);
        double best = 0.0;
        int32_t bm = INT_MAX;
        for (uint32_t R = 1;; R <<= 1) {  // R rounds; more only when a round overfills the table
            bool overfull = false;
            double rbest = 0.0;
            int32_t rbm = INT_MAX;
            unsigned long long rc = 0;
            for (uint32_t r = 0; r < R && !overfull; r++) {
                __syncthreads();
                if (threadIdx.x == 0) nfresh = 0;
                __syncthreads();
                for (int64_t e = b0 + threadIdx.x; e < b1; e += kHubPT) {
                    const int32_t key = p.bkey[e];
                    if (R > 1 && (mix32((uint32_t)key ^ 0x5bd1e995u) & (R - 1)) != r) continue;
                    if (*(volatile int *)&nfresh > kPartCap / 2) break;
                    int sl = tab_slot(key, mask);
                    int32_t prev = atomicCAS(keys + sl, kEmpty, key);
                    for (int probe = 0; prev != kEmpty && prev != key && probe < mask; probe++) {
                        sl = (sl + 1) & mask;
                        prev = atomicCAS(keys + sl, kEmpty, key);
                    }
                    if (prev != kEmpty && prev != key) continue;  // unreachable: the table is never full
                    if (prev == kEmpty) taken[atomicAdd(&nfresh, 1)] = (int16_t)sl;
                    atomic_add_fx(vals + sl, p.bfx[e]);
                }
                __syncthreads();
                // at most kPartCap / 2 + kHubPT slots were taken (every thread checks the
                // count before it inserts), so the table never fills and the list holds them all
                const int nt = nfresh;
                overfull = nt > kPartCap / 2;
                // evaluate the taken slots' candidates (unless the round overfilled) and empty them
                for (int i = threadIdx.x; i < nt; i += kHubPT) {
                    const int s = taken[i];
                    const int32_t k = keys[s];
                    if (!overfull && k != A) {
                        rc++;
                        const double dl = candidate_delta(c, a.mrec[k], vals[s]);
                        if (better(dl, k, rbest, rbm)) {
                            rbest = dl;
                            rbm = k;
                        }
                    }
                    keys[s] = kEmpty;
                    vals[s] = 0;
                }
            }
            __syncthreads();
            if (!overfull) {
                best = rbest;
                bm = rbm;
                cands += rc;
                break;
            }  // else retry with twice the rounds (the table is empty again)
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ob2 = __shfl_xor_sync(kFull, best, o);
            const int32_t om = __shfl_xor_sync(kFull, bm, o);
            if (better(ob2, om, best, bm)) {
                best = ob2;
                bm = om;
            }
        }
        if (lane == 0) {
            sb[w] = best;
            sm[w] = bm;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int q = 1; q < kHubPT / 32; q++)
                if (better(sb[q], sm[q], best, bm)) {
                    best = sb[q];
                    bm = sm[q];
                }
            p.best[pidx] = best;
            p.bmod[pidx] = bm;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cands += __shfl_xor_sync(kFull, cands, o);
    if (lane == 0 && cands) atomicAdd(a.stats + 2, cands);
}

__global__ void k_hub_finish(EvalArgs a, HubPlan p) {
    const int lane = threadIdx.x & 31;
    const int64_t h0 = a.range[0], nu = p.tot[2];
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long seen = 0, units = 0;
    if (p.tot[3]) {  // not laid out (over capacity): no proposals
        for (int64_t i = h0 + gw * 32 + lane; i < a.range[1]; i += nw * 32) a.prop[a.list[i]] = -1;
        return;
    }
    for (int64_t j = gw; j < nu; j += nw) {
        const int32_t u = a.list[h0 + j];
        if (p.nparts[j] == 0) {  // its instance has stopped
            if (lane == 0) {
                a.prop[u] = -1;
                p.act[j] = 0;
            }
            continue;
        }
        double best = 0.0;
        int32_t bm = INT_MAX;
        for (int64_t q = p.poff[j] + lane; q < p.poff[j + 1]; q += 32)
            if (better(p.best[q], p.bmod[q], best, bm)) {
                best = p.best[q];
                bm = p.bmod[q];
            }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ob2 = __shfl_xor_sync(kFull, best, o);
            const int32_t om = __shfl_xor_sync(kFull, bm, o);
            if (better(ob2, om, best, bm)) {
                best = ob2;
                bm = om;
            }
        }
        if (lane == 0) {
            const int32_t A = a.mod[u];
            const UnitCtx c = make_ctx(a.attr[u], a.mrec[A], a.inst_sum_exit[a.uinst[u]], A,
                                       p.own[j]);
            p.act[j] = (uint8_t)finish_unit(a, u, c, best, bm);
            seen += unit_links(a, u);
            units++;
        }
    }
    if (lane == 0) flush_stats_split(a, seen, units, 0);
}

__global__ void __launch_bounds__(kHubPT) k_hub_mark(EvalArgs a, HubPlan p) {
    const int64_t h0 = a.range[0], total = p.tot[0];
    const int32_t nu = (int32_t)p.tot[2];
    for (int64_t item = blockIdx.x; item < total; item += gridDim.x) {
        const int32_t j = p.cunit[item];
        if (!p.act[j]) continue;
        const int32_t u = a.list[h0 + j];
        const int64_t ob = a.out_off[u], ib = a.in_off[u];
        const int64_t dout = a.out_off[u + 1] - ob, d = dout + (a.in_off[u + 1] - ib);
        const int64_t c0 = (item - p.coff[j]) * kHubCh, c1 = min(d, c0 + kHubCh);
        for (int64_t l = c0 + threadIdx.x; l < c1; l += kHubPT)
            a.next_active[l < dout ? a.out_dst[ob + l] : a.in_src[ib + (l - dout)]] = 1;
    }
}

// ---------------------------------------------------------------- commit

struct CommitArgs {
    const int32_t *list;
    const int64_t *range;
    const int32_t *prop;
    int32_t *ptarget;
    int32_t *mod, *prevmod;
    uint32_t *stamp_of;
    const Stat4 *attr;
    const int32_t *uinst, *nnodes;
    Stat4 *mstat;
    int32_t *mcount, *minst;
    unsigned long long *claim;
    const int32_t *free_list;
    const int64_t *n_free;
    unsigned long long *moved_nodes;
    // device {stamp, hseed} of the sub-batch: stamp marks its movers, hseed (a
    // function of attempt seed, sweep and sub-batch) picks the free id a unit bids for
    const uint32_t *sp;
};

__device__ __forceinline__ unsigned long long claim_key(uint32_t stamp, int32_t u) {
    return ((unsigned long long)stamp << 32) | (0xffffffffu - (uint32_t)u);
}

// Units proposing an empty module bid for a free id chosen by hash; the
// smallest unit id wins each id (atomicMax on an inverted key), losers stay.
__global__ void k_claim(CommitArgs a) {
    const uint32_t stamp = a.sp[0], hseed = a.sp[1];
    const int64_t beg = a.range[0], end = a.range[1];
    const int64_t nf = *a.n_free;
    for (int64_t i = beg + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < end;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t u = a.list[i];
        if (a.prop[u] != kNewMod) continue;
        int32_t m = -1;
        if (nf > 0) {
            int64_t s = mix32((uint32_t)u ^ hseed) % nf;
            for (int probe = 0; probe < 8; probe++, s = (s + 1) % nf) {
                const int32_t cand = a.free_list[s];
                if (a.mcount[cand] == 0) {
                    m = cand;
                    break;
                }
            }
        }
        a.ptarget[u] = m;
        if (m >= 0) atomicMax(a.claim + m, claim_key(stamp, u));
    }
}

__global__ void k_commit(CommitArgs a) {
    const uint32_t stamp = a.sp[0];
    const int64_t beg = a.range[0], end = a.range[1];
    unsigned long long moved = 0;
    for (int64_t i = beg + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < end;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t u = a.list[i];
        int32_t t = a.prop[u];
        if (t == -1) continue;
        if (t == kNewMod) {
            t = a.ptarget[u];
            if (t < 0 || a.claim[t] != claim_key(stamp, u)) continue;
            a.minst[t] = a.uinst[u];
        }
        const int32_t A = a.mod[u];
        a.prevmod[u] = A;
        a.mod[u] = t;
        a.stamp_of[u] = stamp;
        const Stat4 s = a.attr[u];
        atomic_add_fx(&a.mstat[t].P, s.P);
        atomic_add_fx(&a.mstat[t].TW, s.TW);
        atomic_add_fx(&a.mstat[t].D, s.D);
        atomic_add_fx(&a.mstat[A].P, -s.P);
        atomic_add_fx(&a.mstat[A].TW, -s.TW);
        atomic_add_fx(&a.mstat[A].D, -s.D);
        atomicAdd(a.mcount + t, 1);
        atomicSub(a.mcount + A, 1);
        moved += a.nnodes ? a.nnodes[u] : 1;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) moved += __shfl_xor_sync(kFull, moved, o);
    if ((threadIdx.x & 31) == 0 && moved) atomicAdd(a.moved_nodes, moved);
}

struct DeltaArgs {
    const int32_t *list;
    const int64_t *beg, *end;  // the units at list[*beg .. *end)
    const int32_t *mod, *prevmod;
    const uint32_t *stamp_of;
    const int64_t *out_off, *in_off;
    const int32_t *out_dst, *in_src;
    const fx_t *out_fx, *in_fx;
    Stat4 *mstat;
    const uint32_t *sp;  // device {stamp, hseed} of the sub-batch
};

// Out-flow bookkeeping for the movers of this sub-batch; warp per unit.
// Link u->w adds its flow to OUT[mod(u)] iff mod(u) != mod(w). When u moves
// A -> T only OUT[A] and OUT[T] change: out-links leave A's count if they
// crossed and join T's if they now cross; in-links from A become crossing
// (OUT[A] grows) and in-links from T stop crossing (OUT[T] shrinks). Links whose
// two ends both moved are handled once, by the source's out-link loop. The
// warp sums its lanes' changes, so each mover costs two atomics.
// Changes of OUT[A] and OUT[T] from the links of mover u, summed by the
// calling thread over links j = first, first + stride, ...
__device__ __forceinline__ void delta_links(const DeltaArgs &a, uint32_t stamp, int32_t u, int32_t A, int32_t T,
                                            int first, int stride, fx_t &dA, fx_t &dT) {
    for (int64_t e = a.out_off[u] + first; e < a.out_off[u + 1]; e += stride) {
        const int32_t w = a.out_dst[e];
        const fx_t q = a.out_fx[e];
        const bool wm = a.stamp_of[w] == stamp;
        const int32_t bn = a.mod[w], bo = wm ? a.prevmod[w] : bn;
        if (A != bo) dA -= q;
        if (T != bn) dT += q;
    }
    for (int64_t e = a.in_off[u] + first; e < a.in_off[u + 1]; e += stride) {
        const int32_t w = a.in_src[e];
        if (a.stamp_of[w] != stamp) {
            const int32_t b = a.mod[w];
            if (b == A)
                dA += a.in_fx[e];
            else if (b == T)
                dT -= a.in_fx[e];
        }
    }
}

__global__ void __launch_bounds__(256, RMX_DELTA_MINB) k_delta(DeltaArgs a) {
    const int lane = threadIdx.x & 31;
    const uint32_t stamp = a.sp[0];
    const int64_t beg = *a.beg, end = *a.end;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = beg + gw; i < end; i += nw) {
        const int32_t u = a.list[i];
        if (a.stamp_of[u] != stamp) continue;  // did not move in this sub-batch
        const int32_t A = a.prevmod[u], T = a.mod[u];
        fx_t dA = 0, dT = 0;
        delta_links(a, stamp, u, A, T, lane, 32, dA, dT);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            dA += __shfl_xor_sync(kFull, dA, o);
            dT += __shfl_xor_sync(kFull, dT, o);
        }
        if (lane == 0) {
            if (dA) atomic_add_fx(&a.mstat[A].OUT, dA);
            if (dT) atomic_add_fx(&a.mstat[T].OUT, dT);
        }
    }
}

// Movers of more than 128 links: a block each, so that one heavy super-node
// does not leave a single warp walking thousands of links.
__global__ void __launch_bounds__(256) k_delta_block(DeltaArgs a) {
    __shared__ fx_t sh[2][8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t stamp = a.sp[0];
    const int64_t beg = *a.beg, end = *a.end;
    for (int64_t i = beg + blockIdx.x; i < end; i += gridDim.x) {
        const int32_t u = a.list[i];
        if (a.stamp_of[u] != stamp) continue;  // uniform across the block
        const int32_t A = a.prevmod[u], T = a.mod[u];
        fx_t dA = 0, dT = 0;
        delta_links(a, stamp, u, A, T, threadIdx.x, 256, dA, dT);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            dA += __shfl_xor_sync(kFull, dA, o);
            dT += __shfl_xor_sync(kFull, dT, o);
        }
        if (lane == 0) {
            sh[0][w] = dA;
            sh[1][w] = dT;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            fx_t tA = 0, tT = 0;
            for (int k = 0; k < 8; k++) {
                tA += sh[0][k];
                tT += sh[1][k];
            }
            if (tA) atomic_add_fx(&a.mstat[A].OUT, tA);
            if (tT) atomic_add_fx(&a.mstat[T].OUT, tT);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- stats

__device__ __forceinline__ double2 module_terms(const Stat4 &st) {
    const double P = from_fx(st.P);
    const double e = exit_flow(P, from_fx(st.TW), from_fx(st.D), from_fx(st.OUT));
    return make_double2(plogp(e), plogp(e + P));
}

// A module's cached terms and its evaluation record.
__device__ __forceinline__ void write_terms(const Stat4 *mstat, double2 *term, ModRec *rec, int32_t m) {
    const Stat4 st = mstat[m];
    const double2 t = module_terms(st);
    term[m] = t;
    rec[m].s = st;
    rec[m].t = t;
}

__global__ void k_terms_all(int32_t cap, const Stat4 *mstat, double2 *term, ModRec *rec) {
    for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < cap; m += (int64_t)gridDim.x * blockDim.x)
        write_terms(mstat, term, rec, (int32_t)m);
}

void refresh_terms(ModState &M, cudaStream_t s) {
    k_terms_all<<<blocks_for(M.cap, 256, num_sms() * 32), 256, 0, s>>>(M.cap, M.stat, M.term, M.rec);
    RMX_LAUNCHED();
}

// After a sub-batch: the two modules of every mover get fresh cached terms
// (a module touched by several movers is written with the same value).
__global__ void k_terms_movers(const int32_t *list, const int64_t *range, const uint32_t *stamp_of, const uint32_t *sp,
                               const int32_t *mod, const int32_t *prevmod, const Stat4 *mstat, double2 *term,
                               ModRec *rec) {
    const uint32_t stamp = sp[0];
    const int64_t beg = range[0], end = range[1];
    for (int64_t i = beg + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < end;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t u = list[i];
        if (stamp_of[u] != stamp) continue;
        const int32_t A = prevmod[u], T = mod[u];
        write_terms(mstat, term, rec, A);
        write_terms(mstat, term, rec, T);
    }
}

__global__ void k_init_singletons(int32_t n, const Stat4 *attr, const int32_t *uinst, int32_t *mod, Stat4 *mstat,
                                  int32_t *mcount, int32_t *minst) {
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n; u += (int64_t)gridDim.x * blockDim.x) {
        mod[u] = (int32_t)u;
        mstat[u] = attr[u];
        mcount[u] = 1;
        minst[u] = uinst[u];
    }
}

void init_singletons(const Level &L, ModState &M, cudaStream_t s) {
    if (L.n > M.cap) throw std::invalid_argument("module capacity below unit count");
    if (M.cap > L.n) {
        RMX_CUDA(cudaMemsetAsync(M.stat + L.n, 0, sizeof(Stat4) * (M.cap - L.n), s));
        RMX_CUDA(cudaMemsetAsync(M.count + L.n, 0, sizeof(int32_t) * (M.cap - L.n), s));
    }
    k_init_singletons<<<blocks_for(L.n, 256, num_sms() * 32), 256, 0, s>>>(L.n, L.attr, L.inst, L.mod, M.stat, M.count,
                                                                           M.inst);
    RMX_LAUNCHED();
    refresh_terms(M, s);
}

__global__ void k_stats_nodes(int32_t n, const Stat4 *attr, const int32_t *mod, const int32_t *uinst, Stat4 *mstat,
                              int32_t *mcount, int32_t *minst) {
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n; u += (int64_t)gridDim.x * blockDim.x) {
        const int32_t m = mod[u];
        const Stat4 s = attr[u];
        atomic_add_fx(&mstat[m].P, s.P);
        atomic_add_fx(&mstat[m].TW, s.TW);
        atomic_add_fx(&mstat[m].D, s.D);
        atomicAdd(mcount + m, 1);
        minst[m] = uinst[u];
    }
}

__global__ void k_stats_links(int32_t n, const int64_t *off, const int32_t *dst, const fx_t *fx, const int32_t *mod,
                              Stat4 *mstat) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t u = gw; u < n; u += nw) {
        const int32_t m = mod[u];
        fx_t o = 0;
        for (int64_t e = off[u] + lane; e < off[u + 1]; e += 32)
            if (mod[dst[e]] != m) o += fx[e];
#pragma unroll
        for (int q = 16; q > 0; q >>= 1) o += __shfl_xor_sync(kFull, o, q);
        if (lane == 0 && o) atomic_add_fx(&mstat[m].OUT, o);
    }
}

void module_stats_from_units(const Level &L, ModState &M, cudaStream_t s) {
    RMX_CUDA(cudaMemsetAsync(M.stat, 0, sizeof(Stat4) * M.cap, s));
    RMX_CUDA(cudaMemsetAsync(M.count, 0, sizeof(int32_t) * M.cap, s));
    k_stats_nodes<<<blocks_for(L.n, 256, num_sms() * 32), 256, 0, s>>>(L.n, L.attr, L.mod, L.inst, M.stat, M.count,
                                                                       M.inst);
    RMX_LAUNCHED();
    k_stats_links<<<blocks_for((int64_t)L.n * 32, 256, num_sms() * 32), 256, 0, s>>>(L.n, L.out_off, L.out_dst,
                                                                                     L.out_fx, L.mod, M.stat);
    RMX_LAUNCHED();
    refresh_terms(M, s);
}

__global__ void k_count_units(int32_t n, const int32_t *mod, int32_t *mcount) {
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n; u += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(mcount + mod[u], 1);
}

void count_units(const Level &L, ModState &M, cudaStream_t s) {
    RMX_CUDA(cudaMemsetAsync(M.count, 0, sizeof(int32_t) * M.cap, s));
    k_count_units<<<blocks_for(L.n, 256, num_sms() * 32), 256, 0, s>>>(L.n, L.mod, M.count);
    RMX_LAUNCHED();
}

// Sum of module terms per instance in fixed point (deterministic).
template <bool SINGLE>
__global__ void __launch_bounds__(256) k_mod_terms(int32_t cap, const Stat4 *mstat, const double2 *mterm,
                                                   const int32_t *mcount, const int32_t *minst, fx_t *acc) {
    __shared__ fx_t sh[3][8];
    fx_t t0 = 0, t1 = 0, t2 = 0;
    for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < cap; m += (int64_t)gridDim.x * blockDim.x) {
        if (mcount[m] <= 0) continue;
        const Stat4 st = mstat[m];
        const double P = from_fx(st.P);
        const double e = exit_flow(P, from_fx(st.TW), from_fx(st.D), from_fx(st.OUT));
        const double2 t = mterm[m];
        const fx_t a0 = to_fxl(e), a1 = to_fxl(t.x), a2 = to_fxl(t.y);
        if (SINGLE) {
            t0 += a0;
            t1 += a1;
            t2 += a2;
        } else {
            fx_t *p = acc + 3 * (int64_t)minst[m];
            atomic_add_fx(p, a0);
            atomic_add_fx(p + 1, a1);
            atomic_add_fx(p + 2, a2);
        }
    }
    if (SINGLE) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            t0 += __shfl_xor_sync(kFull, t0, o);
            t1 += __shfl_xor_sync(kFull, t1, o);
            t2 += __shfl_xor_sync(kFull, t2, o);
        }
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        if (lane == 0) {
            sh[0][w] = t0;
            sh[1][w] = t1;
            sh[2][w] = t2;
        }
        __syncthreads();
        if (threadIdx.x < 3) {
            fx_t v = 0;
            for (int q = 0; q < 8; q++) v += sh[threadIdx.x][q];
            if (v) atomic_add_fx(acc + threadIdx.x, v);
        }
    }
}

__global__ void k_inst_L(int32_t ninst, const fx_t *acc, const fx_t *s0, double *sum_exit, double *L) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < ninst; k += (int64_t)gridDim.x * blockDim.x) {
        const double se = from_fxl(acc[3 * k]);
        sum_exit[k] = se;
        L[k] = plogp(se) - 2.0 * from_fxl(acc[3 * k + 1]) + from_fxl(acc[3 * k + 2]) - from_fxl(s0[k]);  // :2999
    }
}

void instance_codelength(const ModState &M, InstState &I, cudaStream_t s) {
    RMX_CUDA(cudaMemsetAsync(I.acc, 0, sizeof(fx_t) * 3 * I.n, s));
    if (I.n == 1)
        k_mod_terms<true><<<blocks_for(M.cap, 256, num_sms() * 8), 256, 0, s>>>(M.cap, M.stat, M.term, M.count, M.inst,
                                                                                I.acc);
    else
        k_mod_terms<false><<<blocks_for(M.cap, 256, num_sms() * 8), 256, 0, s>>>(M.cap, M.stat, M.term, M.count,
                                                                                 M.inst, I.acc);
    RMX_LAUNCHED();
    k_inst_L<<<blocks_for(I.n, 256, 4096), 256, 0, s>>>(I.n, I.acc, I.s0, I.sum_exit, I.L);
    RMX_LAUNCHED();
}

// ---------------------------------------------------------------- sweep driver

static EvalArgs eval_args(const Level &L, const ModState &M, const InstState &I, SweepWork &W, double vthresh,
                          int allow_new, const uint8_t *allow_unit, int swap_guard) {
    EvalArgs a;
    a.out_off = L.out_off;
    a.in_off = L.in_off;
    a.out_dst = L.out_dst;
    a.in_src = L.in_src;
    a.out_fx = L.out_fx;
    a.in_fx = L.in_fx;
    a.attr = L.attr;
    a.mod = L.mod;
    a.uinst = L.inst;
    a.mrec = M.rec;
    a.mcount = M.count;
    a.inst_sum_exit = I.sum_exit;
    a.inst_active = I.active;
    a.list = W.list2;
    a.range = nullptr;
    a.prop = W.prop;
    a.pdelta = W.pdelta;
    a.stats = reinterpret_cast<unsigned long long *>(W.counters + kCntBins);  // the register bins' (the first)
    a.vthresh = vthresh;
    a.allow_new = allow_new;
    a.allow_new_unit = allow_unit;
    a.swap_guard = swap_guard;
    a.next_active = W.next_active;
    a.mark = 0;
    return a;
}

__global__ void k_hub_level(int32_t n, const int64_t *out_off, const int64_t *in_off, int64_t bound, int64_t part_links,
                            unsigned long long *acc) {
    unsigned long long c0 = 0, c1 = 0, c2 = 0, c3 = 0;
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n; u += (int64_t)gridDim.x * blockDim.x) {
        const int64_t d = (out_off[u + 1] - out_off[u]) + (in_off[u + 1] - in_off[u]);
        if (d <= bound) continue;
        c0++;
        c1 += min((int64_t)kMaxParts, (d + part_links - 1) / part_links);
        c2 += d;
        c3 += (d + kHubCh - 1) / kHubCh;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        c0 += __shfl_xor_sync(kFull, c0, o);
        c1 += __shfl_xor_sync(kFull, c1, o);
        c2 += __shfl_xor_sync(kFull, c2, o);
        c3 += __shfl_xor_sync(kFull, c3, o);
    }
    if ((threadIdx.x & 31) == 0 && c0) {
        atomicAdd(acc, c0);
        atomicAdd(acc + 1, c1);
        atomicAdd(acc + 2, c2);
        atomicAdd(acc + 3, c3);
    }
}

void hub_level_needs(const Level &L, int64_t *out, int64_t *dev_tmp, cudaStream_t s) {
    unsigned long long *acc = reinterpret_cast<unsigned long long *>(dev_tmp);
    RMX_CUDA(cudaMemsetAsync(acc, 0, 4 * sizeof(unsigned long long), s));
    const EvalTuning t = eval_tuning();
    k_hub_level<<<blocks_for(L.n, 256, num_sms() * 8), 256, 0, s>>>(L.n, L.out_off, L.in_off, t.large_max, t.hub_part,
                                                                    acc);
    RMX_LAUNCHED();
    RMX_CUDA(cudaMemcpyAsync(out, acc, 4 * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RMX_CUDA(cudaStreamSynchronize(s));
}

namespace {
EvalTuning g_tuning{8,           RMX_BLK_GRID, RMX_LRG_MINB, RMX_WARP_GRID, RMX_REG_GRID,
                    kWarpMaxDeg, kMidDefault,  kBlkMaxDeg,   kLrgMaxDeg,    kPartLinks};
int g_tuning_gen = 0;
std::mutex g_tuning_mu;  // guards g_tuning and g_tuning_gen
}  // namespace

EvalTuning eval_tuning() {
    std::lock_guard<std::mutex> lk(g_tuning_mu);
    return g_tuning;
}

void set_eval_tuning(const EvalTuning &t) {
    for (int v : {t.mid, t.block, t.large, t.warp, t.reg})
        if (v < 1 || v > 64) throw std::invalid_argument("evaluation grid caps must lie in 1..64 blocks per SM");
    // each bin's bound lies between the previous bin's and its own table's limit
    if (t.warp_max < 32 || t.warp_max > kWarpMaxDeg || t.mid_max < t.warp_max || t.mid_max > kMidMaxDeg ||
        t.block_max < t.mid_max || t.block_max > kBlkMaxDeg || t.large_max < t.block_max || t.large_max > kLrgMaxDeg)
        throw std::invalid_argument("degree bin bounds must satisfy 32 <= warp <= 128, warp <= mid <= 512, "
                                    "mid <= block <= 1024, block <= large <= 4096");
    if (t.hub_part < 64 || t.hub_part > (1 << 30))
        throw std::invalid_argument("hub partitions must hold 64..2^30 links");
    std::lock_guard<std::mutex> lk(g_tuning_mu);
    g_tuning = t;
    g_tuning_gen++;
}

int eval_tuning_generation() {
    std::lock_guard<std::mutex> lk(g_tuning_mu);
    return g_tuning_gen;
}
int64_t block_bin_max_degree() { return eval_tuning().large_max; }

constexpr size_t kBlkSmem = (size_t)kBlkCap * (sizeof(fx_t) + sizeof(int32_t));
constexpr size_t kMidSmem = (size_t)kMidCap * (sizeof(fx_t) + sizeof(int32_t));
constexpr size_t kLrgSmem = (size_t)kLrgCap * (sizeof(fx_t) + sizeof(int32_t));

// Blocks for `items` work items at per_block items a block, at most max_grid.
static unsigned fit_grid(int64_t items, int64_t per_block, int64_t max_grid) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(max_grid, (items + per_block - 1) / per_block));
}

// The bins of a sub-batch run concurrently: mid, block, large + hub, and warp
// bins on four auxiliary streams forked from and joined back into s, the
// register bins on s itself. Only non-empty bins are launched (sizes from the
// host copy of the bucket offsets); a lone bin runs on s without the fork.
static void launch_eval(EvalArgs a, const int64_t *bucket_off, int first_bucket, const SweepWork &W, bool fitted,
                        cudaStream_t s, Timers *tm = nullptr) {
    const int64_t *h = fitted ? W.bucket_host.data() + first_bucket : nullptr;
    // without host sizes every bin counts as non-empty and takes its full grid
    auto cnt = [&](int b0, int b1) { return fitted ? h[b1] - h[b0] : (int64_t)1 << 40; };
    const int64_t n_mid = cnt(kBinMid, kBinMid + 1), n_blk = cnt(kBinBlock, kBinBlock + 1),
                  n_lrg = cnt(kBinLarge, kBinLarge + 1), n_hub = W.hub_links > 0 ? cnt(kBinHub, kBinHub + 1) : 0,
                  n_warp = cnt(kBinWarp, kBinWarp + 1), n_reg = cnt(kBinReg8, kBinReg32 + 1);
    // streams: 0 block, 1 large, 2 warp, 3 mid, 4 hub, the caller's stream the register bins
    const bool use[5] = {n_blk > 0, n_lrg > 0, n_warp > 0, n_mid > 0, n_hub > 0};
    const EvalTuning tg = eval_tuning();
    int streams = n_reg > 0 ? 1 : 0;
    for (bool b : use) streams += b ? 1 : 0;
    const bool fork = streams > 1;
    auto on = [&](int k) { return fork ? W.aux[k] : s; };
    unsigned long long *const stats0 = a.stats;  // each bin counts into its own three slots
    auto bin_stats = [&](int timer) { return stats0 + 3 * (timer - kTimerBinReg); };
    if (fork) {
        RMX_CUDA(cudaEventRecord(W.fork, s));
        for (int k = 0; k < 5; k++)
            if (use[k]) RMX_CUDA(cudaStreamWaitEvent(W.aux[k], W.fork, 0));
    }
    if (n_hub > 0) {  // every hub unit split over many blocks (see k_hub_plan); first: the longest chain
        a.range = bucket_off + first_bucket + kBinHub;
        a.stats = bin_stats(kTimerBinHub);
        HubPlan hp;
        hp.coff = W.hub_coff;
        hp.poff = W.hub_poff;
        hp.loff = W.hub_loff;
        hp.nparts = W.hub_nparts;
        hp.own = W.hub_own;
        hp.act = W.hub_act;
        hp.pcnt = W.hub_pcnt;
        hp.pstart = W.hub_pstart;
        hp.best = W.hub_best;
        hp.bmod = W.hub_bmod;
        hp.bkey = W.hub_bkey;
        hp.lkey = W.hub_lkey;
        hp.bfx = W.hub_bfx;
        hp.tot = W.hub_tot;
        hp.max_units = W.hub_units;
        hp.max_parts = W.hub_parts;
        hp.max_links = W.hub_links;
        hp.max_chunks = W.hub_chunks;
        hp.cunit = W.hub_cunit;
        hp.punit = W.hub_punit;
        hp.part_links = tg.hub_part;
        const cudaStream_t hs = on(4);
        const unsigned G = num_sms() * 8, GE = num_sms() * RMX_HUB_MINB;
        if (tm) tm->begin(kTimerBinHub, hs);
        k_hub_plan<<<1, 1024, 0, hs>>>(a, hp);
        RMX_LAUNCHED();
        k_hub_links<false><<<G, kHubPT, 0, hs>>>(a, hp);
        RMX_LAUNCHED();
        k_hub_offsets<<<1, 1024, 0, hs>>>(hp);
        RMX_LAUNCHED();
        k_hub_links<true><<<G, kHubPT, 0, hs>>>(a, hp);
        RMX_LAUNCHED();
        k_hub_eval<<<GE, kHubPT, kHubEvalSmem, hs>>>(a, hp);
        RMX_LAUNCHED();
        k_hub_finish<<<blocks_for(W.hub_units * 32, 256, num_sms() * 16), 256, 0, hs>>>(a, hp);
        RMX_LAUNCHED();
        if (a.mark) {
            k_hub_mark<<<G, kHubPT, 0, hs>>>(a, hp);
            RMX_LAUNCHED();
        }
        if (tm) tm->end(kTimerBinHub, hs);
    }
    if (n_mid > 0) {
        a.range = bucket_off + first_bucket + kBinMid;
        a.stats = bin_stats(kTimerBinMid);
        if (tm) tm->begin(kTimerBinMid, on(3));
        k_eval_block<kMidT, kMidCap><<<fit_grid(n_mid, 1, (int64_t)num_sms() * tg.mid), kMidT, kMidSmem, on(3)>>>(a);
        RMX_LAUNCHED();
        if (tm) tm->end(kTimerBinMid, on(3));
    }
    if (n_blk > 0) {
        a.range = bucket_off + first_bucket + kBinBlock;
        a.stats = bin_stats(kTimerBinBlock);
        if (tm) tm->begin(kTimerBinBlock, on(0));
        k_eval_block<kBlkT, kBlkCap><<<fit_grid(n_blk, 1, (int64_t)num_sms() * tg.block), kBlkT, kBlkSmem, on(0)>>>(
            a);
        RMX_LAUNCHED();
        if (tm) tm->end(kTimerBinBlock, on(0));
    }
    if (n_lrg > 0) {
        a.range = bucket_off + first_bucket + kBinLarge;
        a.stats = bin_stats(kTimerBinLarge);
        if (tm) tm->begin(kTimerBinLarge, on(1));
        k_eval_block<kLrgT, kLrgCap><<<fit_grid(n_lrg, 1, (int64_t)num_sms() * tg.large), kLrgT, kLrgSmem, on(1)>>>(a);
        RMX_LAUNCHED();
        if (tm) tm->end(kTimerBinLarge, on(1));
    }
    if (n_warp > 0) {
        a.range = bucket_off + first_bucket + kBinWarp;
        a.stats = bin_stats(kTimerBinWarp);
        if (tm) tm->begin(kTimerBinWarp, on(2));
        k_eval_warp<<<fit_grid(n_warp, kEvalWarps, (int64_t)num_sms() * tg.warp), kEvalWarps * 32, 0, on(2)>>>(a);
        RMX_LAUNCHED();
        if (tm) tm->end(kTimerBinWarp, on(2));
    }
    if (n_reg > 0) {
        a.range = bucket_off + first_bucket + kBinReg8;
        a.stats = bin_stats(kTimerBinReg);
        if (tm) tm->begin(kTimerBinReg, s);
        k_eval_reg<<<fit_grid(n_reg, 8, (int64_t)num_sms() * tg.reg), 256, 0, s>>>(a);
        RMX_LAUNCHED();
        if (tm) tm->end(kTimerBinReg, s);
    }
    if (fork)
        for (int k = 0; k < 5; k++)
            if (use[k]) {
                RMX_CUDA(cudaEventRecord(W.join[k], W.aux[k]));
                RMX_CUDA(cudaStreamWaitEvent(s, W.join[k], 0));
            }
}

// Dynamic shared memory and carve-out of the evaluation bins, set once per device.
void configure_eval_kernels() {
    static std::mutex mu;
    static std::vector<bool> configured;
    int dev = 0;
    RMX_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    if ((int)configured.size() <= dev) configured.resize(dev + 1, false);
    if (configured[dev]) return;
    RMX_CUDA(cudaFuncSetAttribute(k_eval_block<kBlkT, kBlkCap>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kBlkSmem));
    RMX_CUDA(cudaFuncSetAttribute(k_eval_block<kLrgT, kLrgCap>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kLrgSmem));
    RMX_CUDA(cudaFuncSetAttribute(k_eval_block<kBlkT, kBlkCap>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  100));
    RMX_CUDA(cudaFuncSetAttribute(k_eval_block<kLrgT, kLrgCap>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  100));
    RMX_CUDA(cudaFuncSetAttribute(k_eval_warp, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    RMX_CUDA(cudaFuncSetAttribute(k_hub_eval, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kHubEvalSmem));
    RMX_CUDA(cudaFuncSetAttribute(k_hub_eval, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    configured[dev] = true;
}

__global__ void k_iota(int32_t *list, int32_t n, int64_t *count) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        list[i] = (int32_t)i;
    if (blockIdx.x == 0 && threadIdx.x == 0) *count = n;
}

void all_units(int32_t n, SweepWork &W, cudaStream_t s) {
    k_iota<<<blocks_for(n, 256, num_sms() * 32), 256, 0, s>>>(W.list, n, W.counters + kCntActive);
    RMX_LAUNCHED();
}

// Upper degree bounds of the warp, mid, block and large bins (run-time tuning).
struct BinBounds {
    int32_t warp, mid, block, large;
};

__global__ void k_bucket(const int32_t *list, const int64_t *n_active, const int64_t *out_off, const int64_t *in_off,
                         uint32_t seed, const uint32_t *seed_dev, int nsub, BinBounds bb, uint16_t *bucket) {
    const int64_t n = *n_active;
    if (seed_dev) seed = *seed_dev;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t u = list[i];
        const int64_t d = (out_off[u + 1] - out_off[u]) + (in_off[u + 1] - in_off[u]);
        const int bin = d <= 8 ? kBinReg8
                        : d <= 16 ? kBinReg16
                        : d <= 32 ? kBinReg32
                        : d <= bb.warp ? kBinWarp
                        : d <= bb.mid ? kBinMid
                        : d <= bb.block ? kBinBlock
                        : d <= bb.large ? kBinLarge
                                        : kBinHub;
        const int sb = nsub > 1 ? (int)(mix32((uint32_t)u ^ seed) % (uint32_t)nsub) : 0;
        bucket[i] = (uint16_t)(sb * kBins + bin);
    }
}

__global__ void k_ranges(const int64_t *bucket_off, int nsub, int64_t *ranges) {
    const int sb = blockIdx.x * blockDim.x + threadIdx.x;
    if (sb < nsub) {
        ranges[2 * sb] = bucket_off[sb * kBins];
        ranges[2 * sb + 1] = bucket_off[sb * kBins + kBins];
    }
}

void bucket_units(const Level &L, SweepWork &W, int64_t n_active, uint32_t seed, int nsub, Arena &ar,
                  cudaStream_t s, bool host_counts) {
    if (nsub * kBins > 256) throw std::invalid_argument("too many sub-batches");
    const EvalTuning t = eval_tuning();
    const BinBounds bb{t.warp_max, t.mid_max, t.block_max, t.large_max};
    k_bucket<<<blocks_for(n_active, 256, num_sms() * 32), 256, 0, s>>>(W.list, W.counters + kCntActive, L.out_off,
                                                                       L.in_off, seed, nullptr, nsub, bb, W.bucket);
    RMX_LAUNCHED();
    bucket_partition(W.bucket, W.list, W.list2, n_active, nsub * kBins, W.bucket_off, ar, s);
    k_ranges<<<1, 128, 0, s>>>(W.bucket_off, nsub, W.ranges);
    RMX_LAUNCHED();
    if (!host_counts) return;
    // the bins' sizes on the host: empty bins are not launched, grids fit the work
    W.bucket_host.resize((size_t)nsub * kBins + 1);
    RMX_CUDA(cudaMemcpyAsync(W.bucket_host.data(), W.bucket_off, sizeof(int64_t) * W.bucket_host.size(),
                             cudaMemcpyDeviceToHost, s));
    RMX_CUDA(cudaStreamSynchronize(s));
}

void bucket_units_dev(const Level &L, SweepWork &W, int64_t n_max, const uint32_t *seed_dev, int nsub, Arena &ar,
                      cudaStream_t s) {
    if (nsub * kBins > 256) throw std::invalid_argument("too many sub-batches");
    const EvalTuning t = eval_tuning();
    const BinBounds bb{t.warp_max, t.mid_max, t.block_max, t.large_max};
    k_bucket<<<blocks_for(n_max, 256, num_sms() * 32), 256, 0, s>>>(W.list, W.counters + kCntActive, L.out_off,
                                                                    L.in_off, 0u, seed_dev, nsub, bb, W.bucket);
    RMX_LAUNCHED();
    bucket_partition_dev(W.bucket, W.list, W.list2, W.counters + kCntActive, n_max, nsub * kBins, W.bucket_off, ar,
                         s);
    k_ranges<<<1, 128, 0, s>>>(W.bucket_off, nsub, W.ranges);
    RMX_LAUNCHED();
}

__global__ void k_iota_dev(int32_t *list, const int64_t *n_dev, int64_t *count) {
    const int64_t n = *n_dev;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        list[i] = (int32_t)i;
    if (blockIdx.x == 0 && threadIdx.x == 0) *count = n;
}

void all_units_dev(const int64_t *n_dev, int64_t n_max, SweepWork &W, cudaStream_t s) {
    k_iota_dev<<<blocks_for(n_max, 256, num_sms() * 32), 256, 0, s>>>(W.list, n_dev, W.counters + kCntActive);
    RMX_LAUNCHED();
}

__global__ void k_empty_flags(int32_t cap, const int32_t *mcount, uint8_t *flag) {
    for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < cap; m += (int64_t)gridDim.x * blockDim.x)
        flag[m] = mcount[m] == 0 ? 1 : 0;
}

void free_modules(const ModState &M, SweepWork &W, Arena &ar, cudaStream_t s) {
    size_t mk = ar.mark();
    uint8_t *flag = ar.alloc<uint8_t>(std::max(M.cap, 1));
    k_empty_flags<<<blocks_for(M.cap, 256, num_sms() * 32), 256, 0, s>>>(M.cap, M.count, flag);
    RMX_LAUNCHED();
    compact_flags(flag, M.cap, W.free_list, W.counters + kCntFree, ar, s);
    ar.release(mk);
}

void sweep_subbatch(const Level &L, ModState &M, const InstState &I, SweepWork &W, const SweepArgs &sa, int sb,
                    const uint32_t *sp, bool mark_active, bool fitted, cudaStream_t s, Timers *tm) {
    // fitted: bin sizes known on the host (skip empty work, size grids); else
    // every kernel is launched with its full grid and reads its range on the
    // device (the form captured into a CUDA graph)
    const int64_t *hb = fitted ? W.bucket_host.data() + sb * kBins : nullptr;
    const int64_t total = fitted ? hb[kBins] - hb[0] : 1, n_light = fitted ? hb[kBinMid] - hb[kBinReg8] : 1,
                  n_heavy = fitted ? hb[kBins] - hb[kBinMid] : 1;
    if (total == 0) return;
    EvalArgs ea = eval_args(L, M, I, W, sa.vthresh, sa.allow_new, nullptr, 1);
    ea.mark = mark_active ? 1 : 0;
    if (tm) tm->begin(kTimerEval, s);
    launch_eval(ea, W.bucket_off, sb * kBins, W, fitted, s, tm);
    if (tm) {
        tm->end(kTimerEval, s);
        tm->log_eval(W.counters, s);
    }
    if (tm) tm->begin(kTimerCommit, s);
    CommitArgs ca;
    ca.list = W.list2;
    ca.range = W.ranges + 2 * sb;
    ca.prop = W.prop;
    ca.ptarget = W.ptarget;
    ca.mod = L.mod;
    ca.prevmod = W.prevmod;
    ca.stamp_of = W.stamp;
    ca.attr = L.attr;
    ca.uinst = L.inst;
    ca.nnodes = L.nnodes;
    ca.mstat = M.stat;
    ca.mcount = M.count;
    ca.minst = M.inst;
    ca.claim = W.claim;
    ca.free_list = W.free_list;
    ca.n_free = W.counters + kCntFree;
    ca.moved_nodes = reinterpret_cast<unsigned long long *>(W.counters + kCntMoved);
    ca.sp = sp;
    const unsigned G = fitted ? fit_grid(total, 256, num_sms() * 8) : num_sms() * 8;
    if (sa.allow_new) {
        k_claim<<<G, 256, 0, s>>>(ca);
        RMX_LAUNCHED();
    }
    k_commit<<<G, 256, 0, s>>>(ca);
    RMX_LAUNCHED();
    DeltaArgs da;
    da.list = W.list2;
    da.mod = L.mod;
    da.prevmod = W.prevmod;
    da.stamp_of = W.stamp;
    da.out_off = L.out_off;
    da.in_off = L.in_off;
    da.out_dst = L.out_dst;
    da.in_src = L.in_src;
    da.out_fx = L.out_fx;
    da.in_fx = L.in_fx;
    da.mstat = M.stat;
    da.sp = sp;
    // light movers (<= 128 links) a warp each, heavy ones a block each
    const int64_t *bo = W.bucket_off + sb * kBins;
    if (n_light > 0) {
        da.beg = bo + kBinReg8;
        da.end = bo + kBinMid;
        k_delta<<<fitted ? fit_grid(n_light, 8, num_sms() * 8) : num_sms() * 8, 256, 0, s>>>(da);
        RMX_LAUNCHED();
    }
    if (n_heavy > 0) {
        da.beg = bo + kBinMid;
        da.end = bo + kBins;
        k_delta_block<<<fitted ? fit_grid(n_heavy, 1, num_sms() * 4) : num_sms() * 4, 256, 0, s>>>(da);
        RMX_LAUNCHED();
    }
    k_terms_movers<<<G, 256, 0, s>>>(W.list2, W.ranges + 2 * sb, W.stamp, sp, L.mod, W.prevmod, M.stat, M.term,
                                     M.rec);
    RMX_LAUNCHED();
    if (tm) tm->end(kTimerCommit, s);
}

void evaluate_all(const Level &L, const ModState &M, const InstState &I, SweepWork &W, const uint8_t *allow_new,
                  double vthresh, Arena &ar, cudaStream_t s) {
    all_units(L.n, W, s);
    bucket_units(L, W, L.n, 0u, 1, ar, s);
    EvalArgs ea = eval_args(L, M, I, W, vthresh, 0, allow_new, 0);
    // allow_new == nullptr means "no empty-module candidate" for the hook
    if (!allow_new) ea.allow_new = 0;
    launch_eval(ea, W.bucket_off, 0, W, true, s);
}

}  // namespace rmx
