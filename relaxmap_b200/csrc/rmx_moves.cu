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

#include "rmx_engine.cuh"

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

// Insert key (linear probing); returns its slot. Capacity >= 2 * keys inserted.
__device__ __forceinline__ int tab_insert(int32_t *keys, int mask, int32_t key) {
    int s = tab_slot(key, mask);
    for (int probe = 0; probe <= mask; probe++) {
        int32_t prev = atomicCAS(keys + s, kEmpty, key);
        if (prev == kEmpty || prev == key) return s;
        s = (s + 1) & mask;
    }
    return -1;
}

__device__ __forceinline__ bool better(double d1, int32_t m1, double d2, int32_t m2) {
    return d1 < d2 || (d1 == d2 && m1 < m2);
}

// Everything about the moving unit that every candidate needs.
struct UnitCtx {
    double pu, tu, du, eu, cu;  // flow, teleport weight, dangling flow, exit, tau*p + (1-tau)*d
    double eA, PA, nexA, nPA;   // old module: exit, flow, exit and flow after leaving
    double sum_exit;
    int32_t A;
};

__device__ __forceinline__ double delta_L(double se, double nse, double e1, double P1, double e2, double P2,
                                          double ne1, double nP1, double ne2, double nP2) {
    // Module.cpp:1109-1115
    double d_all = plogp(nse) - plogp(se);
    double d_exit = plogp(ne1) + plogp(ne2) - plogp(e1) - plogp(e2);
    double d_stay = plogp(ne1 + nP1) + plogp(ne2 + nP2) - plogp(e1 + P1) - plogp(e2 + P2);
    return d_all - 2.0 * d_exit + d_stay;
}

// Change of moving the unit into module with statistics st, given the unit's
// aggregated out-/in-flow (fixed point, before the 1-tau factor) to it.
__device__ __forceinline__ double candidate_delta(const UnitCtx &c, const Stat4 &st, fx_t ofx, fx_t ifx) {
    const double P = from_fx(st.P), TW = from_fx(st.TW), D = from_fx(st.D), OUT = from_fx(st.OUT);
    const double em = exit_flow(P, TW, D, OUT);
    const double om = kBeta * from_fx(ofx) + c.cu * TW;                   // Module.cpp:1058
    const double im = kBeta * from_fx(ifx) + (kAlpha * P + kBeta * D) * c.tu;  // Module.cpp:1059
    const double nexm = em + c.eu - om - im;                              // Module.cpp:1104
    const double nse = c.sum_exit + c.nexA + nexm - c.eA - em;           // Module.cpp:1106
    return delta_L(c.sum_exit, nse, c.eA, c.PA, em, P, c.nexA, c.nPA, nexm, P + c.pu);
}

// The empty-module option: exit e_u, no shared flow (Module.cpp:1072-1077).
__device__ __forceinline__ double newmod_delta(const UnitCtx &c) {
    const double nexm = c.eu;
    const double nse = c.sum_exit + c.nexA + nexm - c.eA;
    return delta_L(c.sum_exit, nse, c.eA, c.PA, 0.0, 0.0, c.nexA, c.nPA, nexm, c.pu);
}

__device__ __forceinline__ UnitCtx make_ctx(const Stat4 &ua, const Stat4 &ma, double sum_exit, int32_t A, fx_t oA,
                                            fx_t iA) {
    UnitCtx c;
    c.pu = from_fx(ua.P);
    c.tu = from_fx(ua.TW);
    c.du = from_fx(ua.D);
    c.eu = exit_flow(c.pu, c.tu, c.du, from_fx(ua.OUT));
    c.cu = kAlpha * c.pu + kBeta * c.du;
    c.PA = from_fx(ma.P);
    const double TWA = from_fx(ma.TW), DA = from_fx(ma.D);
    c.eA = exit_flow(c.PA, TWA, DA, from_fx(ma.OUT));
    const double outA = kBeta * from_fx(oA) + c.cu * (TWA - c.tu);                            // :1047
    const double inA = kBeta * from_fx(iA) + (kAlpha * (c.PA - c.pu) + kBeta * (DA - c.du)) * c.tu;  // :1048
    c.nexA = c.eA - c.eu + outA + inA;                                                         // :1084
    c.nPA = c.PA - c.pu;
    c.sum_exit = sum_exit;
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
    const Stat4 *mstat;
    const int32_t *mcount;
    const double *inst_sum_exit;
    const uint8_t *inst_active;
    // work
    const int32_t *list;
    const int64_t *range;  // [beg, end) at range[0], range[1]
    int32_t *prop;
    double *pdelta;
    unsigned long long *edges_seen;
    double vthresh;
    int allow_new;             // stage-level switch
    const uint8_t *allow_new_unit;  // optional per-unit override (parity hook)
    int swap_guard;            // singleton min-label rule
    fx_t *gtable;              // hub tables: [block][gcap] out, in
    int32_t *gkeys;
    int64_t gcap;
};

// Decide and write the proposal for unit u given the argmin over candidates.
__device__ __forceinline__ void finish_unit(const EvalArgs &a, int32_t u, const UnitCtx &c, double best,
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
}

// ---------------------------------------------------------------- warp kernel
// One warp per unit with out+in degree <= 64: table of up to 128 slots in
// shared memory per warp.

constexpr int kWarpCap = 128, kWarpMaxDeg = 64, kEvalWarps = 8;
constexpr int kBins = 3;  // degree bins: warp, block (shared table), hub (global table)

__global__ void __launch_bounds__(kEvalWarps * 32) k_eval_warp(EvalArgs a) {
    __shared__ int32_t skey[kEvalWarps][kWarpCap];
    __shared__ fx_t sout[kEvalWarps][kWarpCap];
    __shared__ fx_t sin_[kEvalWarps][kWarpCap];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int32_t *keys = skey[w];
    fx_t *vo = sout[w], *vi = sin_[w];
    const int64_t beg = a.range[0], end = a.range[1];
    const int64_t gw = ((int64_t)blockIdx.x * kEvalWarps + w), nw = (int64_t)gridDim.x * kEvalWarps;
    unsigned long long seen = 0;
    for (int64_t i = beg + gw; i < end; i += nw) {
        const int32_t u = a.list[i];
        if (!a.inst_active[a.uinst[u]]) {
            if (lane == 0) a.prop[u] = -1;
            continue;
        }
        const int64_t ob = a.out_off[u], ib = a.in_off[u];
        const int dout = (int)(a.out_off[u + 1] - ob), din = (int)(a.in_off[u + 1] - ib), d = dout + din;
        int cap = 32;
        while (cap < 2 * d) cap <<= 1;
        const int mask = cap - 1;
        for (int s = lane; s < cap; s += 32) {
            keys[s] = kEmpty;
            vo[s] = 0;
            vi[s] = 0;
        }
        __syncwarp();
        for (int j = lane; j < d; j += 32) {
            int32_t nb;
            fx_t q;
            bool isout = j < dout;
            if (isout) {
                nb = a.out_dst[ob + j];
                q = a.out_fx[ob + j];
            } else {
                nb = a.in_src[ib + j - dout];
                q = a.in_fx[ib + j - dout];
            }
            const int s = tab_insert(keys, mask, a.mod[nb]);
            atomic_add_fx(isout ? vo + s : vi + s, q);
        }
        seen += d;
        __syncwarp();
        const int32_t A = a.mod[u];
        // flows to the unit's own module
        fx_t oA = 0, iA = 0;
        for (int s = lane; s < cap; s += 32)
            if (keys[s] == A) {
                oA = vo[s];
                iA = vi[s];
            }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            oA += __shfl_xor_sync(kFull, oA, o);
            iA += __shfl_xor_sync(kFull, iA, o);
        }
        const UnitCtx c = make_ctx(a.attr[u], a.mstat[A], a.inst_sum_exit[a.uinst[u]], A, oA, iA);
        double best = 0.0;
        int32_t bm = INT_MAX;
        for (int s = lane; s < cap; s += 32) {
            const int32_t m = keys[s];
            if (m == kEmpty || m == A) continue;
            const double dl = candidate_delta(c, a.mstat[m], vo[s], vi[s]);
            if (better(dl, m, best, bm)) {
                best = dl;
                bm = m;
            }
        }
        // lanes that saw no candidate hold (0, INT_MAX): never better than a real one
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ob2 = __shfl_xor_sync(kFull, best, o);
            const int32_t om = __shfl_xor_sync(kFull, bm, o);
            if (better(ob2, om, best, bm)) {
                best = ob2;
                bm = om;
            }
        }
        if (lane == 0) finish_unit(a, u, c, best, bm);
        __syncwarp();
    }
    if (lane == 0 && seen) atomicAdd(a.edges_seen, seen);
}

// ---------------------------------------------------------------- block kernel
// One block per unit; the table lives in shared memory (CAP slots) or, for
// hubs, in a per-block slice of a global table.

template <int NT, bool GLOBAL>
__global__ void __launch_bounds__(NT) k_eval_block(EvalArgs a, int cap_smem) {
    extern __shared__ __align__(16) unsigned char dsm[];
    __shared__ double rbest[NT / 32];
    __shared__ int32_t rmod[NT / 32];
    __shared__ fx_t rA[2][NT / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int32_t *keys;
    fx_t *vo, *vi;
    int64_t capmax;
    if (GLOBAL) {
        capmax = a.gcap;
        keys = a.gkeys + (int64_t)blockIdx.x * capmax;
        vo = a.gtable + (int64_t)blockIdx.x * capmax * 2;
        vi = vo + capmax;
    } else {
        capmax = cap_smem;
        vo = reinterpret_cast<fx_t *>(dsm);
        vi = vo + cap_smem;
        keys = reinterpret_cast<int32_t *>(vi + cap_smem);
    }
    const int64_t beg = a.range[0], end = a.range[1];
    unsigned long long seen = 0;
    for (int64_t i = beg + blockIdx.x; i < end; i += gridDim.x) {
        const int32_t u = a.list[i];
        if (!a.inst_active[a.uinst[u]]) {
            if (threadIdx.x == 0) a.prop[u] = -1;
            continue;
        }
        const int64_t ob = a.out_off[u], ib = a.in_off[u];
        const int64_t dout = a.out_off[u + 1] - ob, din = a.in_off[u + 1] - ib, d = dout + din;
        int64_t cap = 64;
        while (cap < 2 * d) cap <<= 1;
        if (cap > capmax) cap = capmax;  // never for correctly binned units
        const int mask = (int)(cap - 1);
        for (int64_t s = threadIdx.x; s < cap; s += NT) {
            keys[s] = kEmpty;
            vo[s] = 0;
            vi[s] = 0;
        }
        __syncthreads();
        for (int64_t j = threadIdx.x; j < d; j += NT) {
            int32_t nb;
            fx_t q;
            bool isout = j < dout;
            if (isout) {
                nb = a.out_dst[ob + j];
                q = a.out_fx[ob + j];
            } else {
                nb = a.in_src[ib + j - dout];
                q = a.in_fx[ib + j - dout];
            }
            const int s = tab_insert(keys, mask, a.mod[nb]);
            if (s >= 0) atomic_add_fx(isout ? vo + s : vi + s, q);
        }
        seen += d;
        __syncthreads();
        const int32_t A = a.mod[u];
        fx_t oA = 0, iA = 0;
        for (int64_t s = threadIdx.x; s < cap; s += NT)
            if (keys[s] == A) {
                oA = vo[s];
                iA = vi[s];
            }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            oA += __shfl_xor_sync(kFull, oA, o);
            iA += __shfl_xor_sync(kFull, iA, o);
        }
        if (lane == 0) {
            rA[0][w] = oA;
            rA[1][w] = iA;
        }
        __syncthreads();
        oA = 0;
        iA = 0;
#pragma unroll
        for (int q = 0; q < NT / 32; q++) {
            oA += rA[0][q];
            iA += rA[1][q];
        }
        const UnitCtx c = make_ctx(a.attr[u], a.mstat[A], a.inst_sum_exit[a.uinst[u]], A, oA, iA);
        double best = 0.0;
        int32_t bm = INT_MAX;
        for (int64_t s = threadIdx.x; s < cap; s += NT) {
            const int32_t m = keys[s];
            if (m == kEmpty || m == A) continue;
            const double dl = candidate_delta(c, a.mstat[m], vo[s], vi[s]);
            if (better(dl, m, best, bm)) {
                best = dl;
                bm = m;
            }
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
            rbest[w] = best;
            rmod[w] = bm;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int q = 1; q < NT / 32; q++)
                if (better(rbest[q], rmod[q], best, bm)) {
                    best = rbest[q];
                    bm = rmod[q];
                }
            finish_unit(a, u, c, best, bm);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && seen) atomicAdd(a.edges_seen, seen);
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
    uint32_t stamp;
};

__device__ __forceinline__ unsigned long long claim_key(uint32_t stamp, int32_t u) {
    return ((unsigned long long)stamp << 32) | (0xffffffffu - (uint32_t)u);
}

// Units proposing an empty module bid for a free id chosen by hash; the
// smallest unit id wins each id (atomicMax on an inverted key), losers stay.
__global__ void k_claim(CommitArgs a) {
    const int64_t beg = a.range[0], end = a.range[1];
    const int64_t nf = *a.n_free;
    for (int64_t i = beg + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < end;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t u = a.list[i];
        if (a.prop[u] != kNewMod) continue;
        int32_t m = -1;
        if (nf > 0) {
            int64_t s = mix32((uint32_t)u ^ (a.stamp * 0x9e3779b9U)) % nf;
            for (int probe = 0; probe < 8; probe++, s = (s + 1) % nf) {
                const int32_t cand = a.free_list[s];
                if (a.mcount[cand] == 0) {
                    m = cand;
                    break;
                }
            }
        }
        a.ptarget[u] = m;
        if (m >= 0) atomicMax(a.claim + m, claim_key(a.stamp, u));
    }
}

__global__ void k_commit(CommitArgs a) {
    const int64_t beg = a.range[0], end = a.range[1];
    unsigned long long moved = 0;
    for (int64_t i = beg + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < end;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t u = a.list[i];
        int32_t t = a.prop[u];
        if (t == -1) continue;
        if (t == kNewMod) {
            t = a.ptarget[u];
            if (t < 0 || a.claim[t] != claim_key(a.stamp, u)) continue;
            a.minst[t] = a.uinst[u];
        }
        const int32_t A = a.mod[u];
        a.prevmod[u] = A;
        a.mod[u] = t;
        a.stamp_of[u] = a.stamp;
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
    const int64_t *range;
    const int32_t *prop;
    const int32_t *mod, *prevmod;
    const uint32_t *stamp_of;
    const int64_t *out_off, *in_off;
    const int32_t *out_dst, *in_src;
    const fx_t *out_fx, *in_fx;
    Stat4 *mstat;
    uint8_t *next_active;
    uint32_t stamp;
    int mark;
};

// Out-flow bookkeeping for the movers of this sub-batch; warp per unit.
// Link u->w adds its flow to OUT[mod(u)] iff mod(u) != mod(w). Links whose
// both ends moved are handled once, by the source's out-link loop.
__global__ void __launch_bounds__(256) k_delta(DeltaArgs a) {
    const int lane = threadIdx.x & 31;
    const int64_t beg = a.range[0], end = a.range[1];
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = beg + gw; i < end; i += nw) {
        const int32_t u = a.list[i];
        if (a.prop[u] == -1) continue;
        const bool moved = a.stamp_of[u] == a.stamp;
        if (!moved && !a.mark) continue;
        const int32_t A = moved ? a.prevmod[u] : a.mod[u], T = a.mod[u];
        for (int64_t e = a.out_off[u] + lane; e < a.out_off[u + 1]; e += 32) {
            const int32_t w = a.out_dst[e];
            if (moved) {
                const fx_t q = a.out_fx[e];
                const bool wm = a.stamp_of[w] == a.stamp;
                const int32_t bn = a.mod[w], bo = wm ? a.prevmod[w] : bn;
                if (A != bo) atomic_add_fx(&a.mstat[A].OUT, -q);
                if (T != bn) atomic_add_fx(&a.mstat[T].OUT, q);
            }
            if (a.mark) a.next_active[w] = 1;
        }
        for (int64_t e = a.in_off[u] + lane; e < a.in_off[u + 1]; e += 32) {
            const int32_t w = a.in_src[e];
            if (moved && a.stamp_of[w] != a.stamp) {
                const int32_t b = a.mod[w];
                if (b == A)
                    atomic_add_fx(&a.mstat[A].OUT, a.in_fx[e]);
                else if (b == T)
                    atomic_add_fx(&a.mstat[T].OUT, -a.in_fx[e]);
            }
            if (a.mark) a.next_active[w] = 1;
        }
    }
}

// ---------------------------------------------------------------- stats

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
__global__ void __launch_bounds__(256) k_mod_terms(int32_t cap, const Stat4 *mstat, const int32_t *mcount,
                                                   const int32_t *minst, fx_t *acc) {
    __shared__ fx_t sh[3][8];
    fx_t t0 = 0, t1 = 0, t2 = 0;
    for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < cap; m += (int64_t)gridDim.x * blockDim.x) {
        if (mcount[m] <= 0) continue;
        const Stat4 st = mstat[m];
        const double P = from_fx(st.P);
        const double e = exit_flow(P, from_fx(st.TW), from_fx(st.D), from_fx(st.OUT));
        const fx_t a0 = to_fxl(e), a1 = to_fxl(plogp(e)), a2 = to_fxl(plogp(e + P));
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
        k_mod_terms<true><<<blocks_for(M.cap, 256, num_sms() * 8), 256, 0, s>>>(M.cap, M.stat, M.count, M.inst, I.acc);
    else
        k_mod_terms<false><<<blocks_for(M.cap, 256, num_sms() * 8), 256, 0, s>>>(M.cap, M.stat, M.count, M.inst,
                                                                                 I.acc);
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
    a.mstat = M.stat;
    a.mcount = M.count;
    a.inst_sum_exit = I.sum_exit;
    a.inst_active = I.active;
    a.list = W.list2;
    a.range = nullptr;
    a.prop = W.prop;
    a.pdelta = W.pdelta;
    a.edges_seen = reinterpret_cast<unsigned long long *>(W.counters + kCntEdges);
    a.vthresh = vthresh;
    a.allow_new = allow_new;
    a.allow_new_unit = allow_unit;
    a.swap_guard = swap_guard;
    a.gtable = W.gtable;
    a.gkeys = W.gkeys;
    a.gcap = W.gcap;
    return a;
}

constexpr int kBlkT = 256, kBlkCap = 4096, kHubT = 512;

int hub_blocks() { return std::min(num_sms(), 64); }
int64_t block_bin_max_degree() { return kBlkCap / 2; }
int64_t warp_bin_max_degree() { return kWarpMaxDeg; }

static void launch_eval(EvalArgs a, const int64_t *bucket_off, int first_bucket, cudaStream_t s) {
    a.range = bucket_off + first_bucket + 0;  // bin 0: warp per unit
    k_eval_warp<<<num_sms() * 8, kEvalWarps * 32, 0, s>>>(a);
    RMX_LAUNCHED();
    a.range = bucket_off + first_bucket + 1;  // bin 1: block per unit, shared-memory table
    const size_t smem = (size_t)kBlkCap * (2 * sizeof(fx_t) + sizeof(int32_t));
    k_eval_block<kBlkT, false><<<num_sms() * 2, kBlkT, smem, s>>>(a, kBlkCap);
    RMX_LAUNCHED();
    if (a.gcap > 0) {  // bin 2: hubs, per-block slice of a global table
        a.range = bucket_off + first_bucket + 2;
        k_eval_block<kHubT, true><<<hub_blocks(), kHubT, 0, s>>>(a, 0);
        RMX_LAUNCHED();
    }
}

void configure_eval_kernels() {
    static bool done = false;
    if (done) return;
    const size_t smem = (size_t)kBlkCap * (2 * sizeof(fx_t) + sizeof(int32_t));
    RMX_CUDA(cudaFuncSetAttribute(k_eval_block<kBlkT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    done = true;
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

__global__ void k_bucket(const int32_t *list, const int64_t *n_active, const int64_t *out_off, const int64_t *in_off,
                         uint32_t seed, int nsub, uint16_t *bucket) {
    const int64_t n = *n_active;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t u = list[i];
        const int64_t d = (out_off[u + 1] - out_off[u]) + (in_off[u + 1] - in_off[u]);
        const int bin = d <= kWarpMaxDeg ? 0 : (d <= kBlkCap / 2 ? 1 : 2);
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
                  cudaStream_t s) {
    if (nsub * kBins > 255) throw std::invalid_argument("too many sub-batches");
    k_bucket<<<blocks_for(n_active, 256, num_sms() * 32), 256, 0, s>>>(W.list, W.counters + kCntActive, L.out_off,
                                                                       L.in_off, seed, nsub, W.bucket);
    RMX_LAUNCHED();
    bucket_partition(W.bucket, W.list, W.list2, n_active, nsub * kBins, W.bucket_off, ar, s);
    k_ranges<<<1, 128, 0, s>>>(W.bucket_off, nsub, W.ranges);
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
                    uint32_t stamp, bool mark_active, cudaStream_t s, Timers *tm) {
    EvalArgs ea = eval_args(L, M, I, W, sa.vthresh, sa.allow_new, nullptr, 1);
    if (tm) tm->begin(kTimerEval, s);
    launch_eval(ea, W.bucket_off, sb * kBins, s);
    if (tm) tm->end(kTimerEval, s);
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
    ca.stamp = stamp;
    const unsigned G = num_sms() * 8;
    if (sa.allow_new) {
        k_claim<<<G, 256, 0, s>>>(ca);
        RMX_LAUNCHED();
    }
    k_commit<<<G, 256, 0, s>>>(ca);
    RMX_LAUNCHED();
    DeltaArgs da;
    da.list = W.list2;
    da.range = W.ranges + 2 * sb;
    da.prop = W.prop;
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
    da.next_active = W.next_active;
    da.stamp = stamp;
    da.mark = mark_active ? 1 : 0;
    k_delta<<<G, 256, 0, s>>>(da);
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
    launch_eval(ea, W.bucket_off, 0, s);
}

}  // namespace rmx
