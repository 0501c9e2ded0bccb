// The optimiser driver: graph construction, initiate, and the superstep loop of
// the reference (OmpRelaxmap.cpp:155-233, stochastic_greedy_partition :263-429,
// generate_sub_modules :502-638) orchestrating the device kernels.
//
// Control flow and stop rules are the reference's; the moves themselves are
// the bulk-synchronous sub-batch sweeps of rmx_moves.cu. Every sweep ends with
// one small device->host read (code length, moved nodes, next active count),
// the only synchronisation inside the loop.
#include <algorithm>
#include <functional>
#include <cmath>
#include <cstring>

#include "rmx_graph.hpp"
#include "rmx_io.hpp"

using namespace rmx;

namespace {

constexpr unsigned kFull = 0xffffffffu;
const double kLn2 = std::log(2.0);

__global__ void k_fill(double *a, int64_t n, double v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        a[i] = v;
}

__global__ void k_flags_nonempty(int32_t cap, const int32_t *count, int64_t *flag) {
    for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < cap; m += (int64_t)gridDim.x * blockDim.x)
        flag[m] = count[m] > 0 ? 1 : 0;
}

// modules -> super-nodes (convertModulesToSuperNodes, Module.cpp:3015-3022 and
// SuperNode(Module, int) Node.cpp:76-106): the super-node carries the module's
// statistics exactly and keeps the module id.
__global__ void k_sn_from_modules(int32_t cap, const int32_t *count, const int64_t *snid, const Stat4 *mstat,
                                  const int32_t *minst, int32_t *sn_mod, Stat4 *sn_attr, int32_t *sn_nnodes,
                                  int32_t *sn_inst) {
    for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < cap; m += (int64_t)gridDim.x * blockDim.x) {
        if (count[m] <= 0) continue;
        const int64_t s = snid[m];
        sn_mod[s] = (int32_t)m;
        sn_attr[s] = mstat[m];
        sn_nnodes[s] = count[m];
        if (minst) sn_inst[s] = minst[m];
    }
}

__global__ void k_group_of_nodes(int32_t n, const int32_t *mod, const int64_t *snid, int32_t *node_sn) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        node_sn[v] = (int32_t)snid[mod[v]];
}

__global__ void k_project(int32_t n, const int32_t *node_sn, const int32_t *sn_mod, int32_t *nmod) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        nmod[v] = sn_mod[node_sn[v]];
}

// Intra-module links for the coarse-tune sub-networks (generate_network_from_module,
// OmpRelaxmap.cpp:664-684): per row, the links whose other end shares the module.
__global__ void k_intra_count(int32_t n, const int64_t *off, const int32_t *nbr, const int32_t *mod, int64_t *cnt) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t u = gw; u < n; u += nw) {
        const int32_t m = mod[u];
        int c = 0;
        for (int64_t e = off[u] + lane; e < off[u + 1]; e += 32) c += mod[nbr[e]] == m;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(kFull, c, o);
        if (lane == 0) cnt[u] = c;
    }
}

__global__ void k_intra_fill(int32_t n, const int64_t *off, const int32_t *nbr, const fx_t *fx, const int32_t *mod,
                             const int64_t *noff, int32_t *nnbr, fx_t *nfx, fx_t *row_sum) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t u = gw; u < n; u += nw) {
        const int32_t m = mod[u];
        int64_t pos = noff[u];
        fx_t sum = 0;
        for (int64_t base = off[u]; base < off[u + 1]; base += 32) {
            const int64_t e = base + lane;
            const bool keep = e < off[u + 1] && mod[nbr[e]] == m;
            const unsigned bal = __ballot_sync(kFull, keep);
            if (keep) {
                const int64_t q = pos + __popc(bal & lt);
                nnbr[q] = nbr[e];
                nfx[q] = fx[e];
                sum += fx[e];
            }
            pos += __popc(bal);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(kFull, sum, o);
        if (row_sum && lane == 0) row_sum[u] = sum;
    }
}

__global__ void k_sub_attr(int32_t n, const Stat4 *nattr, const fx_t *intra_out, Stat4 *sattr) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        Stat4 a = nattr[v];
        a.OUT = intra_out[v];
        sattr[v] = a;
    }
}

__global__ void k_sub_s0(int32_t n, const double *p, const int32_t *inst, fx_t *s0) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        atomic_add_fx(s0 + inst[v], to_fxl(plogp(p[v])));
}

// A parent module is coarse-tuned if it has two or more members and its
// instance is still running.
__global__ void k_inst_active(int32_t n, const int32_t *count, const int32_t *minst, const uint8_t *top_active,
                              uint8_t *active) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        active[k] = count[k] > 1 && top_active[minst[k]] ? 1 : 0;
}

// partition_module_network's stop rule per sub-network (OmpRelaxmap.cpp:458-459).
__global__ void k_inst_stop(int32_t n, const double *L, double *L_prev, uint8_t *active, double threshold,
                            double ln2, unsigned long long *n_active) {
    unsigned long long c = 0;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        if (!active[k]) continue;
        if ((L_prev[k] - L[k]) / ln2 < threshold)
            active[k] = 0;
        else
            c++;
        L_prev[k] = L[k];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(kFull, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(n_active, c);
}

__global__ void k_copy_L(int32_t n, const double *L, double *L_prev) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        L_prev[k] = L[k];
}

// super-nodes of sub-modules (SuperNode(SubModule*,...) Node.cpp:108-137): sums
// of the member nodes; the module is the parent module of the members.
__global__ void k_sn_from_nodes(int32_t n, const int32_t *node_sn, const int32_t *nmod, const Stat4 *nattr,
                                const int32_t *node_inst, int32_t *sn_mod, Stat4 *sn_attr, int32_t *sn_nnodes,
                                int32_t *sn_inst) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t s = node_sn[v];
        sn_mod[s] = nmod[v];
        if (node_inst) sn_inst[s] = node_inst[v];
        const Stat4 a = nattr[v];
        atomic_add_fx(&sn_attr[s].P, a.P);
        atomic_add_fx(&sn_attr[s].TW, a.TW);
        atomic_add_fx(&sn_attr[s].D, a.D);
        atomicAdd(sn_nnodes + s, 1);
    }
}

__global__ void k_sn_set_out(int32_t n, const fx_t *rowsum, Stat4 *attr) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x)
        attr[s].OUT = rowsum[s];
}

__global__ void k_remap(int32_t n, const int32_t *map, int32_t *mod) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x)
        mod[s] = map[mod[s]];
}

__global__ void k_count_nonzero(int32_t cap, const int32_t *count, unsigned long long *out) {
    unsigned long long c = 0;
    for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < cap; m += (int64_t)gridDim.x * blockDim.x)
        c += count[m] > 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(kFull, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

__global__ void k_max_degree(int32_t n, const int64_t *out_off, const int64_t *in_off, unsigned long long *mx) {
    unsigned long long d = 0;
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n; u += (int64_t)gridDim.x * blockDim.x) {
        unsigned long long x = (out_off[u + 1] - out_off[u]) + (in_off[u + 1] - in_off[u]);
        d = x > d ? x : d;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long y = __shfl_xor_sync(kFull, d, o);
        d = y > d ? y : d;
    }
    if ((threadIdx.x & 31) == 0 && d) atomicMax(mx, d);
}

// From-scratch FP64 code length (calculateCodeLength, Module.cpp:2966-3002).
__global__ void k_fp64_nodes(int32_t n, const int32_t *part, const double *p, const double *tw, const uint8_t *dang,
                             double *P, double *TW, double *D, int32_t *cnt) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t m = part[v];
        atomicAdd(P + m, p[v]);
        atomicAdd(TW + m, tw[v]);
        if (dang[v]) atomicAdd(D + m, p[v]);
        atomicAdd(cnt + m, 1);
    }
}

__global__ void k_fp64_out(int32_t n, const int64_t *off, const int32_t *dst, const double *f, const int32_t *part,
                           double *OUT) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t u = gw; u < n; u += nw) {
        const int32_t m = part[u];
        double o = 0.0;
        for (int64_t e = off[u] + lane; e < off[u + 1]; e += 32)
            if (part[dst[e]] != m) o += f[e];
#pragma unroll
        for (int q = 16; q > 0; q >>= 1) o += __shfl_xor_sync(kFull, o, q);
        if (lane == 0 && o != 0.0) atomicAdd(OUT + m, o);
    }
}

__global__ void k_fp64_terms(int32_t n, const double *P, const double *TW, const double *D, const double *OUT,
                             const int32_t *cnt, const double *p, double *parts) {
    __shared__ double sh[4][8];
    double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
    for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < n; m += (int64_t)gridDim.x * blockDim.x) {
        a3 += plogp(p[m]);
        if (cnt[m] <= 0) continue;
        double e = kAlpha * (1.0 - TW[m]) * P[m];
        e += kBeta * (OUT[m] + (1.0 - TW[m]) * D[m]);
        a0 += e;
        a1 += plogp(e);
        a2 += plogp(e + P[m]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(kFull, a0, o);
        a1 += __shfl_xor_sync(kFull, a1, o);
        a2 += __shfl_xor_sync(kFull, a2, o);
        a3 += __shfl_xor_sync(kFull, a3, o);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        sh[0][w] = a0;
        sh[1][w] = a1;
        sh[2][w] = a2;
        sh[3][w] = a3;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double v = 0;
        for (int q = 0; q < 8; q++) v += sh[threadIdx.x][q];
        parts[4 * blockIdx.x + threadIdx.x] = v;
    }
}

__host__ __device__ uint32_t mix_seed(uint32_t a, uint64_t b) {
    uint64_t x = a * 0x9E3779B97F4A7C15ull ^ (b + 0x632BE59BD9B4E019ull);
    x ^= x >> 31;
    x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 29;
    return (uint32_t)(x ^ (x >> 32));
}

// ---- a stage loop captured as one graph (while node; the body is one sweep)

// Start of a sweep, as the host loop does it: the sweep number and its seed,
// each sub-batch's stamp and hash seed (run_subbatches), the instances that
// take part (set_active) and the code lengths before the sweep.
__global__ void k_stage_begin(int64_t *ctl, uint32_t *seed_out, int ns, uint32_t *dparams, int32_t K,
                              const uint8_t *sweeping, uint8_t *active, const double *L, double *oldL) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const uint64_t sw = (uint64_t)ctl[0] + 1;
        const uint32_t seed = mix_seed((uint32_t)ctl[2], sw);
        uint32_t st = (uint32_t)ctl[1];
        for (int sb = 0; sb < ns; sb++) {
            dparams[2 * sb] = ++st;
            dparams[2 * sb + 1] = mix_seed(seed, (uint64_t)sb);
        }
        ctl[0] = (int64_t)sw;
        ctl[1] = (int64_t)st;
        ctl[4] = 0;
        *seed_out = seed;
    }
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < K; k += (int64_t)gridDim.x * blockDim.x) {
        active[k] = sweeping[k];
        oldL[k] = L[k];
    }
}

// The stop rule of stage_sweeps per instance (OmpRelaxmap.cpp:291-339): an
// instance stops when a sweep gained less than threshold bits and did not lose.
__global__ void k_stage_stop(int32_t K, const double *L, const double *oldL, uint8_t *sweeping, double threshold,
                             double ln2, unsigned long long *remaining) {
    unsigned long long c = 0;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < K; k += (int64_t)gridDim.x * blockDim.x) {
        if (!sweeping[k]) continue;
        const double d = oldL[k] - L[k];
        if (d >= 0 && d / ln2 < threshold)
            sweeping[k] = 0;
        else
            c++;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(kFull, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(remaining, c);
}

// Count the sweep and decide whether the while node runs its body again.
__global__ void k_stage_cond(int64_t *ctl, int max_iter, cudaGraphConditionalHandle cond) {
    const int64_t it = ctl[3] + 1;
    ctl[3] = it;
    cudaGraphSetConditional(cond, (ctl[4] > 0 && it < max_iter) ? 1u : 0u);
}

}  // namespace

// ------------------------------------------------------------------ Timers
namespace rmx {

void Timers::begin(int k, cudaStream_t s) {
    if (!on) return;
    if (used == pool.size()) {
        cudaEvent_t e;
        RMX_CUDA(cudaEventCreate(&e));
        pool.push_back(e);
    }
    open[k] = pool[used++];
    RMX_CUDA(cudaEventRecord(open[k], s));
}

void Timers::end(int k, cudaStream_t s) {
    if (!on) return;
    if (used == pool.size()) {
        cudaEvent_t e;
        RMX_CUDA(cudaEventCreate(&e));
        pool.push_back(e);
    }
    cudaEvent_t e = pool[used++];
    RMX_CUDA(cudaEventRecord(e, s));
    pending.push_back({k, open[k], e});
    launches[k]++;
    if (used > 16384) resolve();
}

__global__ void k_snapshot(const int64_t *counters, int64_t *dst) {
    if (threadIdx.x == 0) dst[0] = counters[kCntMods];
    if (threadIdx.x < 3 * kEvalBins) dst[1 + threadIdx.x] = counters[kCntBins + threadIdx.x];
}

void Timers::log_eval(const int64_t *counters, cudaStream_t s) {
    if (!on || !dlog) return;
    if (nlog == logcap) resolve();
    k_snapshot<<<1, 32, 0, s>>>(counters, dlog + kLogWords * nlog);
    RMX_LAUNCHED();
    log_stream = s;
    nlog++;
}

void Timers::resolve() {
    for (auto &p : pending) {
        RMX_CUDA(cudaEventSynchronize(p.b));
        float t = 0;
        RMX_CUDA(cudaEventElapsedTime(&t, p.a, p.b));
        ms[p.k] += t;
    }
    pending.clear();
    used = 0;
    if (nlog > 0) {
        std::vector<int64_t> h(kLogWords * nlog);
        RMX_CUDA(cudaMemcpyAsync(h.data(), dlog, sizeof(int64_t) * h.size(), cudaMemcpyDeviceToHost, log_stream));
        RMX_CUDA(cudaStreamSynchronize(log_stream));
        for (int64_t i = 0; i < nlog; i++) {
            const int64_t *c = h.data() + kLogWords * i;
            const double mods = (double)c[0];
            double tl = 0, tu = 0, tc = 0;
            for (int b = 0; b < kEvalBins; b++) {
                const int64_t *cb = c + 1 + 3 * b, *lb = last + 3 * b;
                const double dl = (double)(cb[0] - lb[0]), du = (double)(cb[1] - lb[1]), dc = (double)(cb[2] - lb[2]);
                eval_bin_bytes[b] += 16.0 * dl + 40.0 * du + 40.0 * std::min(dc, mods);
                tl += dl;
                tu += du;
                tc += dc;
            }
            eval_bytes += 16.0 * tl + 40.0 * tu + 40.0 * std::min(tc, mods);
            for (int q = 0; q < 3 * kEvalBins; q++) last[q] = c[1 + q];
        }
        nlog = 0;
    }
}

void Timers::reset() {
    pending.clear();
    used = 0;
    for (int k = 0; k < kTimerCount; k++) {
        ms[k] = 0;
        launches[k] = 0;
    }
    nlog = 0;
    for (int64_t &v : last) v = 0;
    eval_bytes = 0.0;
    for (double &v : eval_bin_bytes) v = 0.0;
}

void Timers::destroy() {
    for (auto e : pool) cudaEventDestroy(e);
    pool.clear();
    pending.clear();
    used = 0;
}

}  // namespace rmx

// ------------------------------------------------------------------ rmx_graph

rmx_graph::~rmx_graph() {
    timers.destroy();
    for (cudaStream_t a : work.aux)
        if (a) cudaStreamDestroy(a);
    if (work.fork) cudaEventDestroy(work.fork);
    for (cudaEvent_t e : work.join)
        if (e) cudaEventDestroy(e);
    hub_arena.destroy();
    agg_arena.destroy();
    for (SweepGraph &g : sweep_graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    for (StageGraph &g : stage_graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    perm.destroy();
    scratch.destroy();
    if (stream) cudaStreamDestroy(stream);
}

// Copy k of a graph: its node range starts at noff[k], its links at lbase[k];
// both ends of every link are shifted from the canonical copy's numbering
// (nodes from cbase[k]). Offsets: one entry per node plus the final one.
__global__ void k_replicate_csr(int32_t K, const int64_t *noff, const int64_t *cbase, const int64_t *lbase,
                                const int64_t *c_off, const int32_t *c_adj, const double *c_w, int64_t *off,
                                int32_t *adj, double *w) {
    for (int32_t k = blockIdx.x; k < K; k += gridDim.x) {
        const int64_t nb = noff[k], nn = noff[k + 1] - nb, cb = cbase[k], lb = lbase[k];
        const int64_t c0 = c_off[cb], cl = c_off[cb + nn] - c0;
        const int64_t shift = nb - cb;
        for (int64_t i = threadIdx.x; i < nn; i += blockDim.x) off[nb + i] = lb + (c_off[cb + i] - c0);
        for (int64_t j = threadIdx.x; j < cl; j += blockDim.x) {
            adj[lb + j] = (int32_t)(c_adj[c0 + j] + shift);
            w[lb + j] = c_w[c0 + j];
        }
        if (k == K - 1 && threadIdx.x == 0) off[nb + nn] = lb + cl;
    }
}

static void replicate_csr(int32_t K, const int64_t *noff, const int64_t *cbase, const int64_t *lbase,
                          const int64_t *c_off, const int32_t *c_adj, const double *c_w, int64_t *off, int32_t *adj,
                          double *w, cudaStream_t s) {
    k_replicate_csr<<<std::min(K, num_sms() * 16), 256, 0, s>>>(K, noff, cbase, lbase, c_off, c_adj, c_w, off, adj,
                                                                 w);
    RMX_LAUNCHED();
}

void rmx_graph::create(const int32_t *src, const int32_t *dst, const double *w, int64_t n_edges, int32_t n,
                       const double *node_weights, const UnionSpec *u) {
    const NvtxRange range("rmx graph build");
    if (n <= 0) throw std::invalid_argument("graph needs at least one node");
    if (n_edges < 0 || (n_edges > 0 && (!src || !dst))) throw std::invalid_argument("edge arrays missing");
    if (n_edges >= (int64_t(1) << 31)) throw std::invalid_argument("more than 2^31-1 input edges");
    const bool repl = u && u->n_canon > 0;  // edges describe the canonical copies only
    const int32_t n_in = repl ? u->n_canon : n;
    {  // endpoints checked on host threads (one below 4M edges), before any device work
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const int T = (int)std::min<int64_t>(std::min(hw, 16u), std::max<int64_t>(1, n_edges >> 22));
        std::vector<uint8_t> bad(std::max(T, 1), 0);
        rmx::run_parallel(T, [&](int t) {
            const int64_t e0 = n_edges * t / T, e1 = n_edges * (t + 1) / T;
            bool b = false;
            for (int64_t e = e0; e < e1; e++)
                b |= ((uint32_t)src[e] >= (uint32_t)n_in) | ((uint32_t)dst[e] >= (uint32_t)n_in);
            bad[t] = b;
        });
        for (uint8_t b : bad)
            if (b) throw std::invalid_argument("edge endpoint outside 0..N-1");
    }
    N = n;
    tot_w = (double)n;  // FileIO.cpp:229: every node weighs 1 unless the file gives weights
    if (node_weights) {
        node_w.assign(node_weights, node_weights + n);
        tot_w = 0.0;
        for (int32_t i = 0; i < n; i++) tot_w += node_weights[i];
    }
    if (u) {  // a disjoint union of instances: node ranges, canonical copies
        if (u->K < 1 || (int64_t)u->inst_noff[u->K] != n || u->inst_noff[0] != 0)
            throw std::invalid_argument("instance node ranges do not cover the graph");
        K = u->K;
        inst_noff.assign(u->inst_noff, u->inst_noff + K + 1);
        inst_canon.assign(u->inst_canon, u->inst_canon + K);
    }
    RMX_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    configure_eval_kernels();
    // input edges, and an upper bound on the kept links of the whole union
    const int64_t Ein = std::max<int64_t>(n_edges, 1), Eb = std::max<int64_t>(repl ? u->full_edges : n_edges, 1);
    scratch.init((size_t)(88 * Eb + 24 * (int64_t)n + 40 * (int64_t)K) + (64u << 20));
    // long-lived arrays: node CSR/CSC, three levels, module and instance state
    perm.init((size_t)(156 * Eb + 696 * (int64_t)n + (K > 1 ? 16 * (int64_t)n + 64 * (int64_t)K : 0)) + (64u << 20));
    out_off = perm.alloc<int64_t>(n + 1);
    in_off = perm.alloc<int64_t>(n + 1);
    int32_t *d_src = scratch.alloc<int32_t>(Ein), *d_dst = scratch.alloc<int32_t>(Ein);
    double *d_w = scratch.alloc<double>(Ein);
    if (n_edges > 0) {
        RMX_CUDA(cudaMemcpyAsync(d_src, src, sizeof(int32_t) * n_edges, cudaMemcpyHostToDevice, stream));
        RMX_CUDA(cudaMemcpyAsync(d_dst, dst, sizeof(int32_t) * n_edges, cudaMemcpyHostToDevice, stream));
        if (w)
            RMX_CUDA(cudaMemcpyAsync(d_w, w, sizeof(double) * n_edges, cudaMemcpyHostToDevice, stream));
        else {
            k_fill<<<blocks_for(n_edges, 256, 4096), 256, 0, stream>>>(d_w, n_edges, 1.0);
            RMX_LAUNCHED();
        }
    }
    // kept links <= input edges: size link arrays by the input count
    out_dst = perm.alloc<int32_t>(Eb);
    out_w0 = perm.alloc<double>(Eb);
    in_src = perm.alloc<int32_t>(Eb);
    in_w = perm.alloc<double>(Eb);
    dtmp = perm.alloc<int64_t>(16);
    if (!repl) {
        CsrBuild cb = build_csr(n, n_edges, d_src, d_dst, d_w, out_off, out_dst, out_w0, in_off, in_src, in_w,
                                scratch, stream, dtmp);
        E = cb.n_links;
        n_self = cb.n_self;
    } else {
        // CSR/CSC of the canonical copies, then every copy written from its canonical one
        const int32_t nc = u->n_canon;
        int64_t *c_out_off = scratch.alloc<int64_t>(nc + 1), *c_in_off = scratch.alloc<int64_t>(nc + 1);
        int32_t *c_out_dst = scratch.alloc<int32_t>(Ein), *c_in_src = scratch.alloc<int32_t>(Ein);
        double *c_out_w = scratch.alloc<double>(Ein), *c_in_w = scratch.alloc<double>(Ein);
        CsrBuild cb = build_csr(nc, n_edges, d_src, d_dst, d_w, c_out_off, c_out_dst, c_out_w, c_in_off, c_in_src,
                                c_in_w, scratch, stream, dtmp);
        std::vector<int64_t> hoff(nc + 1);
        RMX_CUDA(cudaMemcpyAsync(hoff.data(), c_out_off, sizeof(int64_t) * (nc + 1), cudaMemcpyDeviceToHost, stream));
        RMX_CUDA(cudaStreamSynchronize(stream));
        // per instance: canonical node base and union link base (links of a copy = its canonical copy's)
        std::vector<int64_t> cbase(K), lbase(K + 1, 0);
        std::vector<int64_t> canon_node(K, -1);
        int64_t nb = 0;
        for (int32_t k = 0; k < K; k++)
            if (inst_canon[k] == k) {
                canon_node[k] = nb;
                nb += inst_noff[k + 1] - inst_noff[k];
            }
        if (nb != nc) throw std::invalid_argument("canonical copies do not match the canonical node count");
        for (int32_t k = 0; k < K; k++) {
            cbase[k] = canon_node[inst_canon[k]];
            const int64_t sz = inst_noff[k + 1] - inst_noff[k];
            lbase[k + 1] = lbase[k] + hoff[cbase[k] + sz] - hoff[cbase[k]];
        }
        if (lbase[K] > Eb) throw std::invalid_argument("union link bound too small");
        int64_t *d_cbase = scratch.alloc<int64_t>(K), *d_lbase = scratch.alloc<int64_t>(K + 1),
                *d_noff = scratch.alloc<int64_t>(K + 1);
        RMX_CUDA(cudaMemcpyAsync(d_cbase, cbase.data(), sizeof(int64_t) * K, cudaMemcpyHostToDevice, stream));
        RMX_CUDA(cudaMemcpyAsync(d_lbase, lbase.data(), sizeof(int64_t) * (K + 1), cudaMemcpyHostToDevice, stream));
        RMX_CUDA(cudaMemcpyAsync(d_noff, inst_noff.data(), sizeof(int64_t) * (K + 1), cudaMemcpyHostToDevice, stream));
        replicate_csr(K, d_noff, d_cbase, d_lbase, c_out_off, c_out_dst, c_out_w, out_off, out_dst, out_w0, stream);
        replicate_csr(K, d_noff, d_cbase, d_lbase, c_in_off, c_in_src, c_in_w, in_off, in_src, in_w, stream);
        E = lbase[K];
        n_self = cb.n_self;
    }
    scratch.release(0);
    const int64_t Em = std::max<int64_t>(E, 1);
    out_f = perm.alloc<double>(Em);
    out_fx = perm.alloc<fx_t>(Em);
    in_fx = perm.alloc<fx_t>(Em);
    tw = perm.alloc<double>(n);
    p = perm.alloc<double>(n);
    dangling = perm.alloc<uint8_t>(n);
    // teleport weights w_i / sum w (OmpRelaxmap.cpp:113-115), within every instance of a union
    if (K == 1 && !node_weights) {
        k_fill<<<blocks_for(n, 256, 4096), 256, 0, stream>>>(tw, n, 1.0 / tot_w);
        RMX_LAUNCHED();
    } else {
        std::vector<double> twh(n);
        auto nw = [&](int64_t i) { return node_weights ? node_w[i] : 1.0; };
        if (K == 1) {
            for (int32_t i = 0; i < n; i++) twh[i] = nw(i) / tot_w;
        } else {
            for (int32_t k = 0; k < K; k++) {
                double t = node_weights ? 0.0 : (double)(inst_noff[k + 1] - inst_noff[k]);
                if (node_weights)
                    for (int64_t i = inst_noff[k]; i < inst_noff[k + 1]; i++) t += node_w[i];
                for (int64_t i = inst_noff[k]; i < inst_noff[k + 1]; i++) twh[i] = nw(i) / t;
            }
        }
        RMX_CUDA(cudaMemcpyAsync(tw, twh.data(), sizeof(double) * n, cudaMemcpyHostToDevice, stream));
        RMX_CUDA(cudaStreamSynchronize(stream));  // twh is a local pageable buffer
    }
    nattr = perm.alloc<Stat4>(n);
    nmod = perm.alloc<int32_t>(n);
    zeros = perm.alloc<int32_t>(n);
    node_sn = perm.alloc<int32_t>(n);
    best_part = perm.alloc<int32_t>(n);
    submod = perm.alloc<int32_t>(n);
    s0 = perm.alloc<fx_t>(1);
    RMX_CUDA(cudaMemsetAsync(zeros, 0, sizeof(int32_t) * n, stream));
    if (K > 1) {
        node_inst = perm.alloc<int32_t>(n);
        RMX_CUDA(cudaMemcpyAsync(node_inst, u->node_inst, sizeof(int32_t) * n, cudaMemcpyHostToDevice, stream));
    }
    alloc_engine();
    RMX_CUDA(cudaStreamSynchronize(stream));
    // SpMV sub-warp width from the mean in-degree
    const double avg = (double)E / n;
#ifdef RMX_SPMV_VEC
    spmv_vec = RMX_SPMV_VEC;  // a build option for timing other widths
#else
    spmv_vec = spmv_width(avg);
#endif
}

void rmx_graph::alloc_engine() {
    const int32_t n = N;
    const int64_t Em = std::max<int64_t>(E, 1);
    node_lv.n = n;
    node_lv.m = E;
    node_lv.out_off = out_off;
    node_lv.in_off = in_off;
    node_lv.out_dst = out_dst;
    node_lv.in_src = in_src;
    node_lv.out_fx = out_fx;
    node_lv.in_fx = in_fx;
    node_lv.attr = nattr;
    node_lv.mod = nmod;
    node_lv.inst = K > 1 ? node_inst : zeros;
    node_lv.nnodes = nullptr;
    node_lv.out_src = perm.alloc<int32_t>(Em);  // the coarsening reads every link's row
    if (E > 0) rows_of_links(n, out_off, node_lv.out_src, stream);
    for (Level &lv : sn_buf) lv.out_src = perm.alloc<int32_t>(Em);
    for (Level *lv : {&sn_buf[0], &sn_buf[1], &sub_lv}) {
        lv->out_off = perm.alloc<int64_t>(n + 1);
        lv->in_off = perm.alloc<int64_t>(n + 1);
        lv->out_dst = perm.alloc<int32_t>(Em);
        lv->in_src = perm.alloc<int32_t>(Em);
        lv->out_fx = perm.alloc<fx_t>(Em);
        lv->in_fx = perm.alloc<fx_t>(Em);
        lv->attr = perm.alloc<Stat4>(n);
        lv->nnodes = perm.alloc<int32_t>(n);
    }
    for (Level &lv : sn_buf) {
        lv.mod = perm.alloc<int32_t>(n);
        lv.inst = K > 1 ? perm.alloc<int32_t>(n) : zeros;
    }
    sub_lv.mod = submod;
    sub_lv.inst = nmod;  // instance of a node in coarse-tune = its parent module
    sub_lv.nnodes = nullptr;
    for (ModState *M : {&mods, &submods}) {
        M->cap = n;
        M->stat = perm.alloc<Stat4>(n);
        M->term = perm.alloc<double2>(n);
        M->rec = perm.alloc<ModRec>(n);
        M->count = perm.alloc<int32_t>(n);
        M->inst = perm.alloc<int32_t>(n);
    }
    inst1.n = K;
    instsub.n = n;
    for (InstState *I : {&inst1, &instsub}) {
        const int32_t k = I->n;
        I->sum_exit = perm.alloc<double>(k);
        I->L = perm.alloc<double>(k);
        I->L_prev = perm.alloc<double>(k);
        I->s0 = perm.alloc<fx_t>(k);
        I->acc = perm.alloc<fx_t>(3 * (int64_t)k);
        I->active = perm.alloc<uint8_t>(k);
    }
    if (K == 1) inst1.s0 = s0;
    work.list = perm.alloc<int32_t>(n);
    work.list2 = perm.alloc<int32_t>(n);
    work.bucket = perm.alloc<uint16_t>(n);
    work.bucket_off = perm.alloc<int64_t>(260);
    work.ranges = perm.alloc<int64_t>(2 * 37);
    work.prop = perm.alloc<int32_t>(n);
    work.pdelta = perm.alloc<double>(n);
    work.ptarget = perm.alloc<int32_t>(n);
    work.prevmod = perm.alloc<int32_t>(n);
    work.stamp = perm.alloc<uint32_t>(n);
    work.next_active = perm.alloc<uint8_t>(n);
    work.free_list = perm.alloc<int32_t>(n);
    work.claim = perm.alloc<unsigned long long>(n);
    work.counters = perm.alloc<int64_t>(kCntSlots);
    work.dparams = perm.alloc<uint32_t>(64);
    timers.logcap = 8192;
    timers.dlog = perm.alloc<int64_t>(Timers::kLogWords * timers.logcap);
    stage_ctl = perm.alloc<int64_t>(8);
    stage_seed = perm.alloc<uint32_t>(8);
    stage_sweeping = perm.alloc<uint8_t>(std::max(K, 1));
    stage_oldL = perm.alloc<double>(std::max(K, 1));
    RMX_CUDA(cudaMemsetAsync(work.stamp, 0, sizeof(uint32_t) * n, stream));
    RMX_CUDA(cudaMemsetAsync(work.claim, 0, sizeof(unsigned long long) * n, stream));
    RMX_CUDA(cudaMemsetAsync(work.next_active, 0, n, stream));
    RMX_CUDA(cudaMemsetAsync(work.counters, 0, sizeof(int64_t) * kCntSlots, stream));
    // the hub pipeline's stream (aux[4]) at the highest priority: its chain of
    // dependent kernels is the longest of a sub-batch, so its blocks go first
    // whenever the other bins' blocks leave an SM
    int prio_low = 0, prio_high = 0;
    RMX_CUDA(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
    for (int k = 0; k < 5; k++)
        RMX_CUDA(cudaStreamCreateWithPriority(&work.aux[k], cudaStreamNonBlocking, k == 4 ? prio_high : prio_low));
    RMX_CUDA(cudaEventCreateWithFlags(&work.fork, cudaEventDisableTiming));
    for (cudaEvent_t &e : work.join) RMX_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
}

int64_t rmx_graph::max_degree(const Level &lv) {
    unsigned long long *mx = reinterpret_cast<unsigned long long *>(dtmp + 8);
    RMX_CUDA(cudaMemsetAsync(mx, 0, 8, stream));
    k_max_degree<<<blocks_for(lv.n, 256, num_sms() * 8), 256, 0, stream>>>(lv.n, lv.out_off, lv.in_off, mx);
    RMX_LAUNCHED();
    unsigned long long h = 0;
    RMX_CUDA(cudaMemcpyAsync(&h, mx, 8, cudaMemcpyDeviceToHost, stream));
    RMX_CUDA(cudaStreamSynchronize(stream));
    return (int64_t)h;
}

// The hub pipeline's plan, partition and bucket arrays, sized for every unit
// of lv above the large bin's bound (any sub-batch of the level fits); grown,
// never shrunk.
void rmx_graph::ensure_hub_table(const Level &lv) {
    if (lv.n <= 0) return;
    int64_t need[4];
    hub_level_needs(lv, need, dtmp + 12, stream);
    const int64_t units = need[0], parts = need[1], links = need[2], chunks = need[3];
    if (units == 0 || (units <= work.hub_units && parts <= work.hub_parts && links <= work.hub_links &&
                       chunks <= work.hub_chunks))
        return;
    RMX_CUDA(cudaStreamSynchronize(stream));  // no launch still reads the old arrays
    hub_arena.destroy();
    const int64_t U = std::max(units, work.hub_units) * 5 / 4 + 16, P = std::max(parts, work.hub_parts) * 5 / 4 + 64,
                  Lk = std::max(links, work.hub_links) * 5 / 4 + 1024,
                  C = std::max(chunks, work.hub_chunks) * 5 / 4 + 64;
    work.hub_units = work.hub_parts = work.hub_links = work.hub_chunks = 0;
    work.hub_bkey = work.hub_lkey = nullptr;
    const size_t bytes = (size_t)Lk * (2 * sizeof(int32_t) + sizeof(fx_t)) + (size_t)(U + 1) * 3 * sizeof(int64_t) +
                         (size_t)U * (2 * sizeof(fx_t) + sizeof(int32_t) + 1) +
                         (size_t)P * (sizeof(unsigned long long) + sizeof(double) + sizeof(int32_t)) +
                         (size_t)(P + 1) * sizeof(int64_t) + (size_t)(C + P) * sizeof(int32_t) + 16 * 256;
    hub_arena.init(bytes);
    work.hub_bfx = hub_arena.alloc<fx_t>(Lk);
    work.hub_bkey = hub_arena.alloc<int32_t>(Lk);
    work.hub_lkey = hub_arena.alloc<int32_t>(Lk);
    work.hub_coff = hub_arena.alloc<int64_t>(U + 1);
    work.hub_poff = hub_arena.alloc<int64_t>(U + 1);
    work.hub_loff = hub_arena.alloc<int64_t>(U + 1);
    work.hub_own = hub_arena.alloc<fx_t>(U);
    work.hub_nparts = hub_arena.alloc<int32_t>(U);
    work.hub_act = hub_arena.alloc<uint8_t>(U);
    work.hub_pcnt = hub_arena.alloc<unsigned long long>(P);
    work.hub_best = hub_arena.alloc<double>(P);
    work.hub_pstart = hub_arena.alloc<int64_t>(P + 1);
    work.hub_bmod = hub_arena.alloc<int32_t>(P);
    work.hub_tot = hub_arena.alloc<int64_t>(8);
    work.hub_cunit = hub_arena.alloc<int32_t>(C);
    work.hub_punit = hub_arena.alloc<int32_t>(P);
    work.hub_units = U;
    work.hub_parts = P;
    work.hub_links = Lk;
    work.hub_chunks = C;
    work.hub_gen++;
}

void rmx_graph::initiate() {
    if (initiated) return;
    const NvtxRange range("rmx flow");
    timers.begin(kTimerOther, stream);
    // the CSC weights are normalised in place, once; the CSR flows are rebuilt from the raw weights
    normalise(N, out_off, out_w0, out_f, in_off, in_src, in_w, in_w, dangling, scratch, stream, !cols_normalised);
    cols_normalised = true;
    timers.end(kTimerOther, stream);
    timers.begin(kTimerSpmv, stream);
    if (K == 1)
        power_iters = power_iteration(N, in_off, in_src, in_w, tw, dangling, p, scratch, stream, spmv_vec);
    else
        power_iters = union_flows();
    timers.end(kTimerSpmv, stream);
    timers.begin(kTimerOther, stream);
    edge_flows(N, E, out_off, out_f, out_fx, in_src, in_w, in_fx, p, tw, dangling, nattr, s0, stream);
    if (K > 1) {  // sum p log p of every instance's nodes
        RMX_CUDA(cudaMemsetAsync(inst1.s0, 0, sizeof(fx_t) * K, stream));
        k_sub_s0<<<blocks_for(N, 256, num_sms() * 32), 256, 0, stream>>>(N, p, node_inst, inst1.s0);
        RMX_LAUNCHED();
    }
    timers.end(kTimerOther, stream);
    init_singletons(node_lv, mods, stream);
    RMX_CUDA(cudaMemsetAsync(inst1.active, 1, (size_t)K, stream));
    instance_codelength(mods, inst1, stream);
    L0v.assign(K, 0.0);
    RMX_CUDA(cudaMemcpyAsync(L0v.data(), inst1.L, sizeof(double) * K, cudaMemcpyDeviceToHost, stream));
    RMX_CUDA(cudaStreamSynchronize(stream));
    L0 = L0v[0];
    ensure_hub_table(node_lv);
    initiated = true;
}

// Flows of a disjoint union: each canonical instance (the first copy of a
// graph) iterated on its own, the other copies sharing its flow.
int rmx_graph::union_flows() {
    std::vector<int64_t> comp;
    for (int32_t k = 0; k < K; k++)
        if (inst_canon[k] == k) {
            comp.push_back(inst_noff[k]);
            comp.push_back(inst_noff[k + 1]);
        }
    const int32_t nc = (int32_t)(comp.size() / 2);
    size_t mk = scratch.mark();
    int64_t *d_comp = scratch.alloc<int64_t>(comp.size()), *d_noff = scratch.alloc<int64_t>(K + 1);
    int32_t *d_canon = scratch.alloc<int32_t>(K);
    RMX_CUDA(cudaMemcpyAsync(d_comp, comp.data(), sizeof(int64_t) * comp.size(), cudaMemcpyHostToDevice, stream));
    RMX_CUDA(cudaMemcpyAsync(d_noff, inst_noff.data(), sizeof(int64_t) * (K + 1), cudaMemcpyHostToDevice, stream));
    RMX_CUDA(cudaMemcpyAsync(d_canon, inst_canon.data(), sizeof(int32_t) * K, cudaMemcpyHostToDevice, stream));
    const int it = power_iteration_components(N, nc, d_comp, node_inst, d_noff, d_canon, in_off, in_src, in_w, tw,
                                              dangling, p, scratch, stream, spmv_vec);
    scratch.release(mk);
    return it;
}

// ---------------------------------------------------------------- sweeps

// Buckets the active units of lv into ns sub-batches and runs them. From the
// handle's second run on (capture and instantiation cost more than one run's
// launches save), and without profiling, the sub-batch pipeline (about ten
// launches per sub-batch over five streams) is one CUDA graph, captured once
// per (level, module state, instances, sweep options) and replayed: the
// sub-batches' stamps and hash seeds live in device memory, and every kernel
// reads its unit range there. Otherwise the kernels are launched one by one,
// empty bins skipped and grids fitted to the bin sizes.
void rmx_graph::run_subbatches(Level &lv, int64_t n_active, ModState &M, InstState &I, const SweepArgs &sa, int ns,
                               bool mark, uint32_t seed) {
    // a single run on a handle is cheaper launched directly than captured: graphs
    // start with the handle's second attempt / optimiser run
    const bool graphs = !timers.on && use_graphs && runs_done > 0;
    if (timers.on) {  // non-empty modules, for the evaluation's byte accounting
        RMX_CUDA(cudaMemsetAsync(work.counters + kCntMods, 0, sizeof(int64_t), stream));
        k_count_nonzero<<<blocks_for(M.cap, 256, num_sms() * 8), 256, 0, stream>>>(
            M.cap, M.count, reinterpret_cast<unsigned long long *>(work.counters + kCntMods));
        RMX_LAUNCHED();
    }
    bucket_units(lv, work, n_active, seed, ns, scratch, stream, !graphs);
    for (int sb = 0; sb < ns; sb++) {
        work.hparams[2 * sb] = ++stamp;
        work.hparams[2 * sb + 1] = mix_seed(seed, sb);
    }
    // from pageable memory: staged before the call returns, so hparams is free again at once
    RMX_CUDA(cudaMemcpyAsync(work.dparams, work.hparams, sizeof(uint32_t) * 2 * ns, cudaMemcpyHostToDevice, stream));
    if (!graphs) {
        Timers *tm = timers.on ? &timers : nullptr;
        for (int sb = 0; sb < ns; sb++)
            sweep_subbatch(lv, M, I, work, sa, sb, work.dparams + 2 * sb, mark, true, stream, tm);
        return;
    }
    const SweepGraphKey key{&lv, &M, &I, sa.allow_new, mark ? 1 : 0, sa.vthresh, ns, work.hub_gen,
                            eval_tuning_generation()};
    SweepGraph *gr = nullptr;
    for (SweepGraph &g : sweep_graphs)
        if (g.key == key) gr = &g;
    if (!gr) {
        // graphs captured under another launch tuning are never launched again
        bool stale = false;
        for (const SweepGraph &g : sweep_graphs) stale |= g.key.tuning_gen != key.tuning_gen;
        if (stale) {
            RMX_CUDA(cudaStreamSynchronize(stream));  // none of them is still running
            std::vector<SweepGraph> keep;
            for (SweepGraph &g : sweep_graphs) {
                if (g.key.tuning_gen == key.tuning_gen)
                    keep.push_back(g);
                else if (g.exec)
                    cudaGraphExecDestroy(g.exec);
            }
            sweep_graphs.swap(keep);
        }
        const unsigned long long c0 = __atomic_load_n(&g_kernel_launches, __ATOMIC_RELAXED);
        cudaGraph_t graph = nullptr;
        RMX_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        try {
            for (int sb = 0; sb < ns; sb++)
                sweep_subbatch(lv, M, I, work, sa, sb, work.dparams + 2 * sb, mark, false, stream, nullptr);
        } catch (...) {
            cudaStreamEndCapture(stream, &graph);
            if (graph) cudaGraphDestroy(graph);
            throw;
        }
        RMX_CUDA(cudaStreamEndCapture(stream, &graph));
        const unsigned long long c1 = __atomic_load_n(&g_kernel_launches, __ATOMIC_RELAXED);
        __atomic_fetch_sub(&g_kernel_launches, c1 - c0, __ATOMIC_RELAXED);  // counted when replayed
        cudaGraphExec_t exec = nullptr;
        const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        RMX_CUDA(e);
        sweep_graphs.push_back({key, exec, c1 - c0});
        gr = &sweep_graphs.back();
    }
    RMX_CUDA(cudaGraphLaunch(gr->exec, stream));
    __atomic_fetch_add(&g_kernel_launches, gr->kernels, __ATOMIC_RELAXED);
}

// Uploads which instances take part in the next sweeps (their units are
// evaluated; the others keep their modules).
void rmx_graph::set_active(const std::vector<uint8_t> &m) {
    if (K == 1)
        RMX_CUDA(cudaMemsetAsync(inst1.active, m[0], 1, stream));
    else  // staged from pageable memory before the call returns
        RMX_CUDA(cudaMemcpyAsync(inst1.active, m.data(), (size_t)K, cudaMemcpyHostToDevice, stream));
}

void rmx_graph::sweep_single(Level &lv, bool prior, bool allow_new, double vthresh, int64_t &n_active,
                             std::vector<double> &L) {
    RMX_CUDA(cudaMemsetAsync(work.counters + kCntMoved, 0, sizeof(int64_t), stream));
    if (prior) RMX_CUDA(cudaMemsetAsync(work.next_active, 0, lv.n, stream));
    if (allow_new) free_modules(mods, work, scratch, stream);
    const uint32_t seed = mix_seed(run_seed, ++sweep_no);
    const int ns = sub_batches_for(n_active);
    SweepArgs sa{vthresh, allow_new ? 1 : 0};
    run_subbatches(lv, n_active, mods, inst1, sa, ns, prior, seed);
    timers.begin(kTimerCodelen, stream);
    instance_codelength(mods, inst1, stream);
    timers.end(kTimerCodelen, stream);
    if (prior) compact_flags(work.next_active, lv.n, work.list, work.counters + kCntActive, scratch, stream);
    int64_t cnt[kCntSlots];
    RMX_CUDA(cudaMemcpyAsync(L.data(), inst1.L, sizeof(double) * K, cudaMemcpyDeviceToHost, stream));
    RMX_CUDA(cudaMemcpyAsync(cnt, work.counters, sizeof(cnt), cudaMemcpyDeviceToHost, stream));
    RMX_CUDA(cudaStreamSynchronize(stream));
    prof.sweeps++;
    if (prior) n_active = cnt[kCntActive];
    if (opt.verbose >= 2)
        printf("  sweep: n=%d active=%lld code length = %.17g, moved %lld\n", lv.n, (long long)n_active, L[0] / kLn2,
               (long long)cnt[kCntMoved]);
}

static bool any_set(const std::vector<uint8_t> &m) {
    for (uint8_t v : m)
        if (v) return true;
    return false;
}

// The first loop of stochastic_greedy_partition (OmpRelaxmap.cpp:291-339), or
// the inner super-node loop (:379-411): at most max_iter sweeps, stop when a
// sweep gains less than threshold bits (and did not lose).
//
// Every instance (one graph, or one graph-attempt copy of a batch) follows
// these rules on its own code length; an instance that stops keeps its
// modules while the others continue.
void rmx_graph::stage_sweeps(Level &lv, bool allow_new, std::vector<double> &L, const std::vector<uint8_t> &act) {
    const NvtxRange range(&lv == &node_lv ? "rmx sweeps: nodes" : "rmx sweeps: super-nodes");
    const bool prior = opt.prior != 0;
    const double vthresh = prior ? -opt.vthresh : 0.0;  // OmpRelaxmap.cpp:66, Module.cpp:1490 vs :1127
    int64_t n_active = lv.n;
    all_units(lv.n, work, stream);
    if (lv.n > 0) ensure_hub_table(lv);
    if (stage_graph_ok(lv)) {
        stage_sweeps_graph(lv, allow_new, L, act);
        return;
    }
    std::vector<uint8_t> sweeping = act;
    std::vector<double> oldL;
    const int lvt = &lv == &node_lv ? kTimerLvNode : kTimerLvSN;
    timers.begin(lvt, stream);
    int iter = 0;
    while (any_set(sweeping) && iter < opt.max_iter) {
        oldL = L;
        if (!prior && iter > 0) {
            all_units(lv.n, work, stream);
            n_active = lv.n;
        }
        set_active(sweeping);
        sweep_single(lv, prior, allow_new, vthresh, n_active, L);
        iter++;
        for (int32_t k = 0; k < K; k++)
            if (sweeping[k] && oldL[k] - L[k] >= 0 && (oldL[k] - L[k]) / kLn2 < opt.threshold) sweeping[k] = 0;
    }
    timers.end(lvt, stream);
}

// The stage loop runs as one captured graph once the handle has completed a
// run (as the sweep pipelines: on a small graph capture costs more than one
// cold run saves), or from the first run of a union of instances (a batch
// wave, whose many sweeps each save a host round trip) or of a graph of at
// least 2^22 links (a few captures are small next to its run); never with
// profiling events or per-sweep printing.
bool rmx_graph::stage_graph_ok(const Level &lv) const {
    return use_graphs && (runs_done > 0 || K > 1 || E >= (int64_t(1) << 22)) && !timers.on && opt.verbose < 2 &&
           lv.n > 0;
}

// One sweep of stage_sweeps as the body of the while node: the host loop's
// sweep_single with every size and seed read on the device, then its stop
// rule. cond: the while node's condition handle.
void rmx_graph::stage_body(Level &lv, bool allow_new, bool prior, double vthresh, int ns, unsigned long long cond) {
    const int64_t *n_dev = stage_ctl + 5;
    k_stage_begin<<<blocks_for(K, 256, num_sms() * 4), 256, 0, stream>>>(stage_ctl, stage_seed, ns, work.dparams, K,
                                                                         stage_sweeping, inst1.active, inst1.L,
                                                                         stage_oldL);
    RMX_LAUNCHED();
    if (!prior) all_units_dev(n_dev, N, work, stream);  // normal mode: every sweep takes all units
    RMX_CUDA(cudaMemsetAsync(work.counters + kCntMoved, 0, sizeof(int64_t), stream));
    if (prior) RMX_CUDA(cudaMemsetAsync(work.next_active, 0, (size_t)N, stream));
    if (allow_new) free_modules(mods, work, scratch, stream);
    bucket_units_dev(lv, work, N, stage_seed, ns, scratch, stream);
    SweepArgs sa{vthresh, allow_new ? 1 : 0};
    for (int sb = 0; sb < ns; sb++)
        sweep_subbatch(lv, mods, inst1, work, sa, sb, work.dparams + 2 * sb, prior, false, stream, nullptr);
    instance_codelength(mods, inst1, stream);
    if (prior) compact_flags_dev(work.next_active, n_dev, N, work.list, work.counters + kCntActive, scratch, stream);
    k_stage_stop<<<blocks_for(K, 256, num_sms() * 4), 256, 0, stream>>>(
        K, inst1.L, stage_oldL, stage_sweeping, opt.threshold, kLn2,
        reinterpret_cast<unsigned long long *>(stage_ctl + 4));
    RMX_LAUNCHED();
    k_stage_cond<<<1, 1, 0, stream>>>(stage_ctl, opt.max_iter, (cudaGraphConditionalHandle)cond);
    RMX_LAUNCHED();
}

void rmx_graph::stage_sweeps_graph(Level &lv, bool allow_new, std::vector<double> &L,
                                   const std::vector<uint8_t> &act) {
    const bool prior = opt.prior != 0;
    const double vthresh = prior ? -opt.vthresh : 0.0;  // OmpRelaxmap.cpp:66, Module.cpp:1490 vs :1127
    if (!any_set(act) || opt.max_iter <= 0) return;
    const int ns = sub_batches_for(lv.n);
    const StageGraphKey key{&lv,          &mods, &inst1,   allow_new ? 1 : 0, prior ? 1 : 0,
                            opt.max_iter, ns,    vthresh,  opt.threshold,     work.hub_gen,
                            eval_tuning_generation(), scratch.mark()};
    RMX_CUDA(cudaMemcpyAsync(stage_sweeping, act.data(), (size_t)K, cudaMemcpyHostToDevice, stream));
    loop_graph(key, lv.n, [&](unsigned long long cond) { stage_body(lv, allow_new, prior, vthresh, ns, cond); });
    RMX_CUDA(cudaMemcpyAsync(L.data(), inst1.L, sizeof(double) * K, cudaMemcpyDeviceToHost, stream));
    RMX_CUDA(cudaStreamSynchronize(stream));
}

// One sweep of the coarse-tune sub-problems (generate_sub_modules) as the
// body of the while node, and their stop rule (k_inst_stop) on the device.
void rmx_graph::subtune_body(int ns, unsigned long long cond) {
    k_stage_begin<<<1, 32, 0, stream>>>(stage_ctl, stage_seed, ns, work.dparams, 0, nullptr, nullptr, nullptr,
                                        nullptr);
    RMX_LAUNCHED();
    all_units_dev(stage_ctl + 5, N, work, stream);
    bucket_units_dev(sub_lv, work, N, stage_seed, ns, scratch, stream);
    SweepArgs sa{0.0, 0};  // Network::move: best < 0, no empty module (Module.cpp:606, :667)
    for (int sb = 0; sb < ns; sb++)
        sweep_subbatch(sub_lv, submods, instsub, work, sa, sb, work.dparams + 2 * sb, false, false, stream, nullptr);
    instance_codelength(submods, instsub, stream);
    k_inst_stop<<<blocks_for(N, 256, num_sms() * 8), 256, 0, stream>>>(
        N, instsub.L, instsub.L_prev, instsub.active, opt.threshold, kLn2,
        reinterpret_cast<unsigned long long *>(stage_ctl + 4));
    RMX_LAUNCHED();
    k_stage_cond<<<1, 1, 0, stream>>>(stage_ctl, opt.max_iter, (cudaGraphConditionalHandle)cond);
    RMX_LAUNCHED();
}

// Runs a loop of sweeps as one graph: captured once per key (a while node
// whose body `body` enqueues, given the node's condition handle), launched
// with the host's sweep number, stamp and attempt seed and the level's size
// in stage_ctl, which come back with the number of sweeps run.
void rmx_graph::loop_graph(const StageGraphKey &key, int64_t n_level,
                           const std::function<void(unsigned long long)> &body) {
    StageGraph *gr = nullptr;
    for (StageGraph &g : stage_graphs)
        if (g.key == key) gr = &g;
    if (!gr) {
        bool stale = false;  // graphs captured under another launch tuning are never launched again
        for (const StageGraph &g : stage_graphs) stale |= g.key.tuning_gen != key.tuning_gen;
        if (stale) {
            RMX_CUDA(cudaStreamSynchronize(stream));
            std::vector<StageGraph> keep;
            for (StageGraph &g : stage_graphs) {
                if (g.key.tuning_gen == key.tuning_gen)
                    keep.push_back(g);
                else if (g.exec)
                    cudaGraphExecDestroy(g.exec);
            }
            stage_graphs.swap(keep);
        }
        cudaGraph_t graph = nullptr;
        RMX_CUDA(cudaGraphCreate(&graph, 0));
        cudaGraphExec_t exec = nullptr;
        unsigned long long kernels = 0;
        try {
            cudaGraphConditionalHandle cond;
            RMX_CUDA(cudaGraphConditionalHandleCreate(&cond, graph, 1, cudaGraphCondAssignDefault));
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = cond;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t node;
            RMX_CUDA(cudaGraphAddNode(&node, graph, nullptr, 0, &cp));
            cudaGraph_t bg = cp.conditional.phGraph_out[0];
            const unsigned long long c0 = __atomic_load_n(&g_kernel_launches, __ATOMIC_RELAXED);
            RMX_CUDA(cudaStreamBeginCaptureToGraph(stream, bg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
            try {
                body((unsigned long long)cond);
            } catch (...) {
                cudaGraph_t g2 = nullptr;
                cudaStreamEndCapture(stream, &g2);
                throw;
            }
            cudaGraph_t g2 = nullptr;
            RMX_CUDA(cudaStreamEndCapture(stream, &g2));
            const unsigned long long c1 = __atomic_load_n(&g_kernel_launches, __ATOMIC_RELAXED);
            kernels = c1 - c0;
            __atomic_fetch_sub(&g_kernel_launches, kernels, __ATOMIC_RELAXED);  // counted per sweep replayed
            RMX_CUDA(cudaGraphInstantiate(&exec, graph, 0));
        } catch (...) {
            cudaGraphDestroy(graph);
            throw;
        }
        cudaGraphDestroy(graph);
        stage_graphs.push_back({key, exec, kernels});
        gr = &stage_graphs.back();
    }
    // staged from pageable memory: ctl is free again when the copies return
    int64_t ctl[6] = {(int64_t)sweep_no, (int64_t)stamp, (int64_t)run_seed, 0, 0, n_level};
    RMX_CUDA(cudaMemcpyAsync(stage_ctl, ctl, sizeof ctl, cudaMemcpyHostToDevice, stream));
    RMX_CUDA(cudaGraphLaunch(gr->exec, stream));
    RMX_CUDA(cudaMemcpyAsync(ctl, stage_ctl, sizeof ctl, cudaMemcpyDeviceToHost, stream));
    RMX_CUDA(cudaStreamSynchronize(stream));
    sweep_no = (uint64_t)ctl[0];
    stamp = (uint32_t)ctl[1];
    prof.sweeps += ctl[3];
    __atomic_fetch_add(&g_kernel_launches, gr->kernels * (unsigned long long)ctl[3], __ATOMIC_RELAXED);
}

void rmx_graph::project_sn_to_nodes() {
    k_project<<<blocks_for(N, 256, num_sms() * 32), 256, 0, stream>>>(N, node_sn, sn().mod, nmod);
    RMX_LAUNCHED();
}

// convertModulesToSuperNodes (Module.cpp:3008-3077) on the engine's partition.
// The super-node links carry fixed-point flows, whose sums are exact in any
// order, so after a super-node stage the new level is aggregated from the
// current super-node links (a few times fewer than node links) with the same
// result as from the node links.
void rmx_graph::convert_to_supernodes(bool from_sn) {
    const NvtxRange range("rmx coarsen");
    timers.begin(kTimerCoarsen, stream);
    count_units(node_lv, mods, stream);  // nodes per module
    size_t mk = scratch.mark();
    int64_t *snid = scratch.alloc<int64_t>(N + 1);
    k_flags_nonempty<<<blocks_for(N, 256, num_sms() * 32), 256, 0, stream>>>(N, mods.count, snid);
    RMX_LAUNCHED();
    scan_exclusive(snid, snid, N, dtmp + 0, scratch, stream);
    int64_t nsn = 0;
    RMX_CUDA(cudaMemcpyAsync(&nsn, dtmp + 0, sizeof(int64_t), cudaMemcpyDeviceToHost, stream));
    Level &src = sn(), &dst = sn_buf[1 - sn_cur];
    k_sn_from_modules<<<blocks_for(N, 256, num_sms() * 32), 256, 0, stream>>>(
        N, mods.count, snid, mods.stat, K > 1 ? mods.inst : nullptr, dst.mod, dst.attr, dst.nnodes, dst.inst);
    RMX_LAUNCHED();
    int32_t *group = nullptr;
    if (from_sn) {
        group = scratch.alloc<int32_t>(std::max(src.n, 1));
        k_group_of_nodes<<<blocks_for(src.n, 256, num_sms() * 32), 256, 0, stream>>>(src.n, src.mod, snid, group);
        RMX_LAUNCHED();
    }
    k_group_of_nodes<<<blocks_for(N, 256, num_sms() * 32), 256, 0, stream>>>(N, nmod, snid, node_sn);
    RMX_LAUNCHED();
    RMX_CUDA(cudaStreamSynchronize(stream));
    dst.n = (int32_t)nsn;
    if (from_sn)
        dst.m = aggregate_links(src.n, src.out_off, src.out_dst, src.out_fx, src.out_src, group, dst.n, dst.out_off,
                                dst.out_dst, dst.out_fx, dst.out_src, dst.in_off, dst.in_src, dst.in_fx, nullptr,
                                agg_arena, agg_tab, agg_cap, scratch, stream, &work);
    else
        dst.m = aggregate_links(N, out_off, out_dst, out_fx, node_lv.out_src, node_sn, dst.n, dst.out_off, dst.out_dst,
                                dst.out_fx, dst.out_src, dst.in_off, dst.in_src, dst.in_fx, nullptr, agg_arena, agg_tab,
                                agg_cap, scratch, stream, &work);
    scratch.release(mk);
    sn_cur = 1 - sn_cur;
    count_units(sn(), mods, stream);
    timers.end(kTimerCoarsen, stream);
}

// generate_sub_modules (OmpRelaxmap.cpp:502-638): every module becomes an
// independent sub-network of its members and internal links (flows kept),
// optimised by node moves only (partition_module_network with fast=true:
// Network::move semantics, no empty-module option, stop per sub-network);
// the resulting sub-modules become the super-nodes of the next superstep,
// starting in their parent module.
void rmx_graph::generate_sub_modules() {
    const NvtxRange range("rmx coarse-tune");
    timers.begin(kTimerCoarsen, stream);
    count_units(node_lv, mods, stream);  // nodes per parent module
    size_t mk = scratch.mark();
    int64_t *cnt_out = scratch.alloc<int64_t>(N + 1), *cnt_in = scratch.alloc<int64_t>(N + 1);
    const unsigned GW = blocks_for((int64_t)N * 32, 256, num_sms() * 32);
    RMX_CUDA(cudaMemsetAsync(cnt_out + N, 0, sizeof(int64_t), stream));
    RMX_CUDA(cudaMemsetAsync(cnt_in + N, 0, sizeof(int64_t), stream));
    k_intra_count<<<GW, 256, 0, stream>>>(N, out_off, out_dst, nmod, cnt_out);
    RMX_LAUNCHED();
    k_intra_count<<<GW, 256, 0, stream>>>(N, in_off, in_src, nmod, cnt_in);
    RMX_LAUNCHED();
    scan_exclusive(cnt_out, sub_lv.out_off, N + 1, nullptr, scratch, stream);
    scan_exclusive(cnt_in, sub_lv.in_off, N + 1, nullptr, scratch, stream);
    fx_t *intra_out = reinterpret_cast<fx_t *>(cnt_out);  // counts are consumed by the scans above
    k_intra_fill<<<GW, 256, 0, stream>>>(N, out_off, out_dst, out_fx, nmod, sub_lv.out_off, sub_lv.out_dst,
                                         sub_lv.out_fx, intra_out);
    RMX_LAUNCHED();
    k_intra_fill<<<GW, 256, 0, stream>>>(N, in_off, in_src, in_fx, nmod, sub_lv.in_off, sub_lv.in_src, sub_lv.in_fx,
                                         nullptr);
    RMX_LAUNCHED();
    k_sub_attr<<<blocks_for(N, 256, num_sms() * 32), 256, 0, stream>>>(N, nattr, intra_out, sub_lv.attr);
    RMX_LAUNCHED();
    scratch.release(mk);
    sub_lv.n = N;
    RMX_CUDA(cudaMemcpyAsync(&sub_lv.m, sub_lv.out_off + N, sizeof(int64_t), cudaMemcpyDeviceToHost, stream));
    // sub-problem state: singleton sub-modules, per-parent code lengths
    init_singletons(sub_lv, submods, stream);
    RMX_CUDA(cudaMemsetAsync(instsub.s0, 0, sizeof(fx_t) * N, stream));
    k_sub_s0<<<blocks_for(N, 256, num_sms() * 32), 256, 0, stream>>>(N, p, nmod, instsub.s0);
    RMX_LAUNCHED();
    k_inst_active<<<blocks_for(N, 256, num_sms() * 32), 256, 0, stream>>>(N, mods.count, mods.inst, inst1.active,
                                                                          instsub.active);
    RMX_LAUNCHED();
    instance_codelength(submods, instsub, stream);
    k_copy_L<<<blocks_for(N, 256, num_sms() * 32), 256, 0, stream>>>(N, instsub.L, instsub.L_prev);
    RMX_LAUNCHED();
    RMX_CUDA(cudaStreamSynchronize(stream));
    timers.end(kTimerCoarsen, stream);
    if (sub_lv.m > 0) {
        ensure_hub_table(sub_lv);
        Timers *tm = timers.on ? &timers : nullptr;
        SweepArgs sa{0.0, 0};  // Network::move: best < 0, no empty module (Module.cpp:606, :667)
        timers.begin(kTimerLvSub, stream);
        const int nsg = sub_batches_for(N);
        if (stage_graph_ok(sub_lv) && opt.max_iter > 0) {
            const StageGraphKey key{&sub_lv, &submods, &instsub, 0, 0, opt.max_iter, nsg, 0.0, opt.threshold,
                                    work.hub_gen, eval_tuning_generation(), scratch.mark()};
            loop_graph(key, N, [&](unsigned long long cond) { subtune_body(nsg, cond); });
        }
        for (int iter = 0; iter < opt.max_iter && !stage_graph_ok(sub_lv); iter++) {
            all_units(N, work, stream);
            const uint32_t seed = mix_seed(run_seed, ++sweep_no);
            const int ns = sub_batches_for(N);
            run_subbatches(sub_lv, N, submods, instsub, sa, ns, false, seed);
            timers.begin(kTimerCodelen, stream);
            instance_codelength(submods, instsub, stream);
            unsigned long long *na = reinterpret_cast<unsigned long long *>(dtmp + 9);
            RMX_CUDA(cudaMemsetAsync(na, 0, 8, stream));
            k_inst_stop<<<blocks_for(N, 256, num_sms() * 8), 256, 0, stream>>>(
                N, instsub.L, instsub.L_prev, instsub.active, opt.threshold, kLn2, na);
            RMX_LAUNCHED();
            timers.end(kTimerCodelen, stream);
            unsigned long long h = 0;
            RMX_CUDA(cudaMemcpyAsync(&h, na, 8, cudaMemcpyDeviceToHost, stream));
            RMX_CUDA(cudaStreamSynchronize(stream));
            prof.sweeps++;
            if (h == 0) break;
        }
        timers.end(kTimerLvSub, stream);
    }
    // sub-modules -> super-nodes (generateSuperNodesFromSubModules, Module.cpp:3083-3158)
    timers.begin(kTimerCoarsen, stream);
    count_units(sub_lv, submods, stream);
    mk = scratch.mark();
    int64_t *snid = scratch.alloc<int64_t>(N + 1);
    k_flags_nonempty<<<blocks_for(N, 256, num_sms() * 32), 256, 0, stream>>>(N, submods.count, snid);
    RMX_LAUNCHED();
    scan_exclusive(snid, snid, N, dtmp + 0, scratch, stream);
    k_group_of_nodes<<<blocks_for(N, 256, num_sms() * 32), 256, 0, stream>>>(N, submod, snid, node_sn);
    RMX_LAUNCHED();
    int64_t nsn = 0;
    RMX_CUDA(cudaMemcpyAsync(&nsn, dtmp + 0, sizeof(int64_t), cudaMemcpyDeviceToHost, stream));
    RMX_CUDA(cudaStreamSynchronize(stream));
    Level &sl = sn();
    sl.n = (int32_t)nsn;
    RMX_CUDA(cudaMemsetAsync(sl.attr, 0, sizeof(Stat4) * nsn, stream));
    RMX_CUDA(cudaMemsetAsync(sl.nnodes, 0, sizeof(int32_t) * nsn, stream));
    k_sn_from_nodes<<<blocks_for(N, 256, num_sms() * 32), 256, 0, stream>>>(
        N, node_sn, nmod, nattr, K > 1 ? node_inst : nullptr, sl.mod, sl.attr, sl.nnodes, sl.inst);
    RMX_LAUNCHED();
    {
        fx_t *rowsum = scratch.alloc<fx_t>(std::max<int64_t>(nsn, 1));
        sl.m = aggregate_links(N, out_off, out_dst, out_fx, node_lv.out_src, node_sn, sl.n, sl.out_off, sl.out_dst,
                               sl.out_fx, sl.out_src, sl.in_off, sl.in_src, sl.in_fx, rowsum, agg_arena, agg_tab, agg_cap,
                               scratch, stream, &work);
        k_sn_set_out<<<blocks_for(nsn, 256, num_sms() * 32), 256, 0, stream>>>(sl.n, rowsum, sl.attr);
        RMX_LAUNCHED();
    }
    scratch.release(mk);
    timers.end(kTimerCoarsen, stream);
}

// One superstep (stochastic_greedy_partition, OmpRelaxmap.cpp:263-429).
void rmx_graph::stage(bool fine, std::vector<double> &L, const std::vector<uint8_t> &run) {
    Level &lv = fine ? node_lv : sn();
    count_units(lv, mods, stream);
    // Node sweeps may open a new module only once member lists exist, i.e.
    // after the first superstep (members.size() > 1 test, Module.cpp:1435);
    // super-node sweeps test the live module flow (Module.cpp:2620).
    const bool allow_first = fine ? superstep > 1 : true;
    stage_sweeps(lv, allow_first, L, run);
    if (!fine) project_sn_to_nodes();
    std::vector<uint8_t> act = run;
    std::vector<double> oldL;
    bool from_sn = !fine;  // after node sweeps the first conversion reads the node links
    do {
        oldL = L;
        convert_to_supernodes(from_sn);
        from_sn = true;
        stage_sweeps(sn(), true, L, act);
        project_sn_to_nodes();
        for (int32_t k = 0; k < K; k++)
            if (act[k] && !((oldL[k] - L[k]) / kLn2 > opt.threshold)) act[k] = 0;
    } while (any_set(act));
}

// Sub-batches per sweep. A fixed count for every sweep: fewer sub-batches in
// sweeps with small active sets make those sweeps cheaper but let
// simultaneous moves oscillate, which costs more sweeps than it saves (and
// code length); measured on the planted-partition benchmarks.
int rmx_graph::sub_batches_for(int64_t n_active) const {
    (void)n_active;
    return nsub;
}

int32_t rmx_graph::count_modules() {
    count_units(node_lv, mods, stream);
    unsigned long long *c = reinterpret_cast<unsigned long long *>(dtmp + 10);
    RMX_CUDA(cudaMemsetAsync(c, 0, 8, stream));
    k_count_nonzero<<<blocks_for(N, 256, num_sms() * 8), 256, 0, stream>>>(N, mods.count, c);
    RMX_LAUNCHED();
    unsigned long long h = 0;
    RMX_CUDA(cudaMemcpyAsync(&h, c, 8, cudaMemcpyDeviceToHost, stream));
    RMX_CUDA(cudaStreamSynchronize(stream));
    return (int32_t)h;
}

// main's superstep loop (OmpRelaxmap.cpp:181-219), per instance.
std::vector<double> rmx_graph::run_attempt(uint32_t seed) {
    run_seed = seed;
    sweep_no = 0;  // every random choice derives from (seed, sweep, sub-batch)
    init_singletons(node_lv, mods, stream);
    std::vector<uint8_t> run(K, 1), next(K, 0);
    set_active(run);
    instance_codelength(mods, inst1, stream);  // sum of exits of the singleton state
    std::vector<double> L = L0v, oldL = L;
    step_bits.clear();
    superstep = 1;
    bool fine = true;
    stage(fine, L, run);
    step_bits.push_back(L[0] / kLn2);
    if (opt.verbose)
        printf("SuperStep [%d] - codeLength = %g in %d modules.\n", superstep, L[0] / kLn2, count_modules());
    for (int32_t k = 0; k < K; k++) next[k] = !((oldL[k] - L[k]) / kLn2 < opt.threshold);
    while (any_set(next)) {
        run = next;
        oldL = L;
        superstep++;
        stage(fine, L, run);
        step_bits.push_back(L[0] / kLn2);
        if (opt.verbose)
            printf("SuperStep [%d] - codeLength = %g in %d modules.\n", superstep, L[0] / kLn2, count_modules());
        for (int32_t k = 0; k < K; k++) next[k] = run[k] && !((oldL[k] - L[k]) / kLn2 < opt.threshold);
        fine = !fine;
        if (any_set(next) && !fine) {
            set_active(next);  // coarse-tune only the modules of instances still running
            generate_sub_modules();
        }
    }
    prof.supersteps += superstep;
    runs_done++;
    return L;
}

std::vector<double> rmx_graph::run_union(const rmx_opts &o) {
    opt = o;
    if (opt.max_iter < 0) opt.max_iter = 0;
    nsub = opt.sub_batches > 0 ? std::min(opt.sub_batches, 32) : 4;
    cudaEvent_t t0, t1;
    RMX_CUDA(cudaEventCreate(&t0));
    RMX_CUDA(cudaEventCreate(&t1));
    RMX_CUDA(cudaEventRecord(t0, stream));
    initiate();
    std::vector<double> L = run_attempt(opt.seed);
    RMX_CUDA(cudaEventRecord(t1, stream));
    RMX_CUDA(cudaEventSynchronize(t1));
    float ms = 0;
    RMX_CUDA(cudaEventElapsedTime(&ms, t0, t1));
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    prof.total_ms = ms;
    if (timers.on) timers.resolve();
    return L;
}

double rmx_graph::optimize(const rmx_opts &o, int32_t *part_out, int32_t *n_modules) {
    opt = o;
    if (opt.max_iter < 0) opt.max_iter = 0;
    if (opt.attempts < 1) opt.attempts = 1;
    nsub = opt.sub_batches > 0 ? std::min(opt.sub_batches, 32) : 4;
    cudaEvent_t t0, t1;
    RMX_CUDA(cudaEventCreate(&t0));
    RMX_CUDA(cudaEventCreate(&t1));
    RMX_CUDA(cudaEventRecord(t0, stream));
    initiate();
    double best = INFINITY;
    int32_t best_nm = 0;
    std::vector<double> best_steps;
    // the best attempt's partition stays on the device and is copied out once at the end
    for (int a = 0; a < opt.attempts; a++) {
        const double L = run_attempt(opt.seed + (uint32_t)a)[0];
        if (L < best) {
            best = L;
            best_steps = step_bits;
            best_nm = count_modules();
            if (opt.attempts > 1)
                RMX_CUDA(cudaMemcpyAsync(best_part, nmod, sizeof(int32_t) * N, cudaMemcpyDeviceToDevice, stream));
        }
    }
    step_bits = best_steps;
    if (part_out)
        RMX_CUDA(cudaMemcpyAsync(part_out, opt.attempts > 1 ? best_part : nmod, sizeof(int32_t) * N,
                                 cudaMemcpyDeviceToHost, stream));
    RMX_CUDA(cudaEventRecord(t1, stream));
    RMX_CUDA(cudaEventSynchronize(t1));
    float ms = 0;
    RMX_CUDA(cudaEventElapsedTime(&ms, t0, t1));
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    prof.total_ms = ms;
    if (n_modules) *n_modules = best_nm;
    if (timers.on) timers.resolve();
    return best;
}

// ---------------------------------------------------------------- parity hooks

double rmx_graph::codelength_fp64(const int32_t *part_host) {
    initiate();
    check_partition(part_host);
    size_t mk = scratch.mark();
    int32_t *part = scratch.alloc<int32_t>(N);
    double *P = scratch.alloc<double>(N), *TW = scratch.alloc<double>(N), *D = scratch.alloc<double>(N),
           *OUT = scratch.alloc<double>(N);
    int32_t *cnt = scratch.alloc<int32_t>(N);
    const unsigned G = num_sms() * 4;
    double *parts = scratch.alloc<double>(4 * G);
    RMX_CUDA(cudaMemcpyAsync(part, part_host, sizeof(int32_t) * N, cudaMemcpyHostToDevice, stream));
    for (double *a : {P, TW, D, OUT}) RMX_CUDA(cudaMemsetAsync(a, 0, sizeof(double) * N, stream));
    RMX_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * N, stream));
    k_fp64_nodes<<<blocks_for(N, 256, num_sms() * 32), 256, 0, stream>>>(N, part, p, tw, dangling, P, TW, D, cnt);
    RMX_LAUNCHED();
    k_fp64_out<<<blocks_for((int64_t)N * 32, 256, num_sms() * 32), 256, 0, stream>>>(N, out_off, out_dst, out_f, part,
                                                                                     OUT);
    RMX_LAUNCHED();
    k_fp64_terms<<<G, 256, 0, stream>>>(N, P, TW, D, OUT, cnt, p, parts);
    RMX_LAUNCHED();
    std::vector<double> h(4 * G);
    RMX_CUDA(cudaMemcpyAsync(h.data(), parts, sizeof(double) * 4 * G, cudaMemcpyDeviceToHost, stream));
    RMX_CUDA(cudaStreamSynchronize(stream));
    scratch.release(mk);
    double a[4] = {0, 0, 0, 0};
    for (unsigned b = 0; b < G; b++)
        for (int q = 0; q < 4; q++) a[q] += h[4 * b + q];
    auto pl = [](double x) { return x > 0.0 ? x * std::log(x) : 0.0; };
    return pl(a[0]) - 2.0 * a[1] + a[2] - a[3];
}

void rmx_graph::coarsen_hook(const int32_t *part_host, int32_t *n_sn, int64_t *n_links, int32_t *sn_of_mod,
                             int64_t *o_off, int32_t *o_dst, double *o_f, int64_t *i_off, int32_t *i_src,
                             double *i_f) {
    initiate();
    check_partition(part_host);
    size_t mk = scratch.mark();
    const int64_t Em = std::max<int64_t>(E, 1);
    int32_t *part = scratch.alloc<int32_t>(N);
    int64_t *snid = scratch.alloc<int64_t>(N + 1);
    int32_t *grp = scratch.alloc<int32_t>(N), *cnt = scratch.alloc<int32_t>(N);
    int64_t *g_out_off = scratch.alloc<int64_t>(N + 1), *g_in_off = scratch.alloc<int64_t>(N + 1);
    int32_t *g_dst = scratch.alloc<int32_t>(Em), *g_src = scratch.alloc<int32_t>(Em);
    double *g_f = scratch.alloc<double>(Em), *g_if = scratch.alloc<double>(Em);
    fx_t *g_fx = scratch.alloc<fx_t>(Em), *g_ifx = scratch.alloc<fx_t>(Em);
    RMX_CUDA(cudaMemcpyAsync(part, part_host, sizeof(int32_t) * N, cudaMemcpyHostToDevice, stream));
    RMX_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * N, stream));
    Level tmp = node_lv;
    tmp.mod = part;
    ModState M = mods;
    M.count = cnt;
    count_units(tmp, M, stream);
    k_flags_nonempty<<<blocks_for(N, 256, num_sms() * 32), 256, 0, stream>>>(N, cnt, snid);
    RMX_LAUNCHED();
    scan_exclusive(snid, snid, N, dtmp + 0, scratch, stream);
    k_group_of_nodes<<<blocks_for(N, 256, num_sms() * 32), 256, 0, stream>>>(N, part, snid, grp);
    RMX_LAUNCHED();
    int64_t nsn = 0;
    RMX_CUDA(cudaMemcpyAsync(&nsn, dtmp + 0, sizeof(int64_t), cudaMemcpyDeviceToHost, stream));
    RMX_CUDA(cudaStreamSynchronize(stream));
    const int64_t m = coarsen_links(N, out_off, out_dst, out_f, out_fx, grp, (int32_t)nsn, g_out_off, g_dst, g_f,
                                    g_fx, g_in_off, g_src, g_if, g_ifx, scratch, stream);
    std::vector<int64_t> sid(N);
    RMX_CUDA(cudaMemcpyAsync(sid.data(), snid, sizeof(int64_t) * N, cudaMemcpyDeviceToHost, stream));
    std::vector<int32_t> hc(N);
    RMX_CUDA(cudaMemcpyAsync(hc.data(), cnt, sizeof(int32_t) * N, cudaMemcpyDeviceToHost, stream));
    if (o_off) RMX_CUDA(cudaMemcpyAsync(o_off, g_out_off, sizeof(int64_t) * (nsn + 1), cudaMemcpyDeviceToHost, stream));
    if (i_off) RMX_CUDA(cudaMemcpyAsync(i_off, g_in_off, sizeof(int64_t) * (nsn + 1), cudaMemcpyDeviceToHost, stream));
    if (m > 0) {
        if (o_dst) RMX_CUDA(cudaMemcpyAsync(o_dst, g_dst, sizeof(int32_t) * m, cudaMemcpyDeviceToHost, stream));
        if (o_f) RMX_CUDA(cudaMemcpyAsync(o_f, g_f, sizeof(double) * m, cudaMemcpyDeviceToHost, stream));
        if (i_src) RMX_CUDA(cudaMemcpyAsync(i_src, g_src, sizeof(int32_t) * m, cudaMemcpyDeviceToHost, stream));
        if (i_f) RMX_CUDA(cudaMemcpyAsync(i_f, g_if, sizeof(double) * m, cudaMemcpyDeviceToHost, stream));
    }
    RMX_CUDA(cudaStreamSynchronize(stream));
    scratch.release(mk);
    if (sn_of_mod)
        for (int32_t i = 0; i < N; i++) sn_of_mod[i] = hc[i] > 0 ? (int32_t)sid[i] : -1;
    if (n_sn) *n_sn = (int32_t)nsn;
    if (n_links) *n_links = m;
}

void rmx_graph::check_partition(const int32_t *part_host) const {
    for (int32_t v = 0; v < N; v++)
        if ((uint32_t)part_host[v] >= (uint32_t)N) throw std::invalid_argument("module id outside 0..N-1");
}

// The first super-node level of the partition part, built as the optimiser
// builds it after a node stage (module statistics from the nodes, then
// convert_to_supernodes); returns the number of super-nodes.
int32_t rmx_graph::supernodes_of(const int32_t *part_host) {
    initiate();
    check_partition(part_host);
    RMX_CUDA(cudaMemcpyAsync(nmod, part_host, sizeof(int32_t) * N, cudaMemcpyHostToDevice, stream));
    module_stats_from_units(node_lv, mods, stream);
    convert_to_supernodes(false);
    return sn().n;
}

void rmx_graph::coarsen_engine_hook(const int32_t *part_host, const int32_t *part2_host, int32_t *n_sn,
                                    int64_t *n_links, int32_t *sn_of_mod, int64_t *o_off, int32_t *o_dst, fx_t *o_fx,
                                    int64_t *i_off, int32_t *i_src, fx_t *i_fx, fx_t *sn_stat) {
    if (part2_host) check_partition(part2_host);
    supernodes_of(part_host);
    if (part2_host) {
        // the super-nodes move as whole modules: part2 relabels every first-level
        // module, the nodes follow (project_sn_to_nodes), and the second
        // conversion aggregates the first level's links
        size_t mk = scratch.mark();
        int32_t *map = scratch.alloc<int32_t>(N);
        RMX_CUDA(cudaMemcpyAsync(map, part2_host, sizeof(int32_t) * N, cudaMemcpyHostToDevice, stream));
        Level &l1 = sn();
        k_remap<<<blocks_for(l1.n, 256, num_sms() * 32), 256, 0, stream>>>(l1.n, map, l1.mod);
        RMX_LAUNCHED();
        project_sn_to_nodes();
        module_stats_from_units(node_lv, mods, stream);
        RMX_CUDA(cudaStreamSynchronize(stream));
        scratch.release(mk);
        convert_to_supernodes(true);
    }
    const Level &lv = sn();
    const int32_t ns = lv.n;
    const int64_t m = lv.m;
    std::vector<int32_t> smod(ns);
    RMX_CUDA(cudaMemcpyAsync(smod.data(), lv.mod, sizeof(int32_t) * ns, cudaMemcpyDeviceToHost, stream));
    if (o_off) RMX_CUDA(cudaMemcpyAsync(o_off, lv.out_off, sizeof(int64_t) * (ns + 1), cudaMemcpyDeviceToHost, stream));
    if (i_off) RMX_CUDA(cudaMemcpyAsync(i_off, lv.in_off, sizeof(int64_t) * (ns + 1), cudaMemcpyDeviceToHost, stream));
    if (sn_stat) RMX_CUDA(cudaMemcpyAsync(sn_stat, lv.attr, sizeof(Stat4) * ns, cudaMemcpyDeviceToHost, stream));
    if (m > 0) {
        if (o_dst) RMX_CUDA(cudaMemcpyAsync(o_dst, lv.out_dst, sizeof(int32_t) * m, cudaMemcpyDeviceToHost, stream));
        if (o_fx) RMX_CUDA(cudaMemcpyAsync(o_fx, lv.out_fx, sizeof(fx_t) * m, cudaMemcpyDeviceToHost, stream));
        if (i_src) RMX_CUDA(cudaMemcpyAsync(i_src, lv.in_src, sizeof(int32_t) * m, cudaMemcpyDeviceToHost, stream));
        if (i_fx) RMX_CUDA(cudaMemcpyAsync(i_fx, lv.in_fx, sizeof(fx_t) * m, cudaMemcpyDeviceToHost, stream));
    }
    RMX_CUDA(cudaStreamSynchronize(stream));
    if (sn_of_mod) {
        for (int32_t i = 0; i < N; i++) sn_of_mod[i] = -1;
        for (int32_t s = 0; s < ns; s++) sn_of_mod[smod[s]] = s;
    }
    if (n_sn) *n_sn = ns;
    if (n_links) *n_links = m;
}

void rmx_graph::evaluate_sn_hook(const int32_t *part_host, int32_t n_sn, const int32_t *sn_part_host,
                                 const uint8_t *allow_new_host, int32_t *best_mod, double *best_delta) {
    for (int32_t s = 0; s < n_sn; s++)
        if ((uint32_t)sn_part_host[s] >= (uint32_t)N) throw std::invalid_argument("module id outside 0..N-1");
    if (supernodes_of(part_host) != n_sn)
        throw std::invalid_argument("sn_part length differs from the number of super-nodes of part");
    Level &lv = sn();
    RMX_CUDA(cudaMemcpyAsync(lv.mod, sn_part_host, sizeof(int32_t) * n_sn, cudaMemcpyHostToDevice, stream));
    size_t mk = scratch.mark();
    uint8_t *an = nullptr;
    if (allow_new_host) {
        an = scratch.alloc<uint8_t>(n_sn);
        RMX_CUDA(cudaMemcpyAsync(an, allow_new_host, n_sn, cudaMemcpyHostToDevice, stream));
    }
    module_stats_from_units(lv, mods, stream);
    RMX_CUDA(cudaMemsetAsync(inst1.active, 1, (size_t)K, stream));
    instance_codelength(mods, inst1, stream);
    ensure_hub_table(lv);
    evaluate_all(lv, mods, inst1, work, an, 0.0, scratch, stream);
    RMX_CUDA(cudaMemcpyAsync(best_mod, work.prop, sizeof(int32_t) * n_sn, cudaMemcpyDeviceToHost, stream));
    RMX_CUDA(cudaMemcpyAsync(best_delta, work.pdelta, sizeof(double) * n_sn, cudaMemcpyDeviceToHost, stream));
    RMX_CUDA(cudaStreamSynchronize(stream));
    scratch.release(mk);
}

void rmx_graph::evaluate_hook(const int32_t *part_host, const uint8_t *allow_new_host, int32_t *best_mod,
                              double *best_delta) {
    initiate();
    check_partition(part_host);
    size_t mk = scratch.mark();
    uint8_t *an = nullptr;
    if (allow_new_host) {
        an = scratch.alloc<uint8_t>(N);
        RMX_CUDA(cudaMemcpyAsync(an, allow_new_host, N, cudaMemcpyHostToDevice, stream));
    }
    RMX_CUDA(cudaMemcpyAsync(nmod, part_host, sizeof(int32_t) * N, cudaMemcpyHostToDevice, stream));
    module_stats_from_units(node_lv, mods, stream);
    RMX_CUDA(cudaMemsetAsync(inst1.active, 1, (size_t)K, stream));
    instance_codelength(mods, inst1, stream);
    ensure_hub_table(node_lv);  // the bin bounds may have changed since initiate
    evaluate_all(node_lv, mods, inst1, work, an, 0.0, scratch, stream);
    RMX_CUDA(cudaMemcpyAsync(best_mod, work.prop, sizeof(int32_t) * N, cudaMemcpyDeviceToHost, stream));
    RMX_CUDA(cudaMemcpyAsync(best_delta, work.pdelta, sizeof(double) * N, cudaMemcpyDeviceToHost, stream));
    RMX_CUDA(cudaStreamSynchronize(stream));
    scratch.release(mk);
}
