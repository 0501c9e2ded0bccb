// Graph construction and stationary flow.
//
// build_csr     loader edge map + edge preparation (FileIO.cpp:157, :220;
//               OmpRelaxmap.cpp:117-135, 158-162) as a stable radix sort of
//               (src,dst), sequential in-order duplicate sums, compaction, and
//               a stable transpose for the in-links.
// normalise     Network::initiate's dangling detection and row normalisation
//               (Module.cpp:228-247), sequential row sums as in the reference.
// power_iteration  calculateSteadyState (Module.cpp:340-469) as ONE cooperative
//               persistent launch: pull SpMV over the CSC with the teleport and
//               dangling terms folded in, deterministic grid reductions for the
//               normaliser, L1 change and dangling mass, the reference's stop
//               rule evaluated identically by every block.
// edge_flows    Module.cpp:275-286 plus the fixed-point unit attributes.
#include <cooperative_groups.h>

#include <algorithm>
#include <climits>
#include <vector>

#include "rmx_engine.cuh"

namespace cg = cooperative_groups;

namespace rmx {

constexpr unsigned kFull = 0xffffffffu;

static int bits_for(int64_t n) {
    int b = 1;
    while ((int64_t(1) << b) < n) b++;
    return b;
}

// ------------------------------------------------------------ CSR build

__global__ void k_make_keys(const int32_t *src, const int32_t *dst, int64_t n, int b, uint64_t *keys, uint32_t *vals) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        keys[e] = ((uint64_t)(uint32_t)src[e] << b) | (uint32_t)dst[e];
        vals[e] = (uint32_t)e;
    }
}

__global__ void k_heads(const uint64_t *keys, int64_t n, uint8_t *flag) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
        flag[e] = (e == 0 || keys[e] != keys[e - 1]) ? 1 : 0;
}

// One thread per distinct (src,dst): weights summed sequentially in input order.
__global__ void k_sum_dups(const uint64_t *keys, const uint32_t *vals, const double *w, const int32_t *head,
                           const int64_t *n_heads, int64_t n, int b, int32_t *usrc, int32_t *udst, double *uw,
                           uint8_t *keep, unsigned long long *n_self) {
    int64_t U = *n_heads;
    uint64_t mask = (uint64_t(1) << b) - 1;
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < U; u += (int64_t)gridDim.x * blockDim.x) {
        int64_t beg = head[u], end = (u + 1 < U) ? head[u + 1] : n;
        double s = w[vals[beg]];
        for (int64_t j = beg + 1; j < end; j++) s += w[vals[j]];
        uint64_t k = keys[beg];
        int32_t a = (int32_t)(k >> b), d = (int32_t)(k & mask);
        usrc[u] = a;
        udst[u] = d;
        uw[u] = s;
        bool pos = s > 0.0;
        keep[u] = (pos && a != d) ? 1 : 0;
        if (pos && a == d) atomicAdd(n_self, 1ull);
    }
}

__global__ void k_gather_kept(const int32_t *kept, const int64_t *n_kept, const int32_t *usrc, const int32_t *udst,
                              const double *uw, int32_t *lsrc, int32_t *out_dst, double *out_w0,
                              unsigned long long *row_count) {
    int64_t K = *n_kept;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < K; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t u = kept[i];
        lsrc[i] = usrc[u];
        out_dst[i] = udst[u];
        out_w0[i] = uw[u];
        atomicAdd(&row_count[usrc[u]], 1ull);
    }
}

__global__ void k_dst_keys(const int32_t *dst, int64_t m, uint64_t *keys, uint32_t *vals, unsigned long long *col_count) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        keys[i] = (uint64_t)(uint32_t)dst[i];
        vals[i] = (uint32_t)i;
        atomicAdd(&col_count[dst[i]], 1ull);
    }
}

__global__ void k_gather_csc(const uint32_t *perm, int64_t m, const int32_t *lsrc, const double *w0, int32_t *in_src,
                             double *in_w) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t j = perm[i];
        in_src[i] = lsrc[j];
        in_w[i] = w0[j];
    }
}

CsrBuild build_csr(int32_t n, int64_t n_edges, int32_t *d_src, int32_t *d_dst, double *d_w, int64_t *out_off,
                   int32_t *out_dst, double *out_w0, int64_t *in_off, int32_t *in_src, double *in_w, Arena &ar,
                   cudaStream_t s, int64_t *scratch_dev) {
    CsrBuild r;
    const int T = 256;
    const unsigned G = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n_edges + T - 1) / T, num_sms() * 32));
    RMX_CUDA(cudaMemsetAsync(out_off, 0, sizeof(int64_t) * (n + 1), s));
    RMX_CUDA(cudaMemsetAsync(in_off, 0, sizeof(int64_t) * (n + 1), s));
    if (n_edges == 0) return r;
    size_t mk = ar.mark();
    const int b = bits_for(std::max<int64_t>(n, 2));
    uint64_t *keys = ar.alloc<uint64_t>(n_edges), *keys2 = ar.alloc<uint64_t>(n_edges);
    uint32_t *vals = ar.alloc<uint32_t>(n_edges), *vals2 = ar.alloc<uint32_t>(n_edges);
    k_make_keys<<<G, T, 0, s>>>(d_src, d_dst, n_edges, b, keys, vals);
    RMX_LAUNCHED();
    radix_sort_pairs(keys, vals, keys2, vals2, n_edges, 2 * b, ar, s);
    uint8_t *flag = ar.alloc<uint8_t>(n_edges);
    k_heads<<<G, T, 0, s>>>(keys, n_edges, flag);
    RMX_LAUNCHED();
    int32_t *head = ar.alloc<int32_t>(n_edges);
    int64_t *cnt = scratch_dev;  // [0] heads [1] kept [2] self-loops
    RMX_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int64_t) * 3, s));
    compact_flags(flag, n_edges, head, cnt + 0, ar, s);
    int32_t *usrc = ar.alloc<int32_t>(n_edges), *udst = ar.alloc<int32_t>(n_edges);
    double *uw = ar.alloc<double>(n_edges);
    uint8_t *keep = flag;  // reuse
    k_sum_dups<<<G, T, 0, s>>>(keys, vals, d_w, head, cnt + 0, n_edges, b, usrc, udst, uw, keep,
                               reinterpret_cast<unsigned long long *>(cnt + 2));
    RMX_LAUNCHED();
    int64_t U = 0;
    RMX_CUDA(cudaMemcpyAsync(&U, cnt + 0, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RMX_CUDA(cudaStreamSynchronize(s));
    int32_t *kept = ar.alloc<int32_t>(std::max<int64_t>(U, 1));
    compact_flags(keep, U, kept, cnt + 1, ar, s);
    int32_t *lsrc = ar.alloc<int32_t>(std::max<int64_t>(U, 1));
    k_gather_kept<<<G, T, 0, s>>>(kept, cnt + 1, usrc, udst, uw, lsrc, out_dst, out_w0,
                                  reinterpret_cast<unsigned long long *>(out_off));
    RMX_LAUNCHED();
    int64_t host_cnt[3];
    RMX_CUDA(cudaMemcpyAsync(host_cnt, cnt, sizeof(host_cnt), cudaMemcpyDeviceToHost, s));
    RMX_CUDA(cudaStreamSynchronize(s));
    const int64_t m = host_cnt[1];
    r.n_links = m;
    r.n_self = host_cnt[2];
    scan_exclusive(out_off, out_off, n + 1, nullptr, ar, s);
    if (m > 0) {
        k_dst_keys<<<G, T, 0, s>>>(out_dst, m, keys, vals, reinterpret_cast<unsigned long long *>(in_off));
        RMX_LAUNCHED();
        radix_sort_pairs(keys, vals, keys2, vals2, m, b, ar, s);
        k_gather_csc<<<G, T, 0, s>>>(vals, m, lsrc, out_w0, in_src, in_w);
        RMX_LAUNCHED();
    }
    scan_exclusive(in_off, in_off, n + 1, nullptr, ar, s);
    ar.release(mk);
    return r;
}

// ------------------------------------------------------------ normalise

// Per-row kernels take 32 consecutive rows per warp: a lane handles a row of
// up to kRowSeqMax links by itself, in link order (the reference's order);
// heavier rows (R-MAT hubs reach 10^5-10^6 links) are then taken by the whole
// warp one at a time, lanes striding the links, so that no lane walks a hub
// while the rest of the grid has finished.
constexpr int64_t kRowSeqMax = 256;

// Sum over the warp in a fixed butterfly order: every lane gets the same value.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// Row sums and normalised weights (Module.cpp:237-247: sum of the out-link
// weights in link order, then each weight divided by it; a heavy row's sum is
// formed by the warp, which rounds differently in the last bits).
__global__ void k_normalise_rows(int32_t n, const int64_t *off, const double *w0, double *wn, double *rowsum,
                                 uint8_t *dangling) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = gw * 32; base < n; base += nw * 32) {
        const int64_t i = base + lane;
        bool heavy = false;
        if (i < n) {
            const int64_t b = off[i], e = off[i + 1];
            heavy = e - b > kRowSeqMax;
            if (!heavy) {
                double s = 0.0;
                for (int64_t j = b; j < e; j++) s += w0[j];
                for (int64_t j = b; j < e; j++) wn[j] = w0[j] / s;
                rowsum[i] = s;
            }
            dangling[i] = (b == e) ? 1 : 0;
        }
        for (unsigned hv = __ballot_sync(kFull, heavy); hv; hv &= hv - 1) {
            const int64_t r = base + __ffs(hv) - 1;
            const int64_t b = off[r], e = off[r + 1];
            double s = 0.0;
            for (int64_t j = b + lane; j < e; j += 32) s += w0[j];
            s = warp_sum(s);
            for (int64_t j = b + lane; j < e; j += 32) wn[j] = w0[j] / s;
            if (lane == 0) rowsum[r] = s;
        }
    }
}

__global__ void k_normalise_cols(int64_t m, const int32_t *in_src, const double *raw, double *wn,
                                 const double *rowsum) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x)
        wn[k] = raw[k] / rowsum[in_src[k]];
}

void normalise(int32_t n, const int64_t *out_off, const double *out_w0, double *out_f, const int64_t *in_off,
               const int32_t *in_src, const double *in_w_raw, double *in_w, uint8_t *dangling, Arena &ar,
               cudaStream_t s, bool cols) {
    size_t mk = ar.mark();
    double *rowsum = ar.alloc<double>(std::max(n, 1));
    k_normalise_rows<<<blocks_for(n, 256, num_sms() * 32), 256, 0, s>>>(n, out_off, out_w0, out_f, rowsum, dangling);
    RMX_LAUNCHED();
    int64_t m = 0;
    if (cols) {
        RMX_CUDA(cudaMemcpyAsync(&m, in_off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        RMX_CUDA(cudaStreamSynchronize(s));
    }
    if (m > 0) {
        k_normalise_cols<<<blocks_for(m, 256, num_sms() * 32), 256, 0, s>>>(m, in_src, in_w_raw, in_w, rowsum);
        RMX_LAUNCHED();
    }
    ar.release(mk);
}

// ------------------------------------------------------------ power iteration

template <int NT>
__device__ __forceinline__ double block_sum(double v, double *sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    if (w == 0) {
        t = lane < NT / 32 ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(kFull, t, o);
    }
    __syncthreads();
    return t;  // valid in thread 0
}

// Sum of nb per-block partials in one fixed order; every block and thread gets
// the identical value.
__device__ __forceinline__ double sum_parts(const double *parts, int nb, double *sh) {
    if (threadIdx.x < 32) {
        double v = 0.0;
        for (int i = threadIdx.x; i < nb; i += 32) v += __ldcg(parts + i);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
        if (threadIdx.x == 0) sh[0] = v;
    }
    __syncthreads();
    double r = sh[0];
    __syncthreads();
    return r;
}

constexpr int kPowT = 256;
// resident blocks per SM the power iteration is compiled for (and launched with)
#ifndef RMX_POW_MINB
#define RMX_POW_MINB 6
#endif

// Rows of more than heavy_deg in-links (in-degree hubs) are not left to one
// lane group: their links come in chunks of kPowChunk, a warp per chunk, and
// after a grid barrier every such row sums its chunks' partials in chunk order.
constexpr int64_t kPowChunk = 256;
struct PowSplit {
    const int32_t *rows = nullptr;       // heavy rows
    int32_t n_rows = 0;
    const int64_t *row_chunk = nullptr;  // chunks of heavy row h: row_chunk[h] .. row_chunk[h+1]
    const int64_t *chunk_beg = nullptr, *chunk_end = nullptr;  // link range of every chunk
    int64_t n_chunks = 0;
    double *cpart = nullptr;             // partial pull of every chunk
    int64_t heavy_deg = INT64_MAX;
};

// The flow vector's gathered copy: on graphs whose flow vector is larger
// than L2 the pull gathers from a copy holding only the nodes that have
// out-links (rank[i] >= 0: node i's place in it; gsrc: in_src renumbered to
// those places), small enough to stay in L2. Values are the same doubles,
// so the sums are unchanged.
struct PowGather {
    const int32_t *gsrc = nullptr;  // nullptr: gather from x itself
    const int32_t *rank = nullptr;
    double *xc = nullptr;
};

template <int VEC>
__global__ void __launch_bounds__(kPowT, RMX_POW_MINB) k_power(const int64_t *__restrict__ in_off, const int32_t *__restrict__ in_src,
                                                 const double *__restrict__ in_w, const double *__restrict__ tw,
                                                 const uint8_t *__restrict__ dang, int32_t n, double *x, double *y,
                                                 double *parts, int *iters_out, double alpha, PowSplit sp,
                                                 PowGather pg) {
    cg::grid_group grid = cg::this_grid();
    __shared__ double sh[32];
    const int nb = gridDim.x;
    double *Sp = parts, *Dp = parts + nb, *Ep = parts + 2 * nb;
    const int64_t gtid = (int64_t)blockIdx.x * kPowT + threadIdx.x, gthreads = (int64_t)nb * kPowT;

    // the link arrays are streamed with the evict-first hint so that the
    // gathered vector stays in L2 between iterations
    const double *xg = pg.gsrc ? pg.xc : x;        // the vector the pull gathers from
    const int32_t *gs = pg.gsrc ? pg.gsrc : in_src;  // and the links' places in it
    double dl = 0.0;
    const double x0 = 1.0 / n;
    for (int64_t i = gtid; i < n; i += gthreads) {
        x[i] = x0;
        if (pg.gsrc && pg.rank[i] >= 0) pg.xc[pg.rank[i]] = x0;
        if (dang[i]) dl += x0;
    }
    dl = block_sum<kPowT>(dl, sh);
    if (threadIdx.x == 0) Dp[blockIdx.x] = dl;
    grid.sync();

    constexpr int RPW = 32 / VEC;  // rows per warp per step
    const int lane = threadIdx.x & 31, sub = lane / VEC, lv = lane % VEC;
    const int64_t gwarp = gtid >> 5, nwarps = gthreads >> 5;
    int iter = 0;
    for (;;) {
        const double D = sum_parts(Dp, nb, sh);
        const double beta = 1.0 - alpha;  // 1.0 - 0.15 is kBeta exactly
        const double coef = alpha + beta * D;
        double ls = 0.0;
        for (int64_t base = gwarp * RPW; base < n; base += nwarps * RPW) {
            const int64_t r = base + sub;
            double acc = 0.0;
            bool mine = r < n;
            if (mine) {
                const int64_t b = in_off[r], e = in_off[r + 1];
                mine = e - b <= sp.heavy_deg;
                if (mine)
                    for (int64_t k = b + lv; k < e; k += VEC) acc += beta * __ldcs(in_w + k) * __ldcg(xg + __ldcs(gs + k));
            }
#pragma unroll
            for (int o = VEC / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
            if (mine && lv == 0) {
                const double v = coef * tw[r] + acc;
                y[r] = v;
                ls += v;
            }
        }
        if (sp.n_rows > 0) {  // the same branch in every block
            for (int64_t c = gwarp; c < sp.n_chunks; c += nwarps) {
                double acc = 0.0;
                for (int64_t k = sp.chunk_beg[c] + lane; k < sp.chunk_end[c]; k += 32)
                    acc += beta * __ldcs(in_w + k) * __ldcg(xg + __ldcs(gs + k));
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
                if (lane == 0) sp.cpart[c] = acc;
            }
            grid.sync();
            for (int64_t h = gwarp; h < sp.n_rows; h += nwarps) {
                const int32_t r = sp.rows[h];
                double acc = 0.0;
                for (int64_t c = sp.row_chunk[h] + lane; c < sp.row_chunk[h + 1]; c += 32) acc += __ldcg(sp.cpart + c);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
                if (lane == 0) {
                    const double v = coef * tw[r] + acc;
                    y[r] = v;
                    ls += v;
                }
            }
        }
        ls = block_sum<kPowT>(ls, sh);
        if (threadIdx.x == 0) Sp[blockIdx.x] = ls;
        grid.sync();
        const double S = sum_parts(Sp, nb, sh);
        double el = 0.0;
        dl = 0.0;
        for (int64_t i = gtid; i < n; i += gthreads) {
            const double xn = __ldcg(y + i) / S;
            el += fabs(xn - x[i]);
            x[i] = xn;
            if (pg.gsrc && pg.rank[i] >= 0) pg.xc[pg.rank[i]] = xn;
            if (dang[i]) dl += xn;
        }
        el = block_sum<kPowT>(el, sh);
        dl = block_sum<kPowT>(dl, sh);
        if (threadIdx.x == 0) {
            Ep[blockIdx.x] = el;
            Dp[blockIdx.x] = dl;
        }
        grid.sync();
        const double diff = sum_parts(Ep, nb, sh);
        iter++;
        if (iter >= 200 || (diff <= 1.0e-15 && iter >= 50)) break;  // Module.cpp:460
    }
    if (gtid == 0) *iters_out = iter;
}

__global__ void k_pow_heavy_flags(int32_t n, const int64_t *in_off, int64_t heavy_deg, uint8_t *flag) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        flag[r] = in_off[r + 1] - in_off[r] > heavy_deg ? 1 : 0;
}

__global__ void k_pow_heavy_ranges(const int32_t *rows, int64_t nh, const int64_t *in_off, int64_t *be) {
    for (int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; h < nh; h += (int64_t)gridDim.x * blockDim.x) {
        be[2 * h] = in_off[rows[h]];
        be[2 * h + 1] = in_off[rows[h] + 1];
    }
}

// The heavy rows of a CSC and their chunk tables, in arena memory (released
// with the caller's mark).
static PowSplit heavy_split(int32_t n, const int64_t *in_off, int64_t heavy_deg, Arena &ar, cudaStream_t s) {
    PowSplit sp;
    if (n <= 0) return sp;
    uint8_t *flag = ar.alloc<uint8_t>(n);
    int32_t *rows = ar.alloc<int32_t>(n);
    int64_t *cnt = ar.alloc<int64_t>(1);
    k_pow_heavy_flags<<<blocks_for(n, 256, num_sms() * 32), 256, 0, s>>>(n, in_off, heavy_deg, flag);
    RMX_LAUNCHED();
    compact_flags(flag, n, rows, cnt, ar, s);
    int64_t nh = 0;
    RMX_CUDA(cudaMemcpyAsync(&nh, cnt, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RMX_CUDA(cudaStreamSynchronize(s));
    if (nh == 0) return sp;
    int64_t *be = ar.alloc<int64_t>(2 * nh);
    k_pow_heavy_ranges<<<blocks_for(nh, 256, num_sms() * 8), 256, 0, s>>>(rows, nh, in_off, be);
    RMX_LAUNCHED();
    std::vector<int64_t> hbe(2 * nh);
    RMX_CUDA(cudaMemcpyAsync(hbe.data(), be, sizeof(int64_t) * 2 * nh, cudaMemcpyDeviceToHost, s));
    RMX_CUDA(cudaStreamSynchronize(s));
    std::vector<int64_t> rc(nh + 1, 0), cb, ce;
    for (int64_t h = 0; h < nh; h++) {
        for (int64_t k = hbe[2 * h]; k < hbe[2 * h + 1]; k += kPowChunk) {
            cb.push_back(k);
            ce.push_back(std::min(k + kPowChunk, hbe[2 * h + 1]));
        }
        rc[h + 1] = (int64_t)cb.size();
    }
    const int64_t nc = (int64_t)cb.size();
    int64_t *d_rc = ar.alloc<int64_t>(nh + 1), *d_cb = ar.alloc<int64_t>(nc), *d_ce = ar.alloc<int64_t>(nc);
    double *cpart = ar.alloc<double>(nc);
    RMX_CUDA(cudaMemcpyAsync(d_rc, rc.data(), sizeof(int64_t) * (nh + 1), cudaMemcpyHostToDevice, s));
    RMX_CUDA(cudaMemcpyAsync(d_cb, cb.data(), sizeof(int64_t) * nc, cudaMemcpyHostToDevice, s));
    RMX_CUDA(cudaMemcpyAsync(d_ce, ce.data(), sizeof(int64_t) * nc, cudaMemcpyHostToDevice, s));
    RMX_CUDA(cudaStreamSynchronize(s));  // the host tables are freed on return
    sp.rows = rows;
    sp.n_rows = (int32_t)nh;
    sp.row_chunk = d_rc;
    sp.chunk_beg = d_cb;
    sp.chunk_end = d_ce;
    sp.n_chunks = nc;
    sp.cpart = cpart;
    sp.heavy_deg = heavy_deg;
    return sp;
}

__global__ void k_src_flags(int64_t m, const int32_t *in_src, uint32_t *flag) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x)
        flag[in_src[k]] = 1u;  // every writer stores the same value
}

__global__ void k_src_rank(int32_t n, const uint32_t *flag, const uint32_t *pos, int32_t *rank) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        rank[i] = flag[i] ? (int32_t)pos[i] : -1;
}

__global__ void k_src_remap(int64_t m, const int32_t *in_src, const int32_t *rank, int32_t *gsrc) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x)
        gsrc[k] = rank[in_src[k]];
}

// The gathered copy (PowGather) where the flow vector is larger than three
// quarters of L2 (smaller ones mostly stay there anyway: measured slower at
// 2^22 nodes, the copy's set-up costing more than it saved) and at most three
// quarters of the nodes have out-links; otherwise none. In arena memory
// (released with the caller's mark).
static PowGather gather_copy(int32_t n, const int64_t *in_off, const int32_t *in_src, Arena &ar, cudaStream_t s) {
    PowGather pg;
    constexpr int64_t kMinNodes = (int64_t)96 << 20 >> 3;  // 96 MB of doubles
    if ((int64_t)n < kMinNodes) return pg;
    int64_t m = 0;
    RMX_CUDA(cudaMemcpyAsync(&m, in_off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RMX_CUDA(cudaStreamSynchronize(s));
    if (m <= 0) return pg;
    const size_t mk = ar.mark();
    uint32_t *flag = ar.alloc<uint32_t>(n), *pos = ar.alloc<uint32_t>(n + 1);
    RMX_CUDA(cudaMemsetAsync(flag, 0, sizeof(uint32_t) * n, s));
    k_src_flags<<<blocks_for(m, 256, num_sms() * 32), 256, 0, s>>>(m, in_src, flag);
    RMX_LAUNCHED();
    scan_exclusive(flag, pos, n, pos + n, ar, s);
    uint32_t cnt = 0;
    RMX_CUDA(cudaMemcpyAsync(&cnt, pos + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    RMX_CUDA(cudaStreamSynchronize(s));
    if ((int64_t)cnt * 4 > (int64_t)n * 3) {
        ar.release(mk);
        return pg;
    }
    int32_t *rank = ar.alloc<int32_t>(n), *gsrc = ar.alloc<int32_t>(m);
    double *xc = ar.alloc<double>(std::max<uint32_t>(cnt, 1));
    k_src_rank<<<blocks_for(n, 256, num_sms() * 32), 256, 0, s>>>(n, flag, pos, rank);
    RMX_LAUNCHED();
    k_src_remap<<<blocks_for(m, 256, num_sms() * 32), 256, 0, s>>>(m, in_src, rank, gsrc);
    RMX_LAUNCHED();
    pg.gsrc = gsrc;
    pg.rank = rank;
    pg.xc = xc;
    return pg;
}

template <int VEC>
static int launch_power(int32_t n, const int64_t *in_off, const int32_t *in_src, const double *in_w, const double *tw,
                        const uint8_t *dangling, double *p, Arena &ar, cudaStream_t s, double alpha) {
    int dev = 0, per_sm = 0, coop = 0;
    RMX_CUDA(cudaGetDevice(&dev));
    RMX_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    if (!coop) throw CudaError(cudaErrorNotSupported, "cooperative launch not supported");
    RMX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_power<VEC>, kPowT, 0));
    int nb = std::max(1, std::min(per_sm, RMX_POW_MINB)) * num_sms();
    nb = (int)std::min<int64_t>(nb, std::max<int64_t>(1, ((int64_t)n * VEC + kPowT - 1) / kPowT));
    size_t mk = ar.mark();
    double *y = ar.alloc<double>(std::max(n, 1));
    double *parts = ar.alloc<double>(3 * nb);
    int *iters = ar.alloc<int>(1);
    PowSplit sp = heavy_split(n, in_off, 64 * VEC, ar, s);
    PowGather pg = gather_copy(n, in_off, in_src, ar, s);
    void *args[] = {(void *)&in_off, (void *)&in_src, (void *)&in_w,  (void *)&tw,    (void *)&dangling, (void *)&n,
                    (void *)&p,      (void *)&y,      (void *)&parts, (void *)&iters, (void *)&alpha,    (void *)&sp,
                    (void *)&pg};
    RMX_CUDA(cudaLaunchCooperativeKernel((void *)k_power<VEC>, dim3(nb), dim3(kPowT), args, 0, s));
    RMX_LAUNCHED();
    int h = 0;
    RMX_CUDA(cudaMemcpyAsync(&h, iters, sizeof(int), cudaMemcpyDeviceToHost, s));
    RMX_CUDA(cudaStreamSynchronize(s));
    ar.release(mk);
    return h;
}

// Launch of the same solve into caller-provided scratch: y[n], parts[3 * max_blocks],
// *iters; nothing is allocated and nothing waits on the stream.
template <int VEC>
static void launch_power_into(int32_t n, const int64_t *in_off, const int32_t *in_src, const double *in_w,
                              const double *tw, const uint8_t *dangling, double *p, double *y, double *parts,
                              int max_blocks, int *iters, cudaStream_t s) {
    int dev = 0, per_sm = 0, coop = 0;
    RMX_CUDA(cudaGetDevice(&dev));
    RMX_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    if (!coop) throw CudaError(cudaErrorNotSupported, "cooperative launch not supported on this device");
    RMX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_power<VEC>, kPowT, 0));
    int nb = std::max(1, std::min(per_sm, RMX_POW_MINB)) * num_sms();
    nb = (int)std::min<int64_t>(nb, std::max<int64_t>(1, ((int64_t)n * VEC + kPowT - 1) / kPowT));
    nb = std::min(nb, max_blocks);
    double alpha = kAlpha;
    // No chunked rows: in-degree hubs are pulled in one pass by their own
    // lanes (nothing beyond the caller's scratch), so on graphs with such
    // hubs the sums round differently from power_iteration's. No gathered copy.
    PowSplit sp;
    PowGather pg;
    void *args[] = {(void *)&in_off, (void *)&in_src, (void *)&in_w,  (void *)&tw,    (void *)&dangling, (void *)&n,
                    (void *)&p,      (void *)&y,      (void *)&parts, (void *)&iters, (void *)&alpha,    (void *)&sp,
                    (void *)&pg};
    RMX_CUDA(cudaLaunchCooperativeKernel((void *)k_power<VEC>, dim3(nb), dim3(kPowT), args, 0, s));
    RMX_LAUNCHED();
}

void power_iteration_into(int32_t n, const int64_t *in_off, const int32_t *in_src, const double *in_w,
                          const double *tw, const uint8_t *dangling, double *p, double *y, double *parts,
                          int max_blocks, int *iters, cudaStream_t s, int vec) {
    if (n <= 0) return;
    switch (vec) {
        case 4: return launch_power_into<4>(n, in_off, in_src, in_w, tw, dangling, p, y, parts, max_blocks, iters, s);
        case 8: return launch_power_into<8>(n, in_off, in_src, in_w, tw, dangling, p, y, parts, max_blocks, iters, s);
        case 16:
            return launch_power_into<16>(n, in_off, in_src, in_w, tw, dangling, p, y, parts, max_blocks, iters, s);
        default:
            return launch_power_into<32>(n, in_off, in_src, in_w, tw, dangling, p, y, parts, max_blocks, iters, s);
    }
}

// ------------------------------------------------ per-component power iteration

constexpr int kCompT = 256;

// Sum over the block, returned to every thread.
__device__ __forceinline__ double comp_block_sum(double v, double *sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();  // sh free from the previous use
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
#pragma unroll
    for (int k = 0; k < kCompT / 32; k++) t += sh[k];
    return t;
}

// calculateSteadyState for many independent graphs held as one disjoint union:
// one block per component (node range [lo, hi)), with the component's own
// dangling mass, normaliser, L1 change and the reference's stop rule
// (Module.cpp:340-469). tw is normalised within every component.
template <int VEC>
__global__ void __launch_bounds__(kCompT) k_power_comp(int32_t n_comp, const int64_t *__restrict__ comp,
                                                       const int64_t *__restrict__ in_off,
                                                       const int32_t *__restrict__ in_src,
                                                       const double *__restrict__ in_w, const double *__restrict__ tw,
                                                       const uint8_t *__restrict__ dang, double *x, double *y,
                                                       int *iters) {
    __shared__ double sh[kCompT / 32];
    constexpr int RPW = 32 / VEC;
    const int lane = threadIdx.x & 31, sub = lane / VEC, lv = lane % VEC, warp = threadIdx.x >> 5;
    constexpr int NW = kCompT / 32;
    for (int32_t c = blockIdx.x; c < n_comp; c += gridDim.x) {
        const int64_t lo = comp[2 * c], hi = comp[2 * c + 1];
        const double x0 = 1.0 / (double)(hi - lo);
        double dl = 0.0;
        for (int64_t i = lo + threadIdx.x; i < hi; i += kCompT) {
            x[i] = x0;
            if (dang[i]) dl += x0;
        }
        double D = comp_block_sum(dl, sh);
        int iter = 0;
        for (;;) {
            const double coef = kAlpha + kBeta * D;
            double ls = 0.0;
            for (int64_t base = lo + (int64_t)warp * RPW; base < hi; base += (int64_t)NW * RPW) {
                const int64_t r = base + sub;
                double acc = 0.0;
                if (r < hi) {
                    const int64_t e = in_off[r + 1];
                    for (int64_t k = in_off[r] + lv; k < e; k += VEC) acc += kBeta * in_w[k] * x[in_src[k]];
                }
#pragma unroll
                for (int o = VEC / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
                if (r < hi && lv == 0) {
                    const double v = coef * tw[r] + acc;
                    y[r] = v;
                    ls += v;
                }
            }
            const double S = comp_block_sum(ls, sh);  // also orders the y writes before the reads below
            double el = 0.0;
            dl = 0.0;
            for (int64_t i = lo + threadIdx.x; i < hi; i += kCompT) {
                const double xn = y[i] / S;
                el += fabs(xn - x[i]);
                x[i] = xn;
                if (dang[i]) dl += xn;
            }
            const double diff = comp_block_sum(el, sh);
            D = comp_block_sum(dl, sh);
            iter++;
            if (iter >= 200 || (diff <= 1.0e-15 && iter >= 50)) break;  // Module.cpp:460
        }
        if (threadIdx.x == 0) iters[c] = iter;
        __syncthreads();
    }
}

// Copies of a graph share its flow: p of every non-canonical instance is read
// from its canonical copy.
__global__ void k_replicate_flows(int32_t n, const int32_t *node_inst, const int64_t *inst_noff,
                                  const int32_t *inst_canon, double *p) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t k = node_inst[i], c = inst_canon[k];
        if (c != k) p[i] = p[i - inst_noff[k] + inst_noff[c]];
    }
}

int power_iteration_components(int32_t n, int32_t n_comp, const int64_t *comp, const int32_t *node_inst,
                               const int64_t *inst_noff, const int32_t *inst_canon, const int64_t *in_off,
                               const int32_t *in_src, const double *in_w, const double *tw, const uint8_t *dangling,
                               double *p, Arena &ar, cudaStream_t s, int vec) {
    if (n <= 0 || n_comp <= 0) return 0;
    size_t mk = ar.mark();
    double *y = ar.alloc<double>(n);
    int *iters = ar.alloc<int>(n_comp);
    const unsigned G = (unsigned)std::min<int64_t>(n_comp, (int64_t)num_sms() * 8);
    switch (vec) {
        case 4: k_power_comp<4><<<G, kCompT, 0, s>>>(n_comp, comp, in_off, in_src, in_w, tw, dangling, p, y, iters); break;
        case 8: k_power_comp<8><<<G, kCompT, 0, s>>>(n_comp, comp, in_off, in_src, in_w, tw, dangling, p, y, iters); break;
        case 16: k_power_comp<16><<<G, kCompT, 0, s>>>(n_comp, comp, in_off, in_src, in_w, tw, dangling, p, y, iters); break;
        default: k_power_comp<32><<<G, kCompT, 0, s>>>(n_comp, comp, in_off, in_src, in_w, tw, dangling, p, y, iters); break;
    }
    RMX_LAUNCHED();
    k_replicate_flows<<<blocks_for(n, 256, num_sms() * 32), 256, 0, s>>>(n, node_inst, inst_noff, inst_canon, p);
    RMX_LAUNCHED();
    std::vector<int> h(n_comp);
    RMX_CUDA(cudaMemcpyAsync(h.data(), iters, sizeof(int) * n_comp, cudaMemcpyDeviceToHost, s));
    RMX_CUDA(cudaStreamSynchronize(s));
    ar.release(mk);
    return *std::max_element(h.begin(), h.end());
}

// About 2.5 links per lane: more rows in flight per warp hide the gather
// latency better than idle lanes do (mean in-degree 20: 8 lanes, 6.7 ms
// against 9.2 ms with 16 lanes for 50 iterations on 19.5M links; R-MAT scale
// 24, mean 15.7: 4 lanes 7% faster than 8, 16 lanes 10% slower).
int spmv_width(double mean_in_degree) {
    return mean_in_degree <= 16 ? 4 : (mean_in_degree <= 24 ? 8 : (mean_in_degree <= 48 ? 16 : 32));
}

int power_iteration(int32_t n, const int64_t *in_off, const int32_t *in_src, const double *in_w, const double *tw,
                    const uint8_t *dangling, double *p, Arena &ar, cudaStream_t s, int vec, double alpha) {
    if (n <= 0) return 0;
    switch (vec) {
        case 4: return launch_power<4>(n, in_off, in_src, in_w, tw, dangling, p, ar, s, alpha);
        case 8: return launch_power<8>(n, in_off, in_src, in_w, tw, dangling, p, ar, s, alpha);
        case 16: return launch_power<16>(n, in_off, in_src, in_w, tw, dangling, p, ar, s, alpha);
        default: return launch_power<32>(n, in_off, in_src, in_w, tw, dangling, p, ar, s, alpha);
    }
}

// ------------------------------------------------------------ flows

// Edge flows f = p_u * w~ (Module.cpp:275-286) in FP64 and fixed point, and
// each node's unit statistics; the out-flow sum is a fixed-point (exact,
// order-free) sum, so heavy rows done by the whole warp give the same bits.
__global__ void k_flow_rows(int32_t n, const int64_t *off, double *f, fx_t *fx, const double *p, const double *tw,
                            const uint8_t *dangling, Stat4 *attr, fx_t *s0) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    fx_t s0l = 0;
    for (int64_t base = gw * 32; base < n; base += nw * 32) {
        const int64_t i = base + lane;
        bool heavy = false;
        fx_t out = 0;
        if (i < n) {
            const int64_t b = off[i], e = off[i + 1];
            heavy = e - b > kRowSeqMax;
            const double pi = p[i];
            if (!heavy)
                for (int64_t j = b; j < e; j++) {
                    const double v = pi * f[j];  // Module.cpp:280
                    f[j] = v;
                    const fx_t q = to_fx(v);
                    fx[j] = q;
                    out += q;
                }
            s0l += to_fxl(plogp(pi));
        }
        for (unsigned hv = __ballot_sync(kFull, heavy); hv; hv &= hv - 1) {
            const int src = __ffs(hv) - 1;
            const int64_t r = base + src;
            const int64_t b = off[r], e = off[r + 1];
            const double pr = p[r];
            fx_t o = 0;
            for (int64_t j = b + lane; j < e; j += 32) {
                const double v = pr * f[j];
                f[j] = v;
                const fx_t q = to_fx(v);
                fx[j] = q;
                o += q;
            }
#pragma unroll
            for (int q = 16; q > 0; q >>= 1) o += __shfl_xor_sync(kFull, o, q);
            if (lane == src) out = o;
        }
        if (i < n) {
            Stat4 a;
            a.P = to_fx(p[i]);
            a.TW = to_fx(tw[i]);
            a.D = dangling[i] ? a.P : 0;
            a.OUT = out;
            attr[i] = a;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s0l += __shfl_xor_sync(kFull, s0l, o);
    if (lane == 0 && s0l != 0) atomic_add_fx(s0, s0l);
}

__global__ void k_flow_cols(int64_t m, const int32_t *in_src, const double *in_w, const double *p, fx_t *in_fx) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x)
        in_fx[k] = to_fx(p[in_src[k]] * in_w[k]);
}

void edge_flows(int32_t n, int64_t m, const int64_t *out_off, double *out_f, fx_t *out_fx, const int32_t *in_src,
                const double *in_w, fx_t *in_fx, const double *p, const double *tw, const uint8_t *dangling,
                Stat4 *attr, fx_t *s0_acc, cudaStream_t s) {
    RMX_CUDA(cudaMemsetAsync(s0_acc, 0, sizeof(fx_t), s));
    k_flow_rows<<<blocks_for(n, 256, num_sms() * 32), 256, 0, s>>>(n, out_off, out_f, out_fx, p, tw, dangling, attr,
                                                                   s0_acc);
    RMX_LAUNCHED();
    if (m > 0) {
        k_flow_cols<<<blocks_for(m, 256, num_sms() * 32), 256, 0, s>>>(m, in_src, in_w, p, in_fx);
        RMX_LAUNCHED();
    }
}

// Singleton exit as Module::Module(int, Node*) (Module.cpp:76-95): the
// out-flow summed in link order, by the warp for heavy rows.
__global__ void k_singleton_exit(int32_t n, const int64_t *off, const double *f, const double *p, const double *tw,
                                 const uint8_t *dangling, double *ex) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = gw * 32; base < n; base += nw * 32) {
        const int64_t i = base + lane;
        bool heavy = false;
        double s = 0.0;
        if (i < n) {
            const int64_t b = off[i], e = off[i + 1];
            heavy = e - b > kRowSeqMax;
            if (!heavy)
                for (int64_t j = b; j < e; j++) s += f[j];
        }
        for (unsigned hv = __ballot_sync(kFull, heavy); hv; hv &= hv - 1) {
            const int src = __ffs(hv) - 1;
            const int64_t r = base + src;
            double t = 0.0;
            for (int64_t j = off[r] + lane; j < off[r + 1]; j += 32) t += f[j];
            t = warp_sum(t);
            if (lane == src) s = t;
        }
        if (i < n) ex[i] = dangling[i] ? (1.0 - tw[i]) * p[i] : kAlpha * (1.0 - tw[i]) * p[i] + kBeta * s;
    }
}

void singleton_exits(int32_t n, const int64_t *out_off, const double *out_f, const double *p, const double *tw,
                     const uint8_t *dangling, double *exitpr, cudaStream_t s) {
    k_singleton_exit<<<blocks_for(n, 256, num_sms() * 32), 256, 0, s>>>(n, out_off, out_f, p, tw, dangling, exitpr);
    RMX_LAUNCHED();
}

}  // namespace rmx
