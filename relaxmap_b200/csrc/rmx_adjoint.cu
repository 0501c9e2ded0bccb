// Adjoint of the two-level code length of a FIXED partition with respect to
// the link weights and the teleportation probability. The reference has no
// gradient; the forward model is its own:
//
//   w~_ab = w_ab / sum_c w_ac                       (Module.cpp:237-247)
//   p     = stationary flow of  p = (1-t) W~^T p + (t + (1-t) d.p) tw
//                                                   (Module.cpp:340-469)
//   q_m   = t (1-TW_m) P_m + (1-t) (OUT_m + (1-TW_m) D_m)
//   L     = plogp(sum q) - 2 sum plogp(q_m) + sum plogp(q_m+P_m) - sum plogp(p_a)
//                                                   (Module.cpp:2966-3002)
// with OUT_m the flow p_a w~_ab of links leaving m, D_m the flow of m's
// dangling nodes, TW_m its teleport weight, t the teleportation probability
// (0.15 in the reference).
//
// Backward pass (nothing of the forward iteration is stored; p is recomputed):
//   g_m = log Q - 2 log q_m + log(q_m + P_m),  h_m = log(q_m + P_m) + 1
//   c_a = dL/dp_a at fixed w~ = g_m (1-TW_m)(t + (1-t) d_a) + h_m
//         - (log p_a + 1) + (1-t) g_m sum_{b not in m} w~_ab
//   lambda = c + (1-t) (W~ lambda + d (tw . lambda))       (transposed solve,
//            a pull over the out-links, contraction factor 1-t)
//   dL/dw~_ab = (1-t) p_a (g_m [m(b) != m] + lambda_b)
//   dL/dw_ab  = (dL/dw~_ab - sum_c w~_ac dL/dw~_ac) / sum_c w_ac
//   dL/dt     = sum_m g_m ((1-TW_m) P_m - OUT_m - (1-TW_m) D_m)
//             + (lambda . tw - lambda . p) / (1-t)
// Module sums are fixed-point (exact, order-free); the solve's reductions use
// fixed-order block partials, so results do not depend on scheduling.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "rmx_graph.hpp"

namespace cg = cooperative_groups;

namespace rmx {
namespace {

constexpr unsigned kFullA = 0xffffffffu;
constexpr int kAdjT = 256;
// resident blocks per SM the transposed solve is compiled for (and launched with)
#ifndef RMX_ADJ_MINB
#define RMX_ADJ_MINB 4
#endif
// links per lane in the degree classes up to 16 links (1 or 2)
#ifndef RMX_ADJ_LPL
#define RMX_ADJ_LPL 2
#endif

__device__ __forceinline__ double dlog(double x) { return x > 0.0 ? log(x) : 0.0; }

__global__ void k_adj_rows(int32_t n, const int64_t *off, const int32_t *dst, const double *w0, const int32_t *part,
                           const double *p, const double *tw, const uint8_t *dang, double *rowsum, double *cross,
                           Stat4 *mstat, fx_t *s0) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    fx_t sl = 0;
    for (int64_t a = gw; a < n; a += nw) {
        const int32_t m = part[a];
        double s = 0.0, x = 0.0;
        for (int64_t e = off[a] + lane; e < off[a + 1]; e += 32) {
            s += w0[e];
            if (part[dst[e]] != m) x += w0[e];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            s += __shfl_xor_sync(kFullA, s, o);
            x += __shfl_xor_sync(kFullA, x, o);
        }
        if (lane == 0) {
            const double pa = p[a];
            const double cr = s > 0.0 ? x / s : 0.0;  // sum of w~ over crossing links
            rowsum[a] = s;
            cross[a] = cr;
            atomic_add_fx(&mstat[m].P, to_fx(pa));
            atomic_add_fx(&mstat[m].TW, to_fx(tw[a]));
            if (dang[a]) atomic_add_fx(&mstat[m].D, to_fx(pa));
            if (cr > 0.0) atomic_add_fx(&mstat[m].OUT, to_fx(pa * cr));
            sl += to_fxl(plogp(pa));
        }
    }
    if (lane == 0 && sl != 0) atomic_add_fx(s0, sl);
}

// Per module: q_m and the code-length sums; parts[3*block + k] = block sums of
// q, plogp(q) and plogp(q+P).
__global__ void k_adj_mod1(int32_t n, const Stat4 *mstat, double alpha, double *q, double *parts) {
    __shared__ double sh[3][kAdjT / 32];
    double a0 = 0, a1 = 0, a2 = 0;
    const double beta = 1.0 - alpha;
    for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < n; m += (int64_t)gridDim.x * blockDim.x) {
        const Stat4 st = mstat[m];
        if (st.P == 0 && st.TW == 0) {
            q[m] = 0.0;
            continue;
        }
        const double P = from_fx(st.P), TW = from_fx(st.TW), D = from_fx(st.D), OUT = from_fx(st.OUT);
        const double e = alpha * (1.0 - TW) * P + beta * (OUT + (1.0 - TW) * D);
        q[m] = e;
        a0 += e;
        a1 += plogp(e);
        a2 += plogp(e + P);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(kFullA, a0, o);
        a1 += __shfl_xor_sync(kFullA, a1, o);
        a2 += __shfl_xor_sync(kFullA, a2, o);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        sh[0][w] = a0;
        sh[1][w] = a1;
        sh[2][w] = a2;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double v = 0;
        for (int k = 0; k < kAdjT / 32; k++) v += sh[threadIdx.x][k];
        parts[3 * blockIdx.x + threadIdx.x] = v;
    }
}

// g_m, h_m and the explicit teleportation term sum_m g_m dq_m/dt (block partials).
__global__ void k_adj_mod2(int32_t n, const Stat4 *mstat, const double *q, double logQ, double *gm, double *hm,
                           double *parts) {
    __shared__ double sh[kAdjT / 32];
    double acc = 0;
    for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < n; m += (int64_t)gridDim.x * blockDim.x) {
        const Stat4 st = mstat[m];
        if (st.P == 0 && st.TW == 0) {
            gm[m] = 0.0;
            hm[m] = 0.0;
            continue;
        }
        const double P = from_fx(st.P), TW = from_fx(st.TW), D = from_fx(st.D), OUT = from_fx(st.OUT);
        const double e = q[m];
        const double g = logQ - 2.0 * dlog(e) + dlog(e + P);
        gm[m] = g;
        hm[m] = dlog(e + P) + 1.0;
        acc += g * ((1.0 - TW) * P - OUT - (1.0 - TW) * D);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFullA, acc, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 0;
        for (int k = 0; k < kAdjT / 32; k++) v += sh[k];
        parts[blockIdx.x] = v;
    }
}

__global__ void k_adj_c(int32_t n, const int32_t *part, const double *p, const double *cross, const uint8_t *dang,
                        const Stat4 *mstat, const double *gm, const double *hm, double alpha, double *c) {
    const double beta = 1.0 - alpha;
    for (int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; a < n; a += (int64_t)gridDim.x * blockDim.x) {
        const int32_t m = part[a];
        const double TW = from_fx(mstat[m].TW), g = gm[m];
        c[a] = g * (1.0 - TW) * (alpha + (dang[a] ? beta : 0.0)) + hm[m] - (dlog(p[a]) + 1.0) + beta * g * cross[a];
    }
}

template <int NT>
__device__ __forceinline__ double adj_block_sum(double v, double *sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFullA, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    if (w == 0) {
        t = lane < NT / 32 ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(kFullA, t, o);
    }
    __syncthreads();
    return t;
}

__device__ __forceinline__ double adj_sum_parts(const double *parts, int nb, double *sh) {
    if (threadIdx.x < 32) {
        double v = 0.0;
        for (int i = threadIdx.x; i < nb; i += 32) v += __ldcg(parts + i);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFullA, v, o);
        if (threadIdx.x == 0) sh[0] = v;
    }
    __syncthreads();
    const double r = sh[0];
    __syncthreads();
    return r;
}

// Rows of one degree class, W lanes per row (W <= 32), every warp of the grid
// taking 32/W rows at a time; rows of more than W links loop. Returns the
// thread's share of sum tw_r y_r over the rows it wrote.
template <int W>
__device__ __forceinline__ double adj_pull_rows(const int32_t *__restrict__ rows, int64_t lo, int64_t hi,
                                                const int64_t *__restrict__ off, const int32_t *__restrict__ dst,
                                                const double *__restrict__ w0, const double *__restrict__ rowsum,
                                                const uint8_t *__restrict__ dang, const double *__restrict__ c,
                                                const double *__restrict__ tw, double beta, double T, const double *x,
                                                double *y, int64_t gwarp, int64_t nwarps) {
    constexpr int RPW = 32 / W;
    const int lane = threadIdx.x & 31, sub = lane / W, lv = lane % W;
    double ts = 0.0;
    for (int64_t base = lo + gwarp * RPW; base < hi; base += nwarps * RPW) {
        const int64_t i = base + sub;
        double acc = 0.0;
        int32_t r = -1;
        if (i < hi) {
            r = rows[i];
            const int64_t e = off[r + 1];
            for (int64_t k = off[r] + lv; k < e; k += W) acc += w0[k] * __ldcg(x + dst[k]);
        }
#pragma unroll
        for (int o = W / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (r >= 0 && lv == 0) {
            const double s = rowsum[r];
            const double v = c[r] + beta * ((s > 0.0 ? acc / s : 0.0) + (dang[r] ? T : 0.0));
            y[r] = v;
            ts += tw[r] * v;
        }
    }
    return ts;
}

// The transposed solve lambda = c + beta (W~ lambda + d (tw . lambda)) as one
// cooperative launch, W~ the row-normalised out-links. Plain iteration
// converges only as beta^k: M = W~^T + tw d^T is column-stochastic, so the
// all-ones direction is an eigenvector of M^T with eigenvalue 1. The solution
// obeys one exact linear condition, tw . lambda = p . c / t (multiply the
// system by p^T and use p = beta M p + t tw), so after every sweep the iterate
// is shifted along the ones vector to meet it: a Wielandt deflation of that
// eigenvalue, leaving the contraction factor beta |lambda_2(M)| of the power
// iteration. The dangling term then always uses tw . lambda = p . c / t.
// Stops when the L1 change is below tol * L1 norm, or after max_iter sweeps.
// Out-degrees are heavy-tailed, so rows come grouped by degree class (rows[],
// class boundaries cls[0..7]: <= 1, 2, 4, 8, 16, 32 links, more), each class
// with its own lane width.
__global__ void __launch_bounds__(kAdjT, RMX_ADJ_MINB) k_adj_solve(const int64_t *__restrict__ off, const int32_t *__restrict__ dst,
                                                        const double *__restrict__ w0,
                                                        const double *__restrict__ rowsum,
                                                        const double *__restrict__ tw, const uint8_t *__restrict__ dang,
                                                        const double *__restrict__ c, const double *__restrict__ p,
                                                        int32_t n, double alpha, double *x, double *y, double *parts,
                                                        int max_iter, double tol, int *iters_out,
                                                        const int32_t *__restrict__ rows,
                                                        const int64_t *__restrict__ cls) {
    cg::grid_group grid = cg::this_grid();
    __shared__ double sh[32];
    const int nb = gridDim.x;
    const double beta = 1.0 - alpha;
    double *Sp = parts, *Ep = parts + nb, *Np = parts + 2 * nb;
    const int64_t gtid = (int64_t)blockIdx.x * kAdjT + threadIdx.x, gthreads = (int64_t)nb * kAdjT;
    double pc = 0.0, tc = 0.0;
    for (int64_t i = gtid; i < n; i += gthreads) {
        pc += p[i] * c[i];
        tc += tw[i] * c[i];
    }
    pc = adj_block_sum<kAdjT>(pc, sh);
    tc = adj_block_sum<kAdjT>(tc, sh);
    if (threadIdx.x == 0) {
        Sp[blockIdx.x] = pc;
        Ep[blockIdx.x] = tc;
    }
    grid.sync();
    const double target = adj_sum_parts(Sp, nb, sh) / alpha;  // tw . lambda at the solution
    const double d0 = target - adj_sum_parts(Ep, nb, sh);
    for (int64_t i = gtid; i < n; i += gthreads) x[i] = c[i] + d0;
    grid.sync();
    const int64_t gwarp = gtid >> 5, nwarps = gthreads >> 5;
    int64_t cb[8];
#pragma unroll
    for (int k = 0; k < 8; k++) cb[k] = cls[k];
    int iter = 0;
    for (;;) {
        double ts = 0.0;
        ts += adj_pull_rows<1>(rows, cb[0], cb[1], off, dst, w0, rowsum, dang, c, tw, beta, target, x, y, gwarp, nwarps);
        ts += adj_pull_rows<2 / RMX_ADJ_LPL>(rows, cb[1], cb[2], off, dst, w0, rowsum, dang, c, tw, beta, target, x, y,
                                             gwarp, nwarps);
        ts += adj_pull_rows<4 / RMX_ADJ_LPL>(rows, cb[2], cb[3], off, dst, w0, rowsum, dang, c, tw, beta, target, x, y,
                                             gwarp, nwarps);
        ts += adj_pull_rows<8 / RMX_ADJ_LPL>(rows, cb[3], cb[4], off, dst, w0, rowsum, dang, c, tw, beta, target, x, y,
                                             gwarp, nwarps);
        ts += adj_pull_rows<16 / RMX_ADJ_LPL>(rows, cb[4], cb[5], off, dst, w0, rowsum, dang, c, tw, beta, target, x, y,
                                              gwarp,
                                nwarps);
        ts += adj_pull_rows<32>(rows, cb[5], cb[7], off, dst, w0, rowsum, dang, c, tw, beta, target, x, y, gwarp,
                                nwarps);
        ts = adj_block_sum<kAdjT>(ts, sh);
        if (threadIdx.x == 0) Sp[blockIdx.x] = ts;
        grid.sync();
        const double shift = target - adj_sum_parts(Sp, nb, sh);
        double el = 0.0, nl = 0.0;
        for (int64_t i = gtid; i < n; i += gthreads) {
            const double v = __ldcg(y + i) + shift;
            el += fabs(v - x[i]);
            nl += fabs(v);
            x[i] = v;
        }
        el = adj_block_sum<kAdjT>(el, sh);
        nl = adj_block_sum<kAdjT>(nl, sh);
        if (threadIdx.x == 0) {
            Ep[blockIdx.x] = el;
            Np[blockIdx.x] = nl;
        }
        grid.sync();
        const double diff = adj_sum_parts(Ep, nb, sh), norm = adj_sum_parts(Np, nb, sh);
        iter++;
        if (iter >= max_iter || diff <= tol * norm) break;
    }
    if (gtid == 0) *iters_out = iter;
}

// dL/dw per link (CSR order): G = beta p_a (g_m [m(b) != m] + lambda_b), then
// through the row normalisation. Warp per row.
__global__ void k_adj_grad(int32_t n, const int64_t *off, const int32_t *dst, const double *w0, const double *rowsum,
                           const int32_t *part, const double *p, const double *gm, const double *lam, double beta,
                           double *grad) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t a = gw; a < n; a += nw) {
        const int64_t b0 = off[a], b1 = off[a + 1];
        if (b0 == b1) continue;
        const int32_t m = part[a];
        const double s = rowsum[a], bp = beta * p[a], g = gm[m];
        double r = 0.0;
        for (int64_t e = b0 + lane; e < b1; e += 32) {
            const int32_t b = dst[e];
            const double G = bp * ((part[b] != m ? g : 0.0) + lam[b]);
            r += (w0[e] / s) * G;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(kFullA, r, o);
        for (int64_t e = b0 + lane; e < b1; e += 32) {
            const int32_t b = dst[e];
            const double G = bp * ((part[b] != m ? g : 0.0) + lam[b]);
            grad[e] = (G - r) / s;
        }
    }
}

// Block partials of lambda . tw and lambda . p.
__global__ void k_adj_dots(int32_t n, const double *lam, const double *tw, const double *p, double *parts) {
    __shared__ double sh[2][kAdjT / 32];
    double a0 = 0, a1 = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        a0 += lam[i] * tw[i];
        a1 += lam[i] * p[i];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(kFullA, a0, o);
        a1 += __shfl_xor_sync(kFullA, a1, o);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        sh[0][w] = a0;
        sh[1][w] = a1;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        double v = 0;
        for (int k = 0; k < kAdjT / 32; k++) v += sh[threadIdx.x][k];
        parts[2 * blockIdx.x + threadIdx.x] = v;
    }
}

// Degree class of every row: 0..5 for <= 1, 2, 4, 8, 16, 32 links, 6 beyond.
__global__ void k_adj_classes(int32_t n, const int64_t *off, uint16_t *cls, int32_t *ids) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t d = off[r + 1] - off[r];
        int k = 0;
        while (k < 6 && d > (int64_t(1) << k)) k++;
        cls[r] = (uint16_t)k;
        ids[r] = (int32_t)r;
    }
}

int launch_solve(int32_t n, const int64_t *off, const int32_t *dst, const double *w0, const double *rowsum,
                 const double *tw, const uint8_t *dang, const double *c, const double *p, double alpha, double *x,
                 double *y, double *parts, int max_blocks, int max_iter, double tol, int *iters, Arena &ar,
                 cudaStream_t s) {
    int dev = 0, per_sm = 0;
    RMX_CUDA(cudaGetDevice(&dev));
    RMX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_adj_solve, kAdjT, 0));
    int nb = std::max(1, std::min(per_sm, RMX_ADJ_MINB)) * num_sms();
    nb = (int)std::min<int64_t>(nb, std::max<int64_t>(1, ((int64_t)n * 8 + kAdjT - 1) / kAdjT));
    nb = std::min(nb, max_blocks);
    size_t mk = ar.mark();
    uint16_t *cls = ar.alloc<uint16_t>(std::max(n, 1));
    int32_t *ids = ar.alloc<int32_t>(std::max(n, 1)), *rows = ar.alloc<int32_t>(std::max(n, 1));
    int64_t *bounds = ar.alloc<int64_t>(8);
    k_adj_classes<<<blocks_for(n, 256, num_sms() * 32), 256, 0, s>>>(n, off, cls, ids);
    RMX_LAUNCHED();
    bucket_partition(cls, ids, rows, n, 7, bounds, ar, s);
    void *args[] = {(void *)&off,   (void *)&dst,  (void *)&w0,       (void *)&rowsum, (void *)&tw,
                    (void *)&dang,  (void *)&c,    (void *)&p,        (void *)&n,      (void *)&alpha,
                    (void *)&x,     (void *)&y,    (void *)&parts,    (void *)&max_iter, (void *)&tol,
                    (void *)&iters, (void *)&rows, (void *)&bounds};
    RMX_CUDA(cudaLaunchCooperativeKernel((void *)k_adj_solve, dim3(nb), dim3(kAdjT), args, 0, s));
    RMX_LAUNCHED();
    int h = 0;
    RMX_CUDA(cudaMemcpyAsync(&h, iters, sizeof(int), cudaMemcpyDeviceToHost, s));
    RMX_CUDA(cudaStreamSynchronize(s));
    ar.release(mk);
    return h;
}

struct Workspace {
    Arena ar;
    explicit Workspace(size_t bytes) { ar.init(bytes); }
    ~Workspace() { ar.destroy(); }
};

}  // namespace
}  // namespace rmx

using namespace rmx;

// Forward (and, with grad != nullptr, backward) pass. The partition is
// validated on the host; the workspace is one device allocation of ~160 B per
// node + 8 B per link, released before returning.
void rmx_graph::adjoint(const int32_t *part_host, double tau, double *L_out, double *p_out, double *grad_out,
                        double *dL_dtau, int *solve_iters) {
    const NvtxRange range(grad_out || dL_dtau ? "rmx adjoint backward" : "rmx adjoint forward");
    if (!(tau > 0.0 && tau < 1.0)) throw std::invalid_argument("tau must lie in (0, 1)");
    for (int32_t v = 0; v < N; v++)
        if ((uint32_t)part_host[v] >= (uint32_t)N) throw std::invalid_argument("module id outside 0..N-1");
    initiate();  // row normalisation and the CSC the power iteration reads
    const int64_t Em = std::max<int64_t>(E, 1);
    const unsigned G = num_sms() * 4;
    const int kMaxBlocks = num_sms() * 4;
    Workspace ws((size_t)N * 160 + (size_t)Em * 8 + (size_t)G * 64 + (size_t)kMaxBlocks * 32 + (32u << 20));
    Arena &A = ws.ar;
    int32_t *part = A.alloc<int32_t>(N);
    double *pa = A.alloc<double>(N), *rowsum = A.alloc<double>(N), *cross = A.alloc<double>(N);
    Stat4 *mst = A.alloc<Stat4>(N);
    double *q = A.alloc<double>(N), *gm = A.alloc<double>(N), *hm = A.alloc<double>(N);
    double *parts = A.alloc<double>(3 * G + 3 * kMaxBlocks);
    fx_t *s0 = A.alloc<fx_t>(1);
    int *iters = A.alloc<int>(1);
    RMX_CUDA(cudaMemcpyAsync(part, part_host, sizeof(int32_t) * N, cudaMemcpyHostToDevice, stream));
    RMX_CUDA(cudaMemsetAsync(mst, 0, sizeof(Stat4) * N, stream));
    RMX_CUDA(cudaMemsetAsync(s0, 0, sizeof(fx_t), stream));
    power_iteration(N, in_off, in_src, in_w, tw, dangling, pa, A, stream, spmv_vec, tau);
    k_adj_rows<<<blocks_for((int64_t)N * 32, 256, num_sms() * 32), 256, 0, stream>>>(
        N, out_off, out_dst, out_w0, part, pa, tw, dangling, rowsum, cross, mst, s0);
    RMX_LAUNCHED();
    k_adj_mod1<<<G, kAdjT, 0, stream>>>(N, mst, tau, q, parts);
    RMX_LAUNCHED();
    std::vector<double> h(3 * G);
    fx_t s0h = 0;
    RMX_CUDA(cudaMemcpyAsync(h.data(), parts, sizeof(double) * 3 * G, cudaMemcpyDeviceToHost, stream));
    RMX_CUDA(cudaMemcpyAsync(&s0h, s0, sizeof(fx_t), cudaMemcpyDeviceToHost, stream));
    RMX_CUDA(cudaStreamSynchronize(stream));
    double Q = 0, sq = 0, sqp = 0;
    for (unsigned b = 0; b < G; b++) {
        Q += h[3 * b];
        sq += h[3 * b + 1];
        sqp += h[3 * b + 2];
    }
    const double plq = Q > 0.0 ? Q * std::log(Q) : 0.0;
    const double L = plq - 2.0 * sq + sqp - from_fxl(s0h);
    if (L_out) *L_out = L;
    if (p_out) RMX_CUDA(cudaMemcpyAsync(p_out, pa, sizeof(double) * N, cudaMemcpyDeviceToHost, stream));
    if (grad_out || dL_dtau) {
        const double beta = 1.0 - tau;
        k_adj_mod2<<<G, kAdjT, 0, stream>>>(N, mst, q, Q > 0.0 ? std::log(Q) : 0.0, gm, hm, parts);
        RMX_LAUNCHED();
        double *c = A.alloc<double>(N), *lam = A.alloc<double>(N), *lam2 = A.alloc<double>(N);
        k_adj_c<<<blocks_for(N, 256, num_sms() * 32), 256, 0, stream>>>(N, part, pa, cross, dangling, mst, gm, hm, tau,
                                                                        c);
        RMX_LAUNCHED();
        std::vector<double> ht(G);
        RMX_CUDA(cudaMemcpyAsync(ht.data(), parts, sizeof(double) * G, cudaMemcpyDeviceToHost, stream));
        RMX_CUDA(cudaStreamSynchronize(stream));
        double explicit_t = 0;
        for (unsigned b = 0; b < G; b++) explicit_t += ht[b];
        double *sp = parts + 3 * G;
        // deflated, the error falls as fast as in the power iteration
        const int max_iter = 4000;
        const double tol = 1e-15;
        int it = 0;
        timers.begin(kTimerAdjoint, stream);
        it = launch_solve(N, out_off, out_dst, out_w0, rowsum, tw, dangling, c, pa, tau, lam, lam2, sp, kMaxBlocks,
                          max_iter, tol, iters, A, stream);
        timers.end(kTimerAdjoint, stream);
        if (timers.on) prof.adjoint_iters += it;
        if (solve_iters) *solve_iters = it;
        // Stopped on the sweep cap: the adjoint, and every derivative taken
        // from it, is not within tolerance, so none is returned. (A solve that
        // met the tolerance on exactly the last sweep is reported the same way.)
        // The error falls by about (1 - tau) |lambda_2| per sweep, so this
        // happens for a small tau on a graph whose walk mixes slowly.
        if (it >= max_iter)
            throw NoConvergence("adjoint solve: the L1 change stayed above 1e-15 of the norm for " +
                                std::to_string(max_iter) + " sweeps (tau " + std::to_string(tau) +
                                " is too small for this graph's mixing)");
        if (grad_out) {
            double *grad = A.alloc<double>(Em);
            if (E > 0) {
                k_adj_grad<<<blocks_for((int64_t)N * 32, 256, num_sms() * 32), 256, 0, stream>>>(
                    N, out_off, out_dst, out_w0, rowsum, part, pa, gm, lam, beta, grad);
                RMX_LAUNCHED();
                RMX_CUDA(cudaMemcpyAsync(grad_out, grad, sizeof(double) * E, cudaMemcpyDeviceToHost, stream));
            }
        }
        if (dL_dtau) {
            k_adj_dots<<<G, kAdjT, 0, stream>>>(N, lam, tw, pa, parts);
            RMX_LAUNCHED();
            std::vector<double> hd(2 * G);
            RMX_CUDA(cudaMemcpyAsync(hd.data(), parts, sizeof(double) * 2 * G, cudaMemcpyDeviceToHost, stream));
            RMX_CUDA(cudaStreamSynchronize(stream));
            double lt = 0, lp = 0;
            for (unsigned b = 0; b < G; b++) {
                lt += hd[2 * b];
                lp += hd[2 * b + 1];
            }
            *dL_dtau = explicit_t + (lt - lp) / beta;
        }
    }
    RMX_CUDA(cudaStreamSynchronize(stream));
}
