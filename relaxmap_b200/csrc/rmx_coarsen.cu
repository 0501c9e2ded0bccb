// Coarsening: Network::convertModulesToSuperNodes (Module.cpp:3008-3077) and
// the link aggregation of generateSuperNodesFromSubModules (Module.cpp:3103-3157).
//
// The reference builds, per super-node, a std::map keyed by destination
// super-node, inserting the member nodes' out-links in node order and link
// order, and then appends in-links in ascending source order. Here:
//   1. every node link u->w with group(u) != group(w) gets the key
//      (group(u), group(w)); links are compacted in CSR order,
//   2. a stable LSD radix sort by that key groups equal pairs while keeping
//      their original (u, w) order,
//   3. one thread per distinct pair sums its run sequentially in that order,
//      which is exactly the reference's summation order (bit-identical FP64),
//      and also sums the fixed-point flows used by the move engine,
//   4. rows come out sorted by destination; a stable sort of the pair list by
//      destination gives the in-links in ascending source order.
#include <algorithm>

#include "rmx_engine.cuh"

namespace rmx {

static int bits_for(int64_t n) {
    int b = 1;
    while ((int64_t(1) << b) < n) b++;
    return b;
}

__global__ void k_cross_flags(int32_t n, const int64_t *off, const int32_t *dst, const int32_t *group,
                              uint8_t *flag) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t u = gw; u < n; u += nw) {
        const int32_t a = group[u];
        for (int64_t e = off[u] + lane; e < off[u + 1]; e += 32) flag[e] = group[dst[e]] != a ? 1 : 0;
    }
}

// src of link e is found by binary search in off (links are compacted, so a
// per-row pass cannot index them directly).
__device__ __forceinline__ int32_t row_of(const int64_t *off, int32_t n, int64_t e) {
    int32_t lo = 0, hi = n - 1;
    while (lo < hi) {
        int32_t mid = lo + ((hi - lo + 1) >> 1);
        if (off[mid] <= e)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

__global__ void k_pair_keys(const int32_t *idx, const int64_t *count, int32_t n, const int64_t *off,
                            const int32_t *dst, const int32_t *group, int b, uint64_t *keys, uint32_t *vals) {
    const int64_t C = *count;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < C; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = idx[i];
        const int32_t u = row_of(off, n, e);
        keys[i] = ((uint64_t)(uint32_t)group[u] << b) | (uint32_t)group[dst[e]];
        vals[i] = (uint32_t)e;
    }
}

__global__ void k_pair_heads(const uint64_t *keys, const int64_t *count, uint8_t *flag) {
    const int64_t C = *count;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < C; i += (int64_t)gridDim.x * blockDim.x)
        flag[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

__global__ void k_pair_sums(const uint64_t *keys, const uint32_t *vals, const int32_t *head, const int64_t *n_heads,
                            const int64_t *count, int b, const double *f, const fx_t *fx, int32_t *g_src,
                            int32_t *g_dst, double *g_f, fx_t *g_fx, unsigned long long *row_count) {
    const int64_t H = *n_heads, C = *count;
    const uint64_t mask = (uint64_t(1) << b) - 1;
    for (int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; h < H; h += (int64_t)gridDim.x * blockDim.x) {
        const int64_t beg = head[h], end = (h + 1 < H) ? head[h + 1] : C;
        fx_t q = 0;
        if (g_f) {
            double s = f[vals[beg]];  // first insert, then += in order (Module.cpp:3055-3057)
            for (int64_t j = beg + 1; j < end; j++) s += f[vals[j]];
            g_f[h] = s;
        }
        for (int64_t j = beg; j < end; j++) q += fx[vals[j]];
        const uint64_t k = keys[beg];
        const int32_t a = (int32_t)(k >> b);
        g_src[h] = a;
        g_dst[h] = (int32_t)(k & mask);
        g_fx[h] = q;
        atomicAdd(row_count + a, 1ull);
    }
}

__global__ void k_col_keys(const int32_t *g_dst, int64_t m, uint64_t *keys, uint32_t *vals, unsigned long long *cnt) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        keys[i] = (uint64_t)(uint32_t)g_dst[i];
        vals[i] = (uint32_t)i;
        atomicAdd(cnt + g_dst[i], 1ull);
    }
}

__global__ void k_col_gather(const uint32_t *perm, int64_t m, const int32_t *g_src, const double *g_f,
                             const fx_t *g_fx, int32_t *in_src, double *in_f, fx_t *in_fx) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t j = perm[i];
        in_src[i] = g_src[j];
        if (in_f) in_f[i] = g_f[j];
        in_fx[i] = g_fx[j];
    }
}

int64_t coarsen_links(int32_t n, const int64_t *out_off, const int32_t *out_dst, const double *out_f,
                      const fx_t *out_fx, const int32_t *group, int32_t ng, int64_t *g_out_off, int32_t *g_out_dst,
                      double *g_out_f, fx_t *g_out_fx, int64_t *g_in_off, int32_t *g_in_src, double *g_in_f,
                      fx_t *g_in_fx, Arena &ar, cudaStream_t s) {
    RMX_CUDA(cudaMemsetAsync(g_out_off, 0, sizeof(int64_t) * (ng + 1), s));
    RMX_CUDA(cudaMemsetAsync(g_in_off, 0, sizeof(int64_t) * (ng + 1), s));
    int64_t E = 0;
    RMX_CUDA(cudaMemcpyAsync(&E, out_off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RMX_CUDA(cudaStreamSynchronize(s));
    if (E == 0 || ng <= 1) return 0;
    size_t mk = ar.mark();
    const int b = bits_for(std::max<int64_t>(ng, 2));
    const unsigned G = num_sms() * 16;
    uint8_t *flag = ar.alloc<uint8_t>(E);
    k_cross_flags<<<G, 256, 0, s>>>(n, out_off, out_dst, group, flag);
    RMX_LAUNCHED();
    int32_t *idx = ar.alloc<int32_t>(E);
    int64_t *cnt = ar.alloc<int64_t>(4);
    compact_flags(flag, E, idx, cnt + 0, ar, s);
    int64_t C = 0;
    RMX_CUDA(cudaMemcpyAsync(&C, cnt + 0, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RMX_CUDA(cudaStreamSynchronize(s));
    if (C == 0) {
        ar.release(mk);
        return 0;
    }
    uint64_t *keys = ar.alloc<uint64_t>(C), *keys2 = ar.alloc<uint64_t>(C);
    uint32_t *vals = ar.alloc<uint32_t>(C), *vals2 = ar.alloc<uint32_t>(C);
    k_pair_keys<<<G, 256, 0, s>>>(idx, cnt + 0, n, out_off, out_dst, group, b, keys, vals);
    RMX_LAUNCHED();
    radix_sort_pairs(keys, vals, keys2, vals2, C, 2 * b, ar, s);
    k_pair_heads<<<G, 256, 0, s>>>(keys, cnt + 0, flag);
    RMX_LAUNCHED();
    int32_t *head = idx;  // idx is dead after the keys were built
    compact_flags(flag, C, head, cnt + 1, ar, s);
    int32_t *g_src = ar.alloc<int32_t>(C);
    k_pair_sums<<<G, 256, 0, s>>>(keys, vals, head, cnt + 1, cnt + 0, b, out_f, out_fx, g_src, g_out_dst, g_out_f,
                                  g_out_fx, reinterpret_cast<unsigned long long *>(g_out_off));
    RMX_LAUNCHED();
    int64_t H = 0;
    RMX_CUDA(cudaMemcpyAsync(&H, cnt + 1, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RMX_CUDA(cudaStreamSynchronize(s));
    scan_exclusive(g_out_off, g_out_off, ng + 1, nullptr, ar, s);
    k_col_keys<<<G, 256, 0, s>>>(g_out_dst, H, keys, vals, reinterpret_cast<unsigned long long *>(g_in_off));
    RMX_LAUNCHED();
    radix_sort_pairs(keys, vals, keys2, vals2, H, b, ar, s);
    k_col_gather<<<G, 256, 0, s>>>(vals, H, g_src, g_out_f, g_out_fx, g_in_src, g_in_f, g_in_fx);
    RMX_LAUNCHED();
    scan_exclusive(g_in_off, g_in_off, ng + 1, nullptr, ar, s);
    ar.release(mk);
    return H;
}

}  // namespace rmx
