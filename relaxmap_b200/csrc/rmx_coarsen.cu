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
#include <climits>
#include <mutex>
#include <vector>

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

// ---------------------------------------------------------------------------
// Engine aggregation by hashing (fixed-point flows only).
//
// The move engine needs the group links' fixed-point sums, which are exact in
// any order, and it never depends on the order of links inside a row. So
// instead of sorting every crossing link:
//   1. each group's capacity (its members' links) is counted and scanned;
//   2. one pass over the links in CSR order (every link's row is known)
//      gathers each crossing link's (destination group, flow) into its
//      source group's range, in no particular order;
//   3. one warp (small groups), one block (large groups) or the split
//      pipeline (huge groups) per group sums the range in a hash table keyed
//      by the destination group and writes the distinct destinations back
//      to the start of the range;
//   4. the rows are packed (teams of 8 lanes per row, a block per long row),
//      every packed link's row written beside it, and transposed by a
//      counting sort on the destination (each link placed as one 16-byte
//      (row, flow) record, then split into the CSC arrays in order).
// No pass searches for the row of a link or walks a group's members.
namespace rmx {

constexpr unsigned kFullMask = 0xffffffffu;
constexpr int32_t kNoKey = -1;
constexpr int kAggWarpLinks = 128, kAggWarpCap = 256, kAggWarps = 8;
constexpr int kAggMidT = 128, kAggMidLinks = 1024, kAggMidCap = 2048;
constexpr int kAggT = 512, kAggCap = 8192;
// groups of more member links than this are split over many blocks (k_hg_*)
constexpr int64_t kAggSplit = 16384;
constexpr int kHgCh = 2048;  // links per chunk item (the mean links per partition is the hub_part tuning)

__device__ __forceinline__ uint32_t agg_hash(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

// Slot of key (inserted if absent; fresh = it was absent), or -1 if the table is full.
__device__ __forceinline__ int agg_insert(int32_t *keys, int mask, int32_t key, bool &fresh) {
    int s = (int)(agg_hash((uint32_t)key) & (uint32_t)mask);
    for (int probe = 0; probe <= mask; probe++) {
        const int32_t prev = atomicCAS(keys + s, kNoKey, key);
        if (prev == kNoKey || prev == key) {
            fresh = prev == kNoKey;
            return s;
        }
        s = (s + 1) & mask;
    }
    return -1;
}

__global__ void k_rows_of_links(int32_t n, const int64_t *off, int32_t *src) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = gw; r < n; r += nw)
        for (int64_t e = off[r] + lane; e < off[r + 1]; e += 32) src[e] = (int32_t)r;
}

void rows_of_links(int32_t n, const int64_t *off, int32_t *src, cudaStream_t s) {
    k_rows_of_links<<<blocks_for((int64_t)n * 32, 256, num_sms() * 32), 256, 0, s>>>(n, off, src);
    RMX_LAUNCHED();
}

// glinks[g]: links of g's members (the capacity of g's range).
__global__ void k_agg_count(int32_t n, const int64_t *off, const int32_t *group, unsigned long long *glinks) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t d = off[r + 1] - off[r];
        if (d) atomicAdd(glinks + group[r], (unsigned long long)d);
    }
}

// Every crossing link u->w (group(u) != group(w)) appended to group(u)'s
// range: gk = group(w), gq = its flow; gcross[g] counts them. Lanes of a warp
// with the same source group (consecutive links of one row, mostly) take
// their positions with one counter update.
__global__ void k_agg_gather(int64_t m, const int32_t *src, const int32_t *dst, const fx_t *fx, const int32_t *group,
                             const int64_t *gloff, unsigned long long *gcross, int32_t *gk, fx_t *gq) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t e0 = gw * 32; e0 < m; e0 += nw * 32) {  // warp-uniform
        const int64_t e = e0 + lane;
        int32_t g = -1, b = -1;
        fx_t q = 0;
        if (e < m) {
            g = __ldg(group + __ldcs(src + e));  // links streamed, group ids kept in L2
            b = __ldg(group + __ldcs(dst + e));
            q = __ldcs(fx + e);
            if (b == g) g = -1;  // links inside a group are not kept
        }
        const unsigned peers = __match_any_sync(kFullMask, g);
        const int leader = __ffs(peers) - 1;
        unsigned long long base = 0;
        if (g >= 0 && lane == leader) base = atomicAdd(gcross + g, (unsigned long long)__popc(peers));
        base = __shfl_sync(kFullMask, base, leader);
        if (g >= 0) {
            const int64_t p = gloff[g] + (int64_t)base + __popc(peers & ((1u << lane) - 1u));
            gk[p] = b;
            gq[p] = q;
        }
    }
}

// Groups by the bound on their distinct neighbours, min(crossing links,
// groups): a warp (<= 128), a 128-thread block (<= 1024) or a 512-thread
// block; groups of more than kAggSplit crossing links go to the split
// pipeline instead (groups without one go nowhere). maxlinks: the most links
// of a group outside it; htot: the split pipeline's links, chunks and
// partitions.
__global__ void k_agg_bins(int32_t ng, const unsigned long long *gcross, int64_t part_links, uint8_t *small,
                           uint8_t *mid, uint8_t *large, uint8_t *huge, unsigned long long *maxlinks,
                           unsigned long long *htot) {
    unsigned long long mx = 0, hl = 0, hc = 0, hp = 0;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < ng; g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t l = (int64_t)gcross[g], b = min(l, (int64_t)ng);
        const bool hg = l > kAggSplit;
        small[g] = !hg && b > 0 && b <= kAggWarpLinks ? 1 : 0;
        mid[g] = !hg && b > kAggWarpLinks && b <= kAggMidLinks ? 1 : 0;
        large[g] = !hg && b > kAggMidLinks ? 1 : 0;
        huge[g] = hg ? 1 : 0;
        if (hg) {
            hl += l;
            hc += (l + kHgCh - 1) / kHgCh;
            hp += (l + part_links - 1) / part_links;
        } else {
            mx = max(mx, (unsigned long long)l);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        mx = max(mx, __shfl_xor_sync(kFullMask, mx, o));
        hl += __shfl_xor_sync(kFullMask, hl, o);
        hc += __shfl_xor_sync(kFullMask, hc, o);
        hp += __shfl_xor_sync(kFullMask, hp, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (mx) atomicMax(maxlinks, mx);
        if (hl) {
            atomicAdd(htot, hl);
            atomicAdd(htot + 1, hc);
            atomicAdd(htot + 2, hp);
        }
    }
}

struct AggArgs {
    const int64_t *gloff;                 // start of each group's range
    const unsigned long long *gcross;     // crossing links gathered into it
    int32_t *slab_dst;  // the ranges: gathered links in, distinct destinations out (at the same start)
    fx_t *slab_fx;
    int64_t *rowlen;
    fx_t *rowsum;        // optional: sum of the row's flows (out-flow of the group)
    const int32_t *list; // groups of this bin
    const int64_t *count;
    int32_t *gkeys;      // global tables for groups too large for shared memory
    fx_t *gvals;
    int64_t gcap;
    int32_t ngroups;
};

// One group by a team of NT threads (r = rank); keys/vals: a table of cap
// slots. A table sized below twice the group's link count may hold at most
// `limit` distinct keys: past that the group is abandoned (returns false,
// uniformly across the team) and nothing of it is written. wsh: NT/32 + 3
// ints (block teams only). The team strides the group's gathered range, four
// links per thread loaded before any is inserted.
template <int NT>
__device__ __forceinline__ bool agg_group(const AggArgs &a, int32_t g, int r, int32_t *keys, fx_t *vals, int64_t cap,
                                          int limit, int *wsh) {
    constexpr int ILP = 4;
    const int lane = r & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int mask = (int)(cap - 1);
    int *nkeys = wsh ? wsh + NT / 32 + 1 : nullptr;
    for (int64_t s = r; s < cap; s += NT) {
        keys[s] = kNoKey;
        vals[s] = 0;
    }
    if (NT > 32 && r == 0) *nkeys = 0;
    if (NT == 32) __syncwarp(); else __syncthreads();
    const int64_t b0 = a.gloff[g], b1 = b0 + (int64_t)a.gcross[g];
    for (int64_t j0 = b0 + r; j0 < b1; j0 += (int64_t)NT * ILP) {
        if (NT > 32 && *(volatile int *)nkeys > limit) break;
        int32_t key[ILP];
        fx_t q[ILP];
#pragma unroll
        for (int k = 0; k < ILP; k++) {
            const int64_t j = j0 + (int64_t)k * NT;
            key[k] = j < b1 ? a.slab_dst[j] : kNoKey;
            q[k] = j < b1 ? a.slab_fx[j] : 0;
        }
        bool full = false;
#pragma unroll
        for (int k = 0; k < ILP; k++) {
            if (key[k] == kNoKey || full) continue;
            bool fresh;
            const int s = agg_insert(keys, mask, key[k], fresh);
            if (s < 0) {  // only a table sized below the bound can fill up; nkeys > limit already
                full = true;
                continue;
            }
            if (NT > 32 && fresh) atomicAdd(nkeys, 1);
            atomicAdd(reinterpret_cast<unsigned long long *>(vals + s), (unsigned long long)q[k]);
        }
        if (full) break;
    }
    if (NT == 32) __syncwarp(); else __syncthreads();
    if (NT > 32 && *nkeys > limit) {
        __syncthreads();  // every thread has read the count before the next group resets it
        return false;
    }
    // pack the occupied slots into the group's slab: every warp counts its own
    // contiguous slice, a scan over the warps gives the offsets, then writes
    const int64_t base_out = a.gloff[g];
    const int64_t seg = cap / (NT / 32), lo = (int64_t)(r >> 5) * seg, hi = lo + seg;
    int cnt = 0;
    for (int64_t base = lo; base < hi; base += 32) {
        const int64_t s = base + lane;
        cnt += __popc(__ballot_sync(kFullMask, s < hi && keys[s] != kNoKey));
    }
    int woff = 0, nout = cnt;
    if (NT > 32) {
        if (lane == 0) wsh[r >> 5] = cnt;
        __syncthreads();
        if (r < 32) {
            int x = r < NT / 32 ? wsh[r] : 0;
            const int own = x;
#pragma unroll
            for (int q = 1; q < 32; q <<= 1) {
                const int y = __shfl_up_sync(kFullMask, x, q);
                if (r >= q) x += y;
            }
            if (r < NT / 32) wsh[r] = x - own;
            if (r == 31) wsh[NT / 32] = x;
        }
        __syncthreads();
        woff = wsh[r >> 5];
        nout = wsh[NT / 32];
    }
    fx_t sum = 0;
    int done = 0;
    for (int64_t base = lo; base < hi; base += 32) {
        const int64_t s = base + lane;
        const int32_t k = s < hi ? keys[s] : kNoKey;
        const bool occ = k != kNoKey;
        const unsigned bal = __ballot_sync(kFullMask, occ);
        if (occ) {
            const int64_t p = base_out + woff + done + __popc(bal & lt);
            a.slab_dst[p] = k;
            a.slab_fx[p] = vals[s];
            sum += vals[s];
        }
        done += __popc(bal);
    }
    if (a.rowsum) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(kFullMask, sum, o);
        if (lane == 0 && sum) atomicAdd(reinterpret_cast<unsigned long long *>(a.rowsum + g), (unsigned long long)sum);
    }
    if (r == 0) a.rowlen[g] = nout;
    if (NT == 32) __syncwarp(); else __syncthreads();
    return true;
}

__global__ void __launch_bounds__(kAggWarps * 32) k_agg_warp(AggArgs a) {
    __shared__ int32_t skeys[kAggWarps][kAggWarpCap];
    __shared__ fx_t svals[kAggWarps][kAggWarpCap];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t n = *a.count;
    for (int64_t i = (int64_t)blockIdx.x * kAggWarps + w; i < n; i += (int64_t)gridDim.x * kAggWarps) {
        const int32_t g = a.list[i];
        const int64_t bound = min((int64_t)a.gcross[g], (int64_t)a.ngroups);
        int64_t cap = 32;
        while (cap < 2 * bound) cap <<= 1;
        agg_group<32>(a, g, lane, skeys[w], svals[w], cap, INT_MAX, nullptr);
    }
}

__global__ void __launch_bounds__(kAggMidT) k_agg_mid(AggArgs a) {
    __shared__ int32_t skeys[kAggMidCap];
    __shared__ fx_t svals[kAggMidCap];
    __shared__ int wsh[kAggMidT / 32 + 3];
    const int64_t n = *a.count;
    for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
        const int32_t g = a.list[i];
        const int64_t bound = min((int64_t)a.gcross[g], (int64_t)a.ngroups);
        int64_t cap = 64;
        while (cap < 2 * bound) cap <<= 1;
        agg_group<kAggMidT>(a, g, threadIdx.x, skeys, svals, cap, INT_MAX, wsh);
    }
}

// Large groups: distinct destination groups are usually far fewer than links
// (most links of a module go to a few neighbours), so every group first tries
// the shared-memory table, kept at most 3/4 full, and only a group with more
// distinct neighbours than that is redone in a global slice sized by its links.
__global__ void __launch_bounds__(kAggT, 2) k_agg_block(AggArgs a) {
    extern __shared__ __align__(16) unsigned char dsm[];
    __shared__ int wsh[kAggT / 32 + 3];
    fx_t *svals = reinterpret_cast<fx_t *>(dsm);
    int32_t *skeys = reinterpret_cast<int32_t *>(svals + kAggCap);
    const int64_t n = *a.count;
    for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
        const int32_t g = a.list[i];
        const int64_t bound = min((int64_t)a.gcross[g], (int64_t)a.ngroups);
        int64_t cap = 64;
        while (cap < 2 * bound) cap <<= 1;
        if (cap <= kAggCap) {
            agg_group<kAggT>(a, g, threadIdx.x, skeys, svals, cap, INT_MAX, wsh);
        } else if (!agg_group<kAggT>(a, g, threadIdx.x, skeys, svals, kAggCap, kAggCap / 4 * 3, wsh)) {
            agg_group<kAggT>(a, g, threadIdx.x, a.gkeys + (int64_t)blockIdx.x * a.gcap,
                             a.gvals + (int64_t)blockIdx.x * a.gcap, cap, INT_MAX, wsh);
        }
    }
}

// ---------------------------------------------------------------------------
// Huge groups (more than kAggSplit crossing links: the modules around R-MAT
// hubs, up to millions of links) are not left to one block. Their gathered
// ranges are cut into chunks of kHgCh links and radix-partitioned by a hash
// of the destination group into partitions of about part_links links, so that
// each partition's distinct destinations fit one block's shared table:
//   plan     one block: chunk and partition offsets per huge group
//   count    blocks take chunks (finding each chunk's group once and listing
//            it, and every partition's group) and count each partition's
//            elements
//   offsets  one block turns the counts into bucket offsets
//   scatter  blocks take chunks again and write (destination, flow)
//   reduce   a block per partition sums its bucket in a shared table and
//            appends the distinct destinations to the group's row
// Lanes of a warp that reach the same destination are combined with
// __match_any_sync before any counter update or bucket write (a hub's links
// concentrate on a few large groups); both link passes form the same groups.
constexpr int kHgT = 256, kHgCap = 4096;
constexpr size_t kHgSmem = (size_t)kHgCap * (sizeof(fx_t) + sizeof(int32_t));

struct HugeArgs {
    const int64_t *gloff;                // start of each group's gathered range
    const unsigned long long *gcross;    // its crossing links
    const int32_t *hlist;   // huge groups, ascending
    const int64_t *nh;      // their count (device)
    int64_t *coff, *poff;   // per huge group (+1): first chunk, first partition
    int32_t *cgrp;          // per chunk: huge group
    int32_t *pgrp;          // per partition: huge group
    unsigned long long *pcnt;  // per partition: elements (counted), then the fill position
    int64_t *pstart;        // per partition (+1): first bucket element
    int32_t *bkey;          // bucket elements: destination group
    fx_t *bfx;              //   and flow
    int64_t *tot;           // [0] chunks [1] partitions [2] over capacity
    int64_t max_chunks, max_parts, max_links;
    int64_t part_links;     // mean links per partition
    int32_t *slab_dst;      // the gathered ranges (read by the link passes, written by the reduction)
    fx_t *slab_fx;
    int64_t *rowlen;
    fx_t *rowsum;
};

__device__ __forceinline__ uint32_t hg_part_hash(int32_t key) {
    return agg_hash((uint32_t)key * 0x9E3779B1u + 0x7F4A7C15u);
}

// Exclusive scan over the block (blockDim.x == 1024) of one value per thread.
__device__ __forceinline__ long long hg_block_scan(long long v, long long *ws, long long *total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(kFullMask, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    if (w == 0) {
        long long t = ws[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long y = __shfl_up_sync(kFullMask, t, o);
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

// Largest j < n with off[j] <= x (off ascending, off[0] <= x).
template <typename T>
__device__ __forceinline__ int32_t hg_find(const T *off, int32_t n, int64_t x) {
    int32_t lo = 0, hi = n - 1;
    while (lo < hi) {
        const int32_t mid = lo + ((hi - lo + 1) >> 1);
        if ((int64_t)off[mid] <= x)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(1024) k_hg_plan(HugeArgs a) {
    __shared__ long long ws[32];
    __shared__ int over;
    const int64_t nh = *a.nh;
    long long r0 = 0, r1 = 0;
    for (int64_t base = 0; base < nh; base += 1024) {
        const int64_t h = base + threadIdx.x;
        long long nch = 0, np = 0;
        if (h < nh) {
            const int64_t l = (int64_t)a.gcross[a.hlist[h]];
            nch = (l + kHgCh - 1) / kHgCh;
            np = max(1ll, (long long)((l + a.part_links - 1) / a.part_links));
        }
        long long t0, t1;
        const long long e0 = hg_block_scan(nch, ws, &t0);
        const long long e1 = hg_block_scan(np, ws, &t1);
        if (h < nh) {
            a.coff[h] = r0 + e0;
            a.poff[h] = r1 + e1;
        }
        r0 += t0;
        r1 += t1;
    }
    if (threadIdx.x == 0) {
        over = r0 > a.max_chunks || r1 > a.max_parts;
        a.coff[nh] = r0;
        a.poff[nh] = r1;
        a.tot[0] = over ? 0 : r0;
        a.tot[1] = over ? 0 : r1;
        a.tot[2] = over;
    }
    __syncthreads();
    if (!over)
        for (int64_t q = threadIdx.x; q < r1; q += 1024) a.pcnt[q] = 0;
}

// Count (SCATTER false) or place (SCATTER true) the links of the chunks.
template <bool SCATTER>
__global__ void __launch_bounds__(kHgT) k_hg_links(HugeArgs a) {
    __shared__ fx_t wq[kHgT];
    const int lane = threadIdx.x & 31;
    const int64_t total = a.tot[0];
    const int32_t nh = (int32_t)*a.nh;
    for (int64_t item = blockIdx.x; item < total; item += gridDim.x) {
        const int32_t h = SCATTER ? a.cgrp[item] : hg_find(a.coff, nh, item);
        const int32_t g = a.hlist[h];
        const int64_t np = a.poff[h + 1] - a.poff[h];
        const int64_t c0 = (item - a.coff[h]) * kHgCh;
        const int64_t P0 = a.gloff[g] + c0, P1 = a.gloff[g] + min((int64_t)a.gcross[g], c0 + kHgCh);
        if (!SCATTER) {
            if (threadIdx.x == 0) a.cgrp[item] = h;
            if (c0 == 0)
                for (int64_t q = threadIdx.x; q < np; q += kHgT) a.pgrp[a.poff[h] + q] = h;
        }
        for (int64_t b0 = P0; b0 < P1; b0 += kHgT) {  // uniform over the block
            const int64_t V = b0 + threadIdx.x;
            int32_t key = -1;  // lanes past the chunk
            fx_t q = 0;
            if (V < P1) {
                key = a.slab_dst[V];
                q = a.slab_fx[V];
            }
            const bool valid = key >= 0;
            const unsigned kpeers = __match_any_sync(kFullMask, valid ? key : -1);
            const bool head = valid && lane == __ffs(kpeers) - 1;
            const int32_t part = head ? (int32_t)(hg_part_hash(key) % (uint32_t)np) : -1;
            const unsigned peers = __match_any_sync(kFullMask, part);
            const int leader = __ffs(peers) - 1;
            if (!SCATTER) {
                if (head && lane == leader)
                    atomicAdd(a.pcnt + a.poff[h] + part, (unsigned long long)__popc(peers));
            } else {
                wq[threadIdx.x] = q;
                __syncwarp();
                fx_t sum = 0;
                if (head)
                    for (unsigned m = kpeers; m; m &= m - 1) sum += wq[(threadIdx.x & ~31) + __ffs(m) - 1];
                unsigned long long base = 0;
                const int64_t pidx = a.poff[h] + part;
                if (head && lane == leader) base = atomicAdd(a.pcnt + pidx, (unsigned long long)__popc(peers));
                base = __shfl_sync(kFullMask, base, leader);
                if (head) {
                    const int64_t pos = a.pstart[pidx] + (int64_t)base + __popc(peers & ((1u << lane) - 1u));
                    a.bkey[pos] = key;
                    a.bfx[pos] = sum;
                }
                __syncwarp();
            }
        }
    }
}

__global__ void __launch_bounds__(1024) k_hg_offsets(HugeArgs a) {
    __shared__ long long ws[32];
    const int64_t np = a.tot[1];
    long long r = 0;
    for (int64_t base = 0; base < np; base += 1024) {
        const int64_t q = base + threadIdx.x;
        const long long c = q < np ? (long long)a.pcnt[q] : 0;
        long long t;
        const long long e = hg_block_scan(c, ws, &t);
        if (q < np) {
            a.pstart[q] = r + e;
            a.pcnt[q] = 0;
        }
        r += t;
    }
    if (threadIdx.x == 0) a.pstart[np] = r;
}

// A block per partition: its bucket summed in a shared table and the distinct
// destinations appended to the group's row. A bucket with more distinct
// destinations than half the table is taken in subsets: subset (R, r) holds
// the keys whose second hash h2 (a bijection of the key) has h2 mod R == r;
// a subset that overfills the table is emptied unwritten and replaced by its
// two halves (2R, r) and (2R, r + R). Every key lands in exactly one written
// subset, and a subset of R = 2^31 holds at most two keys, so this ends.
__device__ __forceinline__ uint32_t hg_split_hash(int32_t key) { return agg_hash((uint32_t)key ^ 0x5bd1e995u); }

__global__ void __launch_bounds__(kHgT, 2) k_hg_reduce(HugeArgs a) {
    extern __shared__ __align__(16) unsigned char hg_smem[];  // kHgSmem bytes
    fx_t *vals = reinterpret_cast<fx_t *>(hg_smem);
    int32_t *keys = reinterpret_cast<int32_t *>(vals + kHgCap);
    __shared__ int16_t taken[kHgCap / 2 + kHgT];
    __shared__ int nfresh;
    __shared__ unsigned long long obase;
    const int mask = kHgCap - 1;
    const int64_t total = a.tot[1];
    for (int s = threadIdx.x; s < kHgCap; s += kHgT) {
        keys[s] = kNoKey;
        vals[s] = 0;
    }
    fx_t rsum = 0;
    for (int64_t pidx = blockIdx.x; pidx < total; pidx += gridDim.x) {
        const int32_t h = a.pgrp[pidx], g = a.hlist[h];
        const int64_t b0 = a.pstart[pidx], b1 = a.pstart[pidx + 1];
        uint32_t stR[33], str[33];  // subsets still to take (uniform across the block)
        int sp = 0;
        stR[sp] = 1;
        str[sp++] = 0;
        while (sp > 0) {
            sp--;
            const uint32_t R = stR[sp], r = str[sp];
            __syncthreads();
            if (threadIdx.x == 0) nfresh = 0;
            __syncthreads();
            for (int64_t e = b0 + threadIdx.x; e < b1; e += kHgT) {
                const int32_t key = a.bkey[e];
                if (R > 1 && (hg_split_hash(key) & (R - 1)) != r) continue;
                if (*(volatile int *)&nfresh > kHgCap / 2) break;
                bool fresh;
                const int sl = agg_insert(keys, mask, key, fresh);
                if (sl < 0) continue;  // unreachable: at most kHgCap / 2 + kHgT keys are inserted
                if (fresh) taken[atomicAdd(&nfresh, 1)] = (int16_t)sl;
                atomicAdd(reinterpret_cast<unsigned long long *>(vals + sl), (unsigned long long)a.bfx[e]);
            }
            __syncthreads();
            const int nt = nfresh;
            const bool overfull = nt > kHgCap / 2;
            if (!overfull && threadIdx.x == 0)
                obase = atomicAdd(reinterpret_cast<unsigned long long *>(a.rowlen + g), (unsigned long long)nt);
            __syncthreads();
            for (int i = threadIdx.x; i < nt; i += kHgT) {
                const int sl = taken[i];
                if (!overfull) {
                    const int64_t pos = a.gloff[g] + (int64_t)obase + i;
                    a.slab_dst[pos] = keys[sl];
                    a.slab_fx[pos] = vals[sl];
                    rsum += vals[sl];
                }
                keys[sl] = kNoKey;
                vals[sl] = 0;
            }
            if (overfull) {  // its two halves, the lower one taken first
                stR[sp] = 2 * R;
                str[sp++] = r + R;
                stR[sp] = 2 * R;
                str[sp++] = r;
            }
        }
        if (a.rowsum) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) rsum += __shfl_xor_sync(kFullMask, rsum, o);
            if ((threadIdx.x & 31) == 0 && rsum)
                atomicAdd(reinterpret_cast<unsigned long long *>(a.rowsum + g), (unsigned long long)rsum);
        }
        rsum = 0;
    }
}

// Packed rows: the distinct destinations of row g (at gloff[g]) move to the
// CSR position g_out_off[g], each with its row beside it; columns are counted
// for the transpose (one counter update per destination and warp: hub
// columns take many links). Teams of kPackTeam lanes take a row each; rows
// longer than kPackLong are listed, in chunks of kPackChunk entries, for
// k_agg_pack_long.
constexpr int kPackTeam = 8, kPackLong = 512, kPackChunk = 8192;

__device__ __forceinline__ void pack_link(int64_t i, int64_t len, int64_t from, int64_t to, int32_t g,
                                          const int32_t *slab_dst, const fx_t *slab_fx, int32_t *out_dst,
                                          fx_t *out_fx, int32_t *out_src, unsigned long long *colcnt) {
    int32_t b = -1;
    if (i < len) {
        b = slab_dst[from + i];
        out_dst[to + i] = b;
        out_fx[to + i] = slab_fx[from + i];
        out_src[to + i] = g;
    }
    const unsigned peers = __match_any_sync(kFullMask, b);  // every lane of the warp calls it
    if (b >= 0 && (int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(colcnt + b, (unsigned long long)__popc(peers));
}

__global__ void k_agg_pack(int32_t ng, const int64_t *gloff, const int64_t *g_out_off, const int32_t *slab_dst,
                           const fx_t *slab_fx, int32_t *out_dst, fx_t *out_fx, int32_t *out_src,
                           unsigned long long *colcnt, int64_t *longrows, unsigned long long *nlong) {
    constexpr int kTeams = 32 / kPackTeam;
    const int lane = threadIdx.x & 31, r = lane % kPackTeam;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t g0 = gw * kTeams; g0 < ng; g0 += nw * kTeams) {  // warp-uniform
        const int64_t g = g0 + lane / kPackTeam;
        int64_t len = 0, from = 0, to = 0;
        if (g < ng) {
            to = g_out_off[g];
            len = g_out_off[g + 1] - to;
            from = gloff[g];
        }
        if (len > kPackLong) {  // listed as chunks of kPackChunk entries
            const int64_t nc = (len + kPackChunk - 1) / kPackChunk;
            if (r == 0) {
                const unsigned long long k0 = atomicAdd(nlong, (unsigned long long)nc);
                for (int64_t c = 0; c < nc; c++) longrows[k0 + c] = ((int64_t)g << 32) | c;
            }
            len = 0;
        }
        int64_t mx = len;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(kFullMask, mx, o));
        for (int64_t i0 = 0; i0 < mx; i0 += kPackTeam)
            pack_link(i0 + r, len, from, to, (int32_t)g, slab_dst, slab_fx, out_dst, out_fx, out_src, colcnt);
    }
}

// The listed chunks of long rows (row << 32 | chunk), a block each.
__global__ void k_agg_pack_long(const int64_t *gloff, const int64_t *g_out_off, const int32_t *slab_dst,
                                const fx_t *slab_fx, int32_t *out_dst, fx_t *out_fx, int32_t *out_src,
                                unsigned long long *colcnt, const int64_t *longrows, const unsigned long long *nlong) {
    const int64_t nl = (int64_t)*nlong;
    for (int64_t k = blockIdx.x; k < nl; k += gridDim.x) {
        const int32_t g = (int32_t)(longrows[k] >> 32);
        const int64_t c0 = (longrows[k] & 0xffffffffll) * kPackChunk;
        const int64_t row = g_out_off[g + 1] - g_out_off[g];
        const int64_t to = g_out_off[g] + c0, len = min((int64_t)kPackChunk, row - c0), from = gloff[g] + c0;
        for (int64_t i0 = 0; i0 < len; i0 += blockDim.x)  // uniform over the block
            pack_link(i0 + threadIdx.x, len, from, to, g, slab_dst, slab_fx, out_dst, out_fx, out_src, colcnt);
    }
}

// In-links: every link g->b of the group CSR appended to column b, as one
// 16-byte (row, flow) record in a staging array: one scattered store per
// link instead of two partial-sector ones (k_agg_split then writes the CSC
// arrays in order).
__global__ void k_agg_transpose(int64_t m, const int32_t *out_src, const int32_t *out_dst, const fx_t *out_fx,
                                const int64_t *g_in_off, unsigned long long *colfill, longlong2 *staged) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t e0 = gw * 32; e0 < m; e0 += nw * 32) {  // warp-uniform
        const int64_t e = e0 + lane;
        const int32_t b = e < m ? __ldcs(out_dst + e) : -1;
        const unsigned peers = __match_any_sync(kFullMask, b);
        const int leader = __ffs(peers) - 1;
        unsigned long long base = 0;
        if (b >= 0 && lane == leader) base = atomicAdd(colfill + b, (unsigned long long)__popc(peers));
        base = __shfl_sync(kFullMask, base, leader);
        if (b >= 0) {
            const int64_t q = g_in_off[b] + (int64_t)base + __popc(peers & ((1u << lane) - 1u));
            staged[q] = make_longlong2((long long)__ldcs(out_src + e), (long long)__ldcs(out_fx + e));
        }
    }
}

__global__ void k_agg_split(int64_t m, const longlong2 *staged, int32_t *in_src, fx_t *in_fx) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < m; q += (int64_t)gridDim.x * blockDim.x) {
        const longlong2 r = __ldcs(staged + q);
        in_src[q] = (int32_t)r.x;
        in_fx[q] = (fx_t)r.y;
    }
}

// The block bin's and the split pipeline's dynamic shared memory, set once per device.
static void configure_agg_kernels() {
    static std::mutex mu;
    static std::vector<bool> done;
    int dev = 0;
    RMX_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    if ((int)done.size() <= dev) done.resize(dev + 1, false);
    if (done[dev]) return;
    const int smem = (int)(kAggCap * (sizeof(fx_t) + sizeof(int32_t)));
    RMX_CUDA(cudaFuncSetAttribute(k_agg_block, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    RMX_CUDA(cudaFuncSetAttribute(k_hg_reduce, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kHgSmem));
    done[dev] = true;
}

int64_t aggregate_links(int32_t n, const int64_t *off, const int32_t *dst, const fx_t *fx, const int32_t *src,
                        const int32_t *group, int32_t ng, int64_t *g_out_off, int32_t *g_out_dst, fx_t *g_out_fx,
                        int32_t *g_out_src, int64_t *g_in_off, int32_t *g_in_src, fx_t *g_in_fx, fx_t *rowsum,
                        Arena &gtab_arena, fx_t *&gtab, int64_t &gtab_cap, Arena &ar, cudaStream_t s,
                        const SweepWork *W) {
    configure_agg_kernels();
    int64_t E = 0;
    RMX_CUDA(cudaMemcpyAsync(&E, off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RMX_CUDA(cudaStreamSynchronize(s));
    if (rowsum) RMX_CUDA(cudaMemsetAsync(rowsum, 0, sizeof(fx_t) * std::max(ng, 1), s));
    if (ng <= 0) return 0;
    size_t mk = ar.mark();
    int64_t *gloff = ar.alloc<int64_t>(ng + 1);
    unsigned long long *gcross = ar.alloc<unsigned long long>(ng + 1);
    // tot: [0] small [1] large [2] links out [3] max links [4] mid [5] huge groups, [6..8] their links,
    // chunks and partitions [10] long rows [12..14] split pipeline: chunks, partitions, over capacity
    int64_t *tot = ar.alloc<int64_t>(16);
    RMX_CUDA(cudaMemsetAsync(gloff, 0, sizeof(int64_t) * (ng + 1), s));
    RMX_CUDA(cudaMemsetAsync(gcross, 0, sizeof(unsigned long long) * (ng + 1), s));
    RMX_CUDA(cudaMemsetAsync(tot, 0, sizeof(int64_t) * 16, s));
    k_agg_count<<<blocks_for(n, 256, num_sms() * 32), 256, 0, s>>>(n, off, group,
                                                                    reinterpret_cast<unsigned long long *>(gloff));
    RMX_LAUNCHED();
    scan_exclusive(gloff, gloff, ng + 1, nullptr, ar, s);
    // the gathered ranges; each group's distinct destinations are written back to the start of its range
    int32_t *slab_dst = ar.alloc<int32_t>(std::max<int64_t>(E, 1));
    fx_t *slab_fx = ar.alloc<fx_t>(std::max<int64_t>(E, 1));
    if (E > 0) {
        k_agg_gather<<<blocks_for((E + 31) / 32 * 32, 256, num_sms() * 16), 256, 0, s>>>(E, src, dst, fx, group, gloff,
                                                                                        gcross, slab_dst, slab_fx);
        RMX_LAUNCHED();
    }
    uint8_t *fsmall = ar.alloc<uint8_t>(ng), *fmid = ar.alloc<uint8_t>(ng), *flarge = ar.alloc<uint8_t>(ng),
            *fhuge = ar.alloc<uint8_t>(ng);
    const int64_t part_links = eval_tuning().hub_part;
    k_agg_bins<<<blocks_for(ng, 256, num_sms() * 32), 256, 0, s>>>(
        ng, gcross, part_links, fsmall, fmid, flarge, fhuge, reinterpret_cast<unsigned long long *>(tot + 3),
        reinterpret_cast<unsigned long long *>(tot + 6));
    RMX_LAUNCHED();
    int32_t *lsmall = ar.alloc<int32_t>(ng), *lmid = ar.alloc<int32_t>(ng), *llarge = ar.alloc<int32_t>(ng),
            *lhuge = ar.alloc<int32_t>(ng);
    compact_flags(fsmall, ng, lsmall, tot + 0, ar, s);
    compact_flags(fmid, ng, lmid, tot + 4, ar, s);
    compact_flags(flarge, ng, llarge, tot + 1, ar, s);
    compact_flags(fhuge, ng, lhuge, tot + 5, ar, s);
    int64_t *rowlen = g_out_off;  // row lengths, scanned in place into offsets below
    RMX_CUDA(cudaMemsetAsync(rowlen, 0, sizeof(int64_t) * (ng + 1), s));
    // a group of L links needs a table of next_pow2(2L) slots; beyond shared memory, a global slice per block
    int64_t th[6];  // max links outside the split pipeline; huge groups, their links, chunks, partitions
    RMX_CUDA(cudaMemcpyAsync(th, tot + 3, sizeof th, cudaMemcpyDeviceToHost, s));
    RMX_CUDA(cudaStreamSynchronize(s));
    const int64_t maxlinks = th[0], n_huge = th[2], huge_links = th[3], huge_chunks = th[4], huge_parts = th[5];
    int64_t need = 64;
    while (need < 2 * std::min<int64_t>(maxlinks, ng)) need <<= 1;
    const int nblk = num_sms() * 2;
    if (need > kAggCap && need > gtab_cap) {
        RMX_CUDA(cudaStreamSynchronize(s));  // no launch still reads the old table
        gtab_arena.destroy();
        gtab = nullptr;
        gtab_cap = 0;
        gtab_arena.init((sizeof(fx_t) + sizeof(int32_t)) * need * nblk + 1024);
        gtab = gtab_arena.alloc<fx_t>(need * nblk);
        gtab_arena.alloc<int32_t>(need * nblk);  // the keys follow the values
        gtab_cap = need;
    }
    AggArgs a;
    a.gloff = gloff;
    a.gcross = gcross;
    a.slab_dst = slab_dst;
    a.slab_fx = slab_fx;
    a.rowlen = rowlen;
    a.rowsum = rowsum;
    a.gvals = gtab;
    a.gkeys = gtab ? reinterpret_cast<int32_t *>(gtab + gtab_cap * nblk) : nullptr;
    a.gcap = gtab_cap;
    a.ngroups = ng;
    // the bins run concurrently: the split pipeline (the longest chain, first),
    // warp and mid bins on three auxiliary streams
    cudaStream_t s_small = s, s_mid = s, s_huge = s;
    if (W) {
        RMX_CUDA(cudaEventRecord(W->fork, s));
        for (int k = 0; k < 3; k++) RMX_CUDA(cudaStreamWaitEvent(W->aux[k], W->fork, 0));
        s_small = W->aux[0];
        s_mid = W->aux[1];
        s_huge = W->aux[2];
    }
    if (n_huge > 0) {
        HugeArgs h;
        h.gloff = gloff;
        h.gcross = gcross;
        h.hlist = lhuge;
        h.nh = tot + 5;
        h.coff = ar.alloc<int64_t>(n_huge + 1);
        h.poff = ar.alloc<int64_t>(n_huge + 1);
        h.cgrp = ar.alloc<int32_t>(huge_chunks);
        h.pgrp = ar.alloc<int32_t>(huge_parts);
        h.pcnt = ar.alloc<unsigned long long>(huge_parts);
        h.pstart = ar.alloc<int64_t>(huge_parts + 1);
        h.bkey = ar.alloc<int32_t>(huge_links);
        h.bfx = ar.alloc<fx_t>(huge_links);
        h.tot = tot + 12;
        h.max_chunks = huge_chunks;
        h.max_parts = huge_parts;
        h.max_links = huge_links;
        h.part_links = part_links;
        h.slab_dst = slab_dst;
        h.slab_fx = slab_fx;
        h.rowlen = rowlen;
        h.rowsum = rowsum;
        const cudaStream_t hs = s_huge;
        k_hg_plan<<<1, 1024, 0, hs>>>(h);
        RMX_LAUNCHED();
        const unsigned G = num_sms() * 8;
        k_hg_links<false><<<G, kHgT, 0, hs>>>(h);
        RMX_LAUNCHED();
        k_hg_offsets<<<1, 1024, 0, hs>>>(h);
        RMX_LAUNCHED();
        k_hg_links<true><<<G, kHgT, 0, hs>>>(h);
        RMX_LAUNCHED();
        k_hg_reduce<<<num_sms() * 2, kHgT, kHgSmem, hs>>>(h);
        RMX_LAUNCHED();
    }
    a.list = lsmall;
    a.count = tot + 0;
    k_agg_warp<<<num_sms() * 8, kAggWarps * 32, 0, s_small>>>(a);
    RMX_LAUNCHED();
    a.list = lmid;
    a.count = tot + 4;
    k_agg_mid<<<num_sms() * 8, kAggMidT, 0, s_mid>>>(a);
    RMX_LAUNCHED();
    a.list = llarge;
    a.count = tot + 1;
    k_agg_block<<<nblk, kAggT, kAggCap * (sizeof(fx_t) + sizeof(int32_t)), s>>>(a);
    RMX_LAUNCHED();
    if (W)
        for (int k = 0; k < 3; k++) {
            RMX_CUDA(cudaEventRecord(W->join[k], W->aux[k]));
            RMX_CUDA(cudaStreamWaitEvent(s, W->join[k], 0));
        }
    scan_exclusive(rowlen, g_out_off, ng + 1, tot + 2, ar, s);
    int64_t m = 0, over = 0;
    RMX_CUDA(cudaMemcpyAsync(&m, tot + 2, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    if (n_huge > 0) RMX_CUDA(cudaMemcpyAsync(&over, tot + 14, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RMX_CUDA(cudaMemsetAsync(g_in_off, 0, sizeof(int64_t) * (ng + 1), s));
    RMX_CUDA(cudaStreamSynchronize(s));
    if (over)  // the sizes come from the same counts the plan sums, so this does not happen
        throw std::runtime_error("aggregate_links: split pipeline over its capacity");
    if (m > 0) {
        // chunks of long rows: fewer than ng + m / kPackChunk + 1
        int64_t *longrows = ar.alloc<int64_t>(ng + m / kPackChunk + 1);
        unsigned long long *nlong = reinterpret_cast<unsigned long long *>(tot + 10);
        k_agg_pack<<<blocks_for((int64_t)ng * kPackTeam, 256, num_sms() * 16), 256, 0, s>>>(
            ng, gloff, g_out_off, slab_dst, slab_fx, g_out_dst, g_out_fx, g_out_src,
            reinterpret_cast<unsigned long long *>(g_in_off), longrows, nlong);
        RMX_LAUNCHED();
        k_agg_pack_long<<<num_sms() * 8, 256, 0, s>>>(gloff, g_out_off, slab_dst, slab_fx, g_out_dst, g_out_fx,
                                                     g_out_src, reinterpret_cast<unsigned long long *>(g_in_off),
                                                     longrows, nlong);
        RMX_LAUNCHED();
    }
    scan_exclusive(g_in_off, g_in_off, ng + 1, nullptr, ar, s);
    RMX_CUDA(cudaMemsetAsync(gcross, 0, sizeof(unsigned long long) * (ng + 1), s));  // the column fill counters
    if (m > 0) {
        const unsigned Gm = blocks_for((m + 31) / 32 * 32, 256, num_sms() * 16);
        longlong2 *staged = ar.alloc<longlong2>(m);
        k_agg_transpose<<<Gm, 256, 0, s>>>(m, g_out_src, g_out_dst, g_out_fx, g_in_off, gcross, staged);
        RMX_LAUNCHED();
        k_agg_split<<<blocks_for(m, 256, num_sms() * 16), 256, 0, s>>>(m, staged, g_in_src, g_in_fx);
        RMX_LAUNCHED();
    }
    RMX_CUDA(cudaStreamSynchronize(s));
    ar.release(mk);
    return m;
}

}  // namespace rmx
