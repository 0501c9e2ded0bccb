// Device-wide primitives (see rmx_prims.cuh).
#include <algorithm>
#include <cstddef>
#include <mutex>
#include <vector>

#include "rmx_prims.cuh"

namespace rmx {

unsigned long long g_kernel_launches = 0;

int num_sms() {
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
            n = 148;
    }
    return n;
}

namespace {

// Blocks of destroyed arenas, oldest first, kept for the next arena that fits.
struct CachedBlock {
    char *ptr;
    size_t bytes;
    int dev;
};

std::mutex g_cache_mu;
std::vector<CachedBlock> g_cache;

// Bytes of cached blocks the current device may keep: a quarter of its memory.
size_t cache_budget() {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        (void)cudaGetLastError();
        return 0;
    }
    return total_b / 2;
}

// cudaFree the cached blocks of device dev (current), oldest first, until at
// most keep bytes of them remain. The caller holds g_cache_mu.
void trim_locked(int dev, size_t keep) {
    size_t held = 0;
    for (const CachedBlock &b : g_cache)
        if (b.dev == dev) held += b.bytes;
    for (size_t i = 0; i < g_cache.size() && held > keep;) {
        if (g_cache[i].dev != dev) {
            i++;
            continue;
        }
        cudaFree(g_cache[i].ptr);
        held -= g_cache[i].bytes;
        g_cache.erase(g_cache.begin() + (std::ptrdiff_t)i);
    }
}

// The smallest cached block of device dev that holds `bytes` and is at most
// twice that size, taken out of the cache; null if there is none.
char *take_cached(int dev, size_t bytes, size_t *block_bytes) {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    size_t best = g_cache.size();
    for (size_t i = 0; i < g_cache.size(); i++) {
        const CachedBlock &b = g_cache[i];
        if (b.dev != dev || b.bytes < bytes || b.bytes / 2 > bytes) continue;
        if (best == g_cache.size() || b.bytes < g_cache[best].bytes) best = i;
    }
    if (best == g_cache.size()) return nullptr;
    char *p = g_cache[best].ptr;
    *block_bytes = g_cache[best].bytes;
    g_cache.erase(g_cache.begin() + (std::ptrdiff_t)best);
    return p;
}

}  // namespace

void Arena::init(size_t bytes) {
    RMX_CUDA(cudaGetDevice(&dev));
    base = take_cached(dev, bytes, &block);
    if (!base) {
        cudaError_t e = cudaMalloc(&base, bytes);
        if (e == cudaErrorMemoryAllocation) {  // the cache may hold what is missing
            (void)cudaGetLastError();
            {
                std::lock_guard<std::mutex> lk(g_cache_mu);
                trim_locked(dev, 0);
            }
            e = cudaMalloc(&base, bytes);
        }
        if (e != cudaSuccess) {
            base = nullptr;
            check(e, "cudaMalloc (device arena)", __FILE__, __LINE__);
        }
        block = bytes;
    }
    cap = bytes;
    top = peak = 0;
}

void Arena::destroy() {
    if (base) {
        int cur = -1;
        cudaGetDevice(&cur);
        if (cur != dev) cudaSetDevice(dev);
        // wait for the device first, as cudaFree would: no queued work still
        // uses the block when another arena takes it
        if (cudaDeviceSynchronize() == cudaSuccess) {
            std::lock_guard<std::mutex> lk(g_cache_mu);
            const size_t budget = cache_budget();
            if (block <= budget) {
                g_cache.push_back({base, block, dev});
                trim_locked(dev, budget);
            } else {
                cudaFree(base);
            }
        } else {
            cudaFree(base);
        }
        if (cur >= 0 && cur != dev) cudaSetDevice(cur);
    }
    base = nullptr;
    cap = top = peak = block = 0;
}

void release_device_cache() {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    if (g_cache.empty()) return;  // nothing held: no device call
    int cur = -1;
    RMX_CUDA(cudaGetDevice(&cur));
    cudaError_t first = cudaSuccess;
    while (!g_cache.empty()) {
        const CachedBlock b = g_cache.back();
        g_cache.pop_back();
        cudaError_t e = cudaSetDevice(b.dev);
        if (e == cudaSuccess) e = cudaFree(b.ptr);
        if (first == cudaSuccess) first = e;
    }
    cudaError_t e = cudaSetDevice(cur);
    if (first == cudaSuccess) first = e;
    check(first, "release_device_cache", __FILE__, __LINE__);
}

void *Arena::alloc_bytes(size_t bytes) {
    size_t a = (top + 255) & ~size_t(255);
    if (a + bytes > cap) throw CudaError(cudaErrorMemoryAllocation, "device scratch arena exhausted");
    top = a + bytes;
    peak = std::max(peak, top);
    return base + a;
}

// ------------------------------------------------------------------- scan

constexpr unsigned kFull = 0xffffffffu;
constexpr int kScanT = 512, kScanI = 8, kScanTile = kScanT * kScanI;

// Exclusive scan of one value per thread across the block; *total = block sum.
template <typename T>
__device__ __forceinline__ T block_exclusive(T v, T *warp_sums, T *total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[w] = x;
    __syncthreads();
    if (w == 0) {
        T s = lane < nw ? warp_sums[lane] : T(0);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T y = __shfl_up_sync(kFull, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) warp_sums[lane] = s;
    }
    __syncthreads();
    T pre = (w > 0 ? warp_sums[w - 1] : T(0)) + x - v;
    *total = warp_sums[nw - 1];
    __syncthreads();
    return pre;
}

template <typename T>
__global__ void k_scan_block_sums(const T *in, int64_t n, T *bsum) {
    __shared__ T ws[32];
    int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanI;
    T s = 0;
#pragma unroll
    for (int i = 0; i < kScanI; i++)
        if (base + i < n) s += in[base + i];
    T tot;
    block_exclusive(s, ws, &tot);
    if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

template <typename T>
__global__ void k_scan_apply(const T *in, T *out, int64_t n, const T *boff, T *total) {
    __shared__ T ws[32];
    int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanI;
    T v[kScanI];
    T s = 0;
#pragma unroll
    for (int i = 0; i < kScanI; i++) {
        v[i] = base + i < n ? in[base + i] : T(0);
        s += v[i];
    }
    T tot;
    T pre = block_exclusive(s, ws, &tot) + (boff ? boff[blockIdx.x] : T(0));
#pragma unroll
    for (int i = 0; i < kScanI; i++) {
        if (base + i < n) out[base + i] = pre;
        pre += v[i];
    }
    if (total && !boff && threadIdx.x == 0) *total = tot;
}

template <typename T>
static void scan_impl(const T *in, T *out, int64_t n, T *total, Arena &ar, cudaStream_t s) {
    if (n <= 0) {
        if (total) RMX_CUDA(cudaMemsetAsync(total, 0, sizeof(T), s));
        return;
    }
    int64_t nb = (n + kScanTile - 1) / kScanTile;
    if (nb == 1) {
        k_scan_apply<T><<<1, kScanT, 0, s>>>(in, out, n, nullptr, total);
        RMX_LAUNCHED();
        return;
    }
    size_t m = ar.mark();
    T *bsum = ar.alloc<T>(nb);
    k_scan_block_sums<T><<<(unsigned)nb, kScanT, 0, s>>>(in, n, bsum);
    RMX_LAUNCHED();
    scan_impl<T>(bsum, bsum, nb, total, ar, s);
    k_scan_apply<T><<<(unsigned)nb, kScanT, 0, s>>>(in, out, n, bsum, nullptr);
    RMX_LAUNCHED();
    ar.release(m);
}

void scan_exclusive(const int64_t *in, int64_t *out, int64_t n, int64_t *total, Arena &ar, cudaStream_t s) {
    scan_impl<long long>(reinterpret_cast<const long long *>(in), reinterpret_cast<long long *>(out), n,
                         reinterpret_cast<long long *>(total), ar, s);
}
void scan_exclusive(const uint32_t *in, uint32_t *out, int64_t n, uint32_t *total, Arena &ar, cudaStream_t s) {
    scan_impl<unsigned>(in, out, n, total, ar, s);
}

// ------------------------------------------------------------- compaction

__global__ void k_flag_count(const uint8_t *flags, int64_t n, const int64_t *n_dev, long long *bsum) {
    __shared__ long long ws[32];
    if (n_dev) n = *n_dev;
    int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanI;
    long long c = 0;
#pragma unroll
    for (int i = 0; i < kScanI; i++)
        if (base + i < n && flags[base + i]) c++;
    long long tot;
    block_exclusive(c, ws, &tot);
    if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

__global__ void k_flag_scatter(const uint8_t *flags, int64_t n, const int64_t *n_dev, const long long *boff,
                               int32_t *out) {
    __shared__ long long ws[32];
    if (n_dev) n = *n_dev;
    int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanI;
    uint8_t f[kScanI];
    long long c = 0;
#pragma unroll
    for (int i = 0; i < kScanI; i++) {
        f[i] = (base + i < n) ? flags[base + i] : 0;
        c += f[i] != 0;
    }
    long long tot;
    long long pre = block_exclusive(c, ws, &tot) + boff[blockIdx.x];
#pragma unroll
    for (int i = 0; i < kScanI; i++)
        if (f[i]) out[pre++] = (int32_t)(base + i);
}

static void compact_impl(const uint8_t *flags, int64_t n, const int64_t *n_dev, int32_t *out, int64_t *count,
                         Arena &ar, cudaStream_t s) {
    if (n <= 0) {
        RMX_CUDA(cudaMemsetAsync(count, 0, sizeof(int64_t), s));
        return;
    }
    size_t m = ar.mark();
    int64_t nb = (n + kScanTile - 1) / kScanTile;
    long long *bsum = ar.alloc<long long>(nb);
    k_flag_count<<<(unsigned)nb, kScanT, 0, s>>>(flags, n, n_dev, bsum);
    RMX_LAUNCHED();
    scan_impl<long long>(bsum, bsum, nb, reinterpret_cast<long long *>(count), ar, s);
    k_flag_scatter<<<(unsigned)nb, kScanT, 0, s>>>(flags, n, n_dev, bsum, out);
    RMX_LAUNCHED();
    ar.release(m);
}

void compact_flags(const uint8_t *flags, int64_t n, int32_t *out, int64_t *count, Arena &ar, cudaStream_t s) {
    compact_impl(flags, n, nullptr, out, count, ar, s);
}

void compact_flags_dev(const uint8_t *flags, const int64_t *n_dev, int64_t n_max, int32_t *out, int64_t *count,
                       Arena &ar, cudaStream_t s) {
    compact_impl(flags, n_max, n_dev, out, count, ar, s);
}

// ------------------------------------------------------------- radix sort
// One stable counting pass: per-tile digit histograms laid out digit-major,
// an exclusive scan over them gives each (digit, tile) its output offset, and
// the scatter ranks equal digits within a tile in input order (warp match +
// per-warp counters). Tiles hold kRsT * kRsI elements in round-major order.

constexpr int kRsT = 256, kRsI = 16, kRsTile = kRsT * kRsI, kRsW = kRsT / 32;

struct KeyDigit {
    const uint64_t *k;
    int shift;
    unsigned mask;
    __device__ unsigned operator()(int64_t e) const { return (unsigned)(k[e] >> shift) & mask; }
};
struct ArrDigit {
    const uint16_t *d;
    __device__ unsigned operator()(int64_t e) const { return d[e]; }
};

template <typename Dig>
__global__ void __launch_bounds__(kRsT) k_rs_hist(Dig dig, int64_t n, const int64_t *n_dev, int nb, unsigned *hist,
                                                  int64_t ntiles) {
    __shared__ unsigned cnt[256];
    if (n_dev) n = *n_dev;
    for (int i = threadIdx.x; i < nb; i += kRsT) cnt[i] = 0;
    __syncthreads();
    int64_t base = (int64_t)blockIdx.x * kRsTile;
#pragma unroll 4
    for (int r = 0; r < kRsI; r++) {
        int64_t e = base + (int64_t)r * kRsT + threadIdx.x;
        if (e < n) atomicAdd(&cnt[dig(e)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nb; i += kRsT) hist[(int64_t)i * ntiles + blockIdx.x] = cnt[i];
}

// The scatter stages half a tile (kRsHalf elements) in shared memory in
// output order before writing it, so that each digit's run of the half leaves
// as consecutive stores instead of one scattered store per element. Output
// positions are those of the plain per-element scatter: input order within a
// digit (rows, then warps, then lanes).
constexpr int kRsRows = kRsI / 2, kRsHalf = kRsT * kRsRows;

template <typename Dig, typename K, typename V>
__global__ void __launch_bounds__(kRsT) k_rs_scatter(Dig dig, const K *kin, K *kout, const V *vin, V *vout, int64_t n,
                                                     const int64_t *n_dev, int nb, const unsigned *offs,
                                                     int64_t ntiles) {
    __shared__ unsigned run[256];            // global output position of each digit's next element
    __shared__ unsigned hc[256], hs[256];    // the half's count and start of each digit
    __shared__ unsigned wc[kRsW][256];       // one row's count per warp and digit
    __shared__ K skey[kRsHalf];
    __shared__ V sval[kRsHalf];
    __shared__ uint16_t sdig[kRsHalf];
    if (n_dev) n = *n_dev;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < 256; i += kRsT) {
        run[i] = i < nb ? offs[(int64_t)i * ntiles + blockIdx.x] : 0u;
        hc[i] = 0;
#pragma unroll
        for (int q = 0; q < kRsW; q++) wc[q][i] = 0;
    }
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
    const int64_t base = (int64_t)blockIdx.x * kRsTile;
    for (int half = 0; half < 2; half++) {
        unsigned dg[kRsRows], lr[kRsRows];
        for (int r = 0; r < kRsRows; r++) {
            const int64_t e = base + (int64_t)(half * kRsRows + r) * kRsT + threadIdx.x;
            const bool valid = e < n;
            const unsigned d = valid ? dig(e) : 0x10000u;
            const unsigned peers = __match_any_sync(kFull, d);
            const unsigned rank = __popc(peers & lt);
            if (valid && rank == 0) wc[w][d] = __popc(peers);
            __syncthreads();
            dg[r] = d;
            if (valid) {
                unsigned pos = hc[d] + rank;
                for (int q = 0; q < w; q++) pos += wc[q][d];
                lr[r] = pos;
            }
            __syncthreads();
            for (int i = threadIdx.x; i < nb; i += kRsT) {
                unsigned t = 0;
#pragma unroll
                for (int q = 0; q < kRsW; q++) {
                    t += wc[q][i];
                    wc[q][i] = 0;
                }
                hc[i] += t;
            }
            __syncthreads();
        }
        // digit starts within the half (nb <= 256: one warp scans 8 per lane)
        if (w == 0) {
            unsigned v[8], t = 0;
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int i = lane * 8 + k;
                v[k] = i < nb ? hc[i] : 0u;
                t += v[k];
            }
            unsigned x = t;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned y = __shfl_up_sync(kFull, x, o);
                if (lane >= o) x += y;
            }
            unsigned acc = x - t;
#pragma unroll
            for (int k = 0; k < 8; k++) {
                hs[lane * 8 + k] = acc;
                acc += v[k];
            }
        }
        __syncthreads();
        for (int r = 0; r < kRsRows; r++) {
            const int64_t e = base + (int64_t)(half * kRsRows + r) * kRsT + threadIdx.x;
            if (e < n) {
                const unsigned q = hs[dg[r]] + lr[r];
                if (kout) skey[q] = kin[e];
                sval[q] = vin[e];
                sdig[q] = (uint16_t)dg[r];
            }
        }
        __syncthreads();
        const int64_t rem = n - (base + (int64_t)half * kRsHalf);
        const int cnt = rem <= 0 ? 0 : (rem < kRsHalf ? (int)rem : kRsHalf);
        for (int q = threadIdx.x; q < cnt; q += kRsT) {
            const unsigned d = sdig[q];
            const unsigned g = run[d] + (unsigned)q - hs[d];
            if (kout) kout[g] = skey[q];
            vout[g] = sval[q];
        }
        __syncthreads();
        for (int i = threadIdx.x; i < nb; i += kRsT) {
            run[i] += hc[i];
            hc[i] = 0;
        }
        __syncthreads();
    }
}

void radix_sort_pairs(uint64_t *keys, uint32_t *vals, uint64_t *keys_alt, uint32_t *vals_alt, int64_t n,
                      int key_bits, Arena &ar, cudaStream_t s) {
    if (n <= 1 || key_bits <= 0) return;
    if (n >= (int64_t(1) << 32)) throw std::invalid_argument("radix_sort_pairs: more than 2^32 items");
    int64_t ntiles = (n + kRsTile - 1) / kRsTile;
    size_t m = ar.mark();
    unsigned *hist = ar.alloc<unsigned>(256 * ntiles);
    uint64_t *ks = keys, *kd = keys_alt;
    uint32_t *vs = vals, *vd = vals_alt;
    for (int shift = 0; shift < key_bits; shift += 8) {
        int bits = std::min(8, key_bits - shift);
        int nb = 1 << bits;
        KeyDigit dig{ks, shift, (unsigned)nb - 1u};
        k_rs_hist<<<(unsigned)ntiles, kRsT, 0, s>>>(dig, n, nullptr, nb, hist, ntiles);
        RMX_LAUNCHED();
        scan_impl<unsigned>(hist, hist, (int64_t)nb * ntiles, nullptr, ar, s);
        k_rs_scatter<<<(unsigned)ntiles, kRsT, 0, s>>>(dig, ks, kd, vs, vd, n, nullptr, nb, hist, ntiles);
        RMX_LAUNCHED();
        std::swap(ks, kd);
        std::swap(vs, vd);
    }
    if (ks != keys) {
        RMX_CUDA(cudaMemcpyAsync(keys, ks, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, s));
        RMX_CUDA(cudaMemcpyAsync(vals, vs, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
    }
    ar.release(m);
}

__global__ void k_bucket_bounds(const unsigned *offs, int64_t ntiles, int nb, int64_t n, const int64_t *n_dev,
                                int64_t *bucket_off) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nb) bucket_off[i] = offs[(int64_t)i * ntiles];
    if (i == nb) bucket_off[nb] = n_dev ? *n_dev : n;
}

static void bucket_impl(const uint16_t *bucket, const int32_t *vals_in, int32_t *vals_out, int64_t n,
                        const int64_t *n_dev, int nb, int64_t *bucket_off, Arena &ar, cudaStream_t s) {
    if (nb < 1 || nb > 256) throw std::invalid_argument("bucket_partition: 1..256 buckets");
    if (n <= 0) {
        RMX_CUDA(cudaMemsetAsync(bucket_off, 0, sizeof(int64_t) * (nb + 1), s));
        return;
    }
    int64_t ntiles = (n + kRsTile - 1) / kRsTile;
    size_t m = ar.mark();
    unsigned *hist = ar.alloc<unsigned>((size_t)nb * ntiles);
    ArrDigit dig{bucket};
    k_rs_hist<<<(unsigned)ntiles, kRsT, 0, s>>>(dig, n, n_dev, nb, hist, ntiles);
    RMX_LAUNCHED();
    scan_impl<unsigned>(hist, hist, (int64_t)nb * ntiles, nullptr, ar, s);
    k_rs_scatter<ArrDigit, int32_t, int32_t>
        <<<(unsigned)ntiles, kRsT, 0, s>>>(dig, nullptr, nullptr, vals_in, vals_out, n, n_dev, nb, hist, ntiles);
    RMX_LAUNCHED();
    k_bucket_bounds<<<1, 288, 0, s>>>(hist, ntiles, nb, n, n_dev, bucket_off);
    RMX_LAUNCHED();
    ar.release(m);
}

void bucket_partition(const uint16_t *bucket, const int32_t *vals_in, int32_t *vals_out, int64_t n, int nb,
                      int64_t *bucket_off, Arena &ar, cudaStream_t s) {
    bucket_impl(bucket, vals_in, vals_out, n, nullptr, nb, bucket_off, ar, s);
}

void bucket_partition_dev(const uint16_t *bucket, const int32_t *vals_in, int32_t *vals_out, const int64_t *n_dev,
                          int64_t n_max, int nb, int64_t *bucket_off, Arena &ar, cudaStream_t s) {
    bucket_impl(bucket, vals_in, vals_out, n_max, n_dev, nb, bucket_off, ar, s);
}

}  // namespace rmx
