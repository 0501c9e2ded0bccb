// Device-wide primitives: exclusive scan, stable compaction, stable LSD radix
// sort and stable bucket partition. All are deterministic (results do not
// depend on scheduling) and run on the caller's stream with scratch from an
// Arena (no allocation inside).
#pragma once
#include "rmx_common.cuh"

namespace rmx {

// Bump allocator over one device allocation. mark()/release() give scoped
// scratch; alloc() throws CudaError(cudaErrorMemoryAllocation) when full.
// The block is a cudaMalloc allocation that destroy() keeps in a process-wide
// cache (up to a quarter of the device's memory) instead of freeing: the next
// arena that fits (at most twice its size) takes it, so closing a graph handle
// and opening another of similar size costs no cudaMalloc / cudaFree pair.
// release_device_cache() frees the cached blocks.
struct Arena {
    char *base = nullptr;
    size_t cap = 0, top = 0, peak = 0;
    size_t block = 0;  // size of the underlying allocation (>= cap)
    int dev = -1;      // device of the allocation
    void init(size_t bytes);
    void destroy();
    void *alloc_bytes(size_t bytes);
    template <typename T>
    T *alloc(size_t n) {
        return static_cast<T *>(alloc_bytes(n * sizeof(T)));
    }
    size_t mark() const { return top; }
    void release(size_t m) { top = m; }
};

// cudaFree every cached arena block (all devices). Arenas in use are untouched.
void release_device_cache();

// out[i] = sum_{j<i} in[i] for i < n; if total != nullptr, *total (device) =
// sum of all n. in and out may alias.
void scan_exclusive(const int64_t *in, int64_t *out, int64_t n, int64_t *total, Arena &ar, cudaStream_t s);
void scan_exclusive(const uint32_t *in, uint32_t *out, int64_t n, uint32_t *total, Arena &ar, cudaStream_t s);

// Indices i (ascending) with flags[i] != 0 written to out; *count (device).
void compact_flags(const uint8_t *flags, int64_t n, int32_t *out, int64_t *count, Arena &ar, cudaStream_t s);
// The same over the first *n_dev flags (device, at most n_max): grids are
// sized for n_max, so the launches do not depend on the count (the form a
// captured graph replays with changing sizes).
void compact_flags_dev(const uint8_t *flags, const int64_t *n_dev, int64_t n_max, int32_t *out, int64_t *count,
                       Arena &ar, cudaStream_t s);

// Stable sort of (key, value) pairs by key bits [0, key_bits). Sorted data ends
// in keys/vals (the alt buffers are scratch of the same size).
void radix_sort_pairs(uint64_t *keys, uint32_t *vals, uint64_t *keys_alt, uint32_t *vals_alt, int64_t n,
                      int key_bits, Arena &ar, cudaStream_t s);

// Stable partition of items by a small bucket id (< nb <= 256): vals_out holds
// the values grouped by bucket, input order kept within a bucket; bucket_off
// (device, nb+1 entries) receives the bucket boundaries.
void bucket_partition(const uint16_t *bucket, const int32_t *vals_in, int32_t *vals_out, int64_t n, int nb,
                      int64_t *bucket_off, Arena &ar, cudaStream_t s);
// The same for the first *n_dev items (device, at most n_max), grids sized for n_max.
void bucket_partition_dev(const uint16_t *bucket, const int32_t *vals_in, int32_t *vals_out, const int64_t *n_dev,
                          int64_t n_max, int nb, int64_t *bucket_off, Arena &ar, cudaStream_t s);

}  // namespace rmx
