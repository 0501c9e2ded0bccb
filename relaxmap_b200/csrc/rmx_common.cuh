// Shared device definitions for the B200 map-equation engine.
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>

#include <cstdio>
#include <stdexcept>
#include <string>

namespace rmx {

// Teleportation as fixed in the reference (Module.h:114-116).
constexpr double kAlpha = 0.15;
constexpr double kBeta = 1.0 - 0.15;

// Fixed-point representation of flows and module statistics. Every module
// statistic is an exact integer sum of per-node / per-link fixed-point values,
// so incremental updates from any number of concurrent atomic adds are exact,
// associative and deterministic: the running statistics always equal the
// from-scratch sums bit for bit. 2^-62 ~ 2.2e-19 absolute resolution; all
// quantities lie in [0, 1] (range +-2).
typedef long long fx_t;
constexpr double kFxScale = 4611686018427387904.0;  // 2^62
constexpr double kFxInv = 1.0 / 4611686018427387904.0;
// Accumulators of code-length terms (|sum| up to ~log N nats): 2^-58.
constexpr double kFxLScale = 288230376151711744.0;  // 2^58
constexpr double kFxLInv = 1.0 / 288230376151711744.0;

__host__ __device__ __forceinline__ fx_t to_fx(double x) {
#ifdef __CUDA_ARCH__
    return __double2ll_rn(x * kFxScale);
#else
    return (fx_t)llrint(x * kFxScale);
#endif
}
__host__ __device__ __forceinline__ double from_fx(fx_t v) { return (double)v * kFxInv; }
__device__ __forceinline__ fx_t to_fxl(double x) { return __double2ll_rn(x * kFxLScale); }
__host__ __device__ __forceinline__ double from_fxl(fx_t v) { return (double)v * kFxLInv; }

// p log p with 0 log 0 = 0 (Module.h:23-25).
__device__ __forceinline__ double plogp(double x) { return x > 0.0 ? x * log(x) : 0.0; }

// Statistics of a module or of a moving unit: flow P, teleport weight TW,
// dangling flow D and out-flow to other modules OUT. 32 bytes: one sector.
struct __align__(32) Stat4 {
    fx_t P, TW, D, OUT;
};

// Exit flow q = tau (1 - TW) P + (1 - tau) (OUT + (1 - TW) D)
// (calculateCodeLength, Module.cpp:2978-2991; singleton form Module.cpp:86-95).
__device__ __forceinline__ double exit_flow(double P, double TW, double D, double OUT) {
    double e = kAlpha * (1.0 - TW) * P;
    return e + kBeta * (OUT + (1.0 - TW) * D);
}

__device__ __forceinline__ void atomic_add_fx(fx_t *a, fx_t v) {
    atomicAdd(reinterpret_cast<unsigned long long *>(a), static_cast<unsigned long long>(v));
}

// Grid sizing: a multiple of the SM count (148 on B200).
int num_sms();

// An NVTX range over the object's lifetime: host-side phase markers (graph
// build, flow, sweeps, coarsening, coarse-tune, adjoint, batch waves) for a
// profiler's timeline; without a profiler attached the calls return at once.
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

struct CudaError : std::runtime_error {
    cudaError_t code;
    CudaError(cudaError_t c, const std::string &m) : std::runtime_error(m), code(c) {}
};

// An iteration that must converge stopped on its cap (RMX_ERR_NO_CONVERGENCE).
struct NoConvergence : std::runtime_error {
    using std::runtime_error::runtime_error;
};

inline void check(cudaError_t e, const char *what, const char *file, int line) {
    if (e != cudaSuccess) {
        char buf[512];
        snprintf(buf, sizeof buf, "%s failed at %s:%d: %s", what, file, line, cudaGetErrorString(e));
        throw CudaError(e, buf);
    }
}
// Kernels launched by this library since load (every launch site goes through
// RMX_LAUNCHED).
extern unsigned long long g_kernel_launches;
inline void launched(const char *file, int line) {
    __atomic_fetch_add(&g_kernel_launches, 1ull, __ATOMIC_RELAXED);
    check(cudaGetLastError(), "kernel launch", file, line);
}
#define RMX_CUDA(x) ::rmx::check((x), #x, __FILE__, __LINE__)
#define RMX_LAUNCHED() ::rmx::launched(__FILE__, __LINE__)

inline unsigned blocks_for(int64_t n, int threads, int64_t cap = 1 << 20) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (unsigned)b;
}

}  // namespace rmx
