// Stationary flow for callers that cannot allocate device memory.
//
// Some callers own every byte of device memory themselves or must not allocate
// while they run: a framework that hands out memory only from its own pool
// under a fixed budget, or a latency-bound service that cannot afford the
// device-wide synchronisation an allocation implies. rmx_steady_state_noalloc
// runs rmx_initiate's power iteration on arrays such a caller already holds on
// the device, with its temporary storage in one fixed array compiled into this
// library.
#include <mutex>

#include "../../include/relaxmap_b200.h"
#include "rmx_engine.cuh"

namespace {

// Working storage of the solve: y[RMX_NOALLOC_MAX_NODES] (unnormalised next
// flow) and 3 x kMaxBlocks per-block partial sums. About 8.1 MB, held on every
// device that loads the library until the process exits.
constexpr int kMaxBlocks = 4096;
constexpr size_t kScratchBytes = sizeof(double) * ((size_t)RMX_NOALLOC_MAX_NODES + 3 * kMaxBlocks) + 256;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of g_noalloc_scratch per device, found once per device with
// that device current (host code cannot take the address of a __device__
// array directly: the name is only a host-side stand-in). Kept for the life of
// the process, so a cudaDeviceReset after the first call leaves it stale (the
// header says not to call again after one).
constexpr int kMaxDevices = 64;
void *g_addr[kMaxDevices] = {};
std::mutex g_mu;

void *scratch_address(int dev) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void *ptr = nullptr;
        rmx::check(cudaGetSymbolAddress(&ptr, g_noalloc_scratch), "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__,
                   __LINE__);
        g_addr[dev] = ptr;
    }
    return g_addr[dev];
}

thread_local std::string g_err;

}  // namespace

extern "C" const char *rmx_noalloc_last_error(void) { return g_err.c_str(); }

extern "C" rmx_status rmx_steady_state_noalloc(int32_t n_nodes, int64_t n_links, const int64_t *in_off,
                                               const int32_t *in_src, const double *in_w, const double *teleport,
                                               const uint8_t *dangling, double *p_out, int32_t *iters_out,
                                               void *stream) {
    if (n_nodes <= 0 || n_nodes > RMX_NOALLOC_MAX_NODES) {
        g_err = "rmx_steady_state_noalloc: n_nodes must be in 1.." + std::to_string(RMX_NOALLOC_MAX_NODES);
        return RMX_ERR_INVALID;
    }
    if (n_links < 0 || !in_off || (n_links > 0 && (!in_src || !in_w)) || !teleport || !dangling || !p_out) {
        g_err = "rmx_steady_state_noalloc: a required device pointer is NULL";
        return RMX_ERR_INVALID;
    }
    try {
        int dev = 0;
        rmx::check(cudaGetDevice(&dev), "cudaGetDevice", __FILE__, __LINE__);
        if (dev < 0 || dev >= kMaxDevices) {
            g_err = "rmx_steady_state_noalloc: device ordinal beyond the supported range";
            return RMX_ERR_INVALID;
        }
        unsigned char *base = static_cast<unsigned char *>(scratch_address(dev));
        double *y = reinterpret_cast<double *>(base);
        double *parts = y + RMX_NOALLOC_MAX_NODES;
        // The iteration count goes to the caller's int (device memory) or,
        // without one, to the last word of the scratch. Every scratch word is
        // written by the solve before it is read, so nothing is cleared.
        int *iters = iters_out ? reinterpret_cast<int *>(iters_out) : reinterpret_cast<int *>(parts + 3 * kMaxBlocks);
        rmx::power_iteration_into(n_nodes, in_off, in_src, in_w, teleport, dangling, p_out, y, parts, kMaxBlocks,
                                  iters, static_cast<cudaStream_t>(stream),
                                  rmx::spmv_width((double)n_links / n_nodes));
    } catch (const std::exception &e) {
        g_err = e.what();
        return RMX_ERR_CUDA;
    }
    return RMX_OK;
}
