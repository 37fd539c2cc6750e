// Fixed device scratch for ddfmm_eval_device_noalloc (include/ddfmm.h).
//
// The low-frequency V-list pass writes one (2P)^3 FFT spectrum per
// low-frequency box and reads them back in the same eval; normally the
// session holds that scratch.  This file holds a process-wide alternative: a
// statically sized device array, present on every GPU that loads the library
// until the process exits.  Host code cannot use the array's name as a device
// address, so the first use on each device resolves it with
// cudaGetSymbolAddress while that device is current, and later calls reuse the
// cached address.
#include <cuda_runtime.h>

#include <mutex>
#include <stdexcept>
#include <string>

#include "kernels.cuh"

namespace ddfmm {

constexpr size_t NOALLOC_SCRATCH_BYTES = 16u << 20;  // 16 MiB

static __device__ __align__(256) double2 g_vlist_scratch[NOALLOC_SCRATCH_BYTES / sizeof(double2)];

namespace {
std::mutex g_mu;
constexpr int kMaxDevices = 64;
void* g_addr[kMaxDevices] = {};
}  // namespace

// Device address and capacity (in double2) of the scratch on the current device.
double2* noalloc_scratch(size_t* capacity) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) throw std::runtime_error("CUDA error: device ordinal beyond the scratch table");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_vlist_scratch);
        if (e != cudaSuccess)
            throw std::runtime_error(std::string("CUDA error: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_addr[dev] = p;
    }
    *capacity = NOALLOC_SCRATCH_BYTES / sizeof(double2);
    return static_cast<double2*>(g_addr[dev]);
}

}  // namespace ddfmm
