// Fixed device scratch for ddfmm_eval_device_noalloc (include/ddfmm.h).
//
// The low-frequency V-list pass writes one (2P)^3 FFT spectrum per
// low-frequency box and reads them back in the same eval; normally the
// session holds that scratch.  This file holds a process-wide alternative: a
// statically sized device array, present on every GPU that loads the library
// until the process exits.  Host code cannot use the array's name as a device
// address, so every call resolves it with cudaGetSymbolAddress on the current
// device (no allocation; the first call on a device may load the module).
// Nothing is cached, so the address stays right after a cudaDeviceReset
// gives the device a new primary context.
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "kernels.cuh"

namespace ddfmm {

constexpr size_t NOALLOC_SCRATCH_BYTES = 16u << 20;  // 16 MiB

static __device__ __align__(256) double2 g_vlist_scratch[NOALLOC_SCRATCH_BYTES / sizeof(double2)];

// Device address and capacity (in double2) of the scratch on the current device.
double2* noalloc_scratch(size_t* capacity) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_vlist_scratch);
    if (e != cudaSuccess)
        throw std::runtime_error(std::string("CUDA error: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    *capacity = NOALLOC_SCRATCH_BYTES / sizeof(double2);
    return static_cast<double2*>(p);
}

}  // namespace ddfmm
