// launch_util.h -- host helpers shared by the engine and the no-allocation
// entry point.
#pragma once
#include <cuda_runtime.h>

#include <mutex>

namespace pscfg {

// Raise a kernel's dynamic shared-memory limit to the device's opt-in
// maximum (minus its static shared memory), once per (kernel, device).
// Engines on different host threads launch the same kernels with different
// sizes, so the limit is never lowered to one caller's size.  Uses a fixed
// table (no heap allocation).
inline cudaError_t allow_dyn_smem(const void *func)
{
    static std::mutex mu;
    static const void *fn[512];
    static int dv[512];
    static int n = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    for (int i = 0; i < n; i++)
        if (fn[i] == func && dv[i] == dev) return cudaSuccess;
    cudaFuncAttributes a;
    if ((e = cudaFuncGetAttributes(&a, func)) != cudaSuccess) return e;
    int mx = 0;
    if ((e = cudaDeviceGetAttribute(&mx, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, mx - (int)a.sharedSizeBytes)) !=
        cudaSuccess)
        return e;
    if (n < 512) {
        fn[n] = func;
        dv[n] = dev;
        n++;
    }
    return cudaSuccess;
}

}  // namespace pscfg
