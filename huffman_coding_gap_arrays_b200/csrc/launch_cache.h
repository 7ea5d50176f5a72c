// launch_cache.h -- per-device launch facts of one kernel, for the host-side
// launchers: the device's SM count and how many CTAs of the kernel fit on an
// SM at its launch shape.  A kernel that needs more than 48 KiB of dynamic
// shared memory gets cudaFuncAttributeMaxDynamicSharedMemorySize set first;
// that attribute belongs to the device's context, so everything is done once
// PER DEVICE (the device current at the call), under std::call_once, so two
// host threads never see a half-filled entry.
#pragma once

#include <cuda_runtime.h>

#include <mutex>

namespace hgap {

constexpr int kMaxDevices = 64;

struct LaunchFacts {
    int sms = 0;
    int per_sm = 0;
    cudaError_t err = cudaSuccess;
};

class LaunchCache {
public:
    // `func`: the kernel; `threads`, `smem`: its block size and dynamic shared memory.
    LaunchFacts get(const void* func, int threads, size_t smem) {
        LaunchFacts bad;
        int dev = -1;
        const cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) {
            bad.err = e;
            return bad;
        }
        if (dev < 0 || dev >= kMaxDevices) {
            bad.err = cudaErrorInvalidDevice;
            return bad;
        }
        std::call_once(once_[dev], [&] {
            LaunchFacts& f = facts_[dev];
            f.err = cudaDeviceGetAttribute(&f.sms, cudaDevAttrMultiProcessorCount, dev);
            if (f.err == cudaSuccess && smem > 48 * 1024)
                f.err = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (f.err == cudaSuccess)
                f.err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&f.per_sm, func, threads, smem);
            if (f.per_sm < 1) f.per_sm = 1;
        });
        return facts_[dev];
    }

private:
    std::once_flag once_[kMaxDevices];
    LaunchFacts facts_[kMaxDevices];
};

// The number of SMs of the current device (cached per device).
inline int current_sm_count() {
    static std::once_flag once[kMaxDevices];
    static int sms[kMaxDevices];
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 0;
    std::call_once(once[dev], [&] {
        if (cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms[dev] = 0;
    });
    return sms[dev];
}

}  // namespace hgap
