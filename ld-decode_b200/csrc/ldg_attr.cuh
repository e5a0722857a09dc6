// Per-device kernel attributes.
//
// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) applies to the device that
// is current when it is called, so a kernel launched on several devices from
// one process needs it once per device.  SmemAttr remembers, per device, the
// largest size already set, under a mutex (launches come from several host
// threads).  The caller makes the launch's device current first.
#pragma once
#include <cuda_runtime.h>

#include <mutex>

namespace ldg {

class SmemAttr {
   public:
    static constexpr int kMaxDevices = 64;

    template <class K>
    cudaError_t ensure(K* kernel, size_t bytes) {
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
        std::lock_guard<std::mutex> lk(mu_);
        if (set_[dev] >= bytes) return cudaSuccess;
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e == cudaSuccess) set_[dev] = bytes;
        return e;
    }

   private:
    std::mutex mu_;
    size_t set_[kMaxDevices] = {};
};

}  // namespace ldg
