// eu3d_attr.hpp — dynamic shared-memory limits of kernels, set per device.
//
// cudaFuncSetAttribute(..., cudaFuncAttributeMaxDynamicSharedMemorySize, ...)
// applies to the current device only, so a launcher that raises a kernel's
// limit above the 48 KB default must do it once on every device it launches
// on. SmemLimit keeps, per device ordinal, the largest size already set for
// one kernel; concurrent callers may both set it, which is harmless.
#pragma once

#include <atomic>
#include <cstddef>

#include <cuda_runtime.h>

namespace eu3d {

class SmemLimit {
public:
    static constexpr int kDevices = 64;

    // Raise `kernel`'s limit on the current device to at least `bytes`.
    template <class Kernel>
    cudaError_t ensure(Kernel kernel, size_t bytes)
    {
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess)
            return e;
        std::atomic<size_t> *slot = (dev >= 0 && dev < kDevices) ? &set_[dev] : nullptr;
        if (slot && slot->load(std::memory_order_acquire) >= bytes)
            return cudaSuccess;
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
        if (e != cudaSuccess)
            return e;
        if (slot) {
            size_t cur = slot->load(std::memory_order_relaxed);
            while (cur < bytes && !slot->compare_exchange_weak(cur, bytes, std::memory_order_acq_rel)) {
            }
        }
        return cudaSuccess;
    }

private:
    std::atomic<size_t> set_[kDevices] = {};
};

} // namespace eu3d
