// oza_internal.h -- executor state shared by the C-ABI translation units
// (internal to liboza_b200).
#pragma once

#include <cuda_runtime.h>

#include <mutex>

struct oza_executor {
    int device = 0;
    int sms = 0;
    cudaStream_t stream = nullptr;   // legacy default stream unless set
    void* blas = nullptr;            // cuBLAS handle created on first request
    std::mutex blas_mu;
};

namespace oza {

// Make the executor's device current for the duration of a call.
struct DeviceGuard {
    int prev = -1;
    bool ok = true;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) ok = cudaSetDevice(dev) == cudaSuccess;
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace oza
