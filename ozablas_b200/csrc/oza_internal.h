// oza_internal.h -- executor state shared by the C-ABI translation units
// (internal to liboza_b200).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include <mutex>

#include "oza_capi.h"

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

// The size limits every GEMM entry point enforces (oza_ws_create,
// oza_gemm_noalloc, oza_group_create, oza_server_submit), in one place:
//   scheme 1 or 2; slices 1..20 (Scheme II: the reference's range; Scheme I:
//   this build's limit); Scheme II products exact in INT32, K * 125^2 < 2^31
//   (K <= 137438); TMA coordinates are 32-bit, so S * Mp, S * Np and Kp stay
//   below 2^31 for the padded extents Mp, Np, Kp of the device layouts.
// Returns OZA_OK, or OZA_INVALID_ARG / OZA_UNSUPPORTED with the text for
// oza_last_error_string() set ("who" prefixes messages that are not the
// reference's own).
oza_status_t check_problem(const char* who, int scheme, size_t M, size_t N, size_t K, int slices);

}  // namespace oza
