// ref_gpu_driver.cpp -- extern "C" handle over the reference's GPU pipeline.
//
// Comparison infrastructure, not the product.  Linked by baseline/Makefile with
// the reference's own sources (src/cuda/pipeline.cu, src/core/*.cpp,
// src/ozablas.cpp) into baseline/_ref/libozablas_ref_gpu.so.  It drives the
// unmodified reference through its public C++ API
// (include/ozablas/ozablas.hpp, core/executor.hpp, core/workspace.hpp) so that
// tests can compare intermediates and results with the reference itself on a
// B200, and bench.py can time the reference's cuBLAS-backed pipeline and
// cuBLAS DGEMM beside the sm_100a kernels.
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <memory>
#include <stdexcept>

#include "ozablas/core/executor.hpp"
#include "ozablas/core/workspace.hpp"
#include "ozablas/ozablas.hpp"

namespace {
std::shared_ptr<ozablas::CudaExecutor> g_exec;

struct RefWs {
    int scheme;
    std::unique_ptr<ozablas::WorkspaceScheme1> ws1;
    std::unique_ptr<ozablas::WorkspaceScheme2> ws2;
};
}  // namespace

extern "C" {

int refgpu_init(int device) {
    try {
        if (!g_exec) g_exec = std::make_shared<ozablas::CudaExecutor>(device);
        return 0;
    } catch (...) {
        return -1;
    }
}

void* refgpu_ws_create(int scheme, size_t M, size_t N, size_t K, int slices) {
    if (!g_exec) return nullptr;
    try {
        auto* w = new RefWs{scheme, nullptr, nullptr};
        if (scheme == 1) w->ws1 = std::make_unique<ozablas::WorkspaceScheme1>(g_exec, M, N, K, slices);
        else w->ws2 = std::make_unique<ozablas::WorkspaceScheme2>(g_exec, M, N, K, slices);
        return w;
    } catch (...) {
        return nullptr;
    }
}

void refgpu_ws_destroy(void* h) { delete static_cast<RefWs*>(h); }

// which: 0 shift_A, 1 shift_B, 2 A_slices, 3 B_slices, 4 C_tc
void* refgpu_ws_ptr(void* h, int which) {
    auto* w = static_cast<RefWs*>(h);
    if (w->scheme == 1) {
        auto& ws = *w->ws1;
        void* p[5] = {ws.get_shift_A(), ws.get_shift_B(), ws.get_A_slices(), ws.get_B_slices(), ws.get_C_tc()};
        return p[which];
    }
    auto& ws = *w->ws2;
    void* p[5] = {ws.get_shift_A(), ws.get_shift_B(), ws.get_A_slices(), ws.get_B_slices(), ws.get_C_tc()};
    return p[which];
}

// Runs the reference pipeline on device pointers.  timings (5 floats) may be null.
int refgpu_gemm(void* h, const double* A, const double* B, double* C, float* timings) {
    auto* w = static_cast<RefWs*>(h);
    try {
        ozablas::OzaTimings t;
        ozablas::OzaTimings* tp = timings ? &t : nullptr;
        if (w->scheme == 1) ozablas::ozaki_scheme1_gemm(*w->ws1, A, B, C, tp);
        else ozablas::ozaki_scheme2_gemm(*w->ws2, A, B, C, tp);
        if (timings) {
            timings[0] = t.step1_ms; timings[1] = t.step2_ms; timings[2] = t.step3_ms;
            timings[3] = t.step4_ms; timings[4] = t.total_ms;
        }
        return cudaGetLastError() == cudaSuccess ? 0 : -2;
    } catch (...) {
        return -1;
    }
}

// Native cuBLAS DGEMM on row-major operands, as the reference harness calls it
// (performance_benchmarks/01_ozaki_scheme1_2_raw_performance.cpp:59-62).
int refgpu_dgemm(const double* A, const double* B, double* C, int M, int N, int K) {
    if (!g_exec) return -1;
    const double alpha = 1.0, beta = 0.0;
    auto handle = static_cast<cublasHandle_t>(g_exec->get_blas_handle());
    cublasStatus_t st = cublasDgemm(handle, CUBLAS_OP_N, CUBLAS_OP_N, N, M, K, &alpha, B, N, A, K, &beta, C, N);
    return st == CUBLAS_STATUS_SUCCESS ? 0 : -3;
}

int refgpu_sync() { return cudaDeviceSynchronize() == cudaSuccess ? 0 : -2; }

}  // extern "C"
