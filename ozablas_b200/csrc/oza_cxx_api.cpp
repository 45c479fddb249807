// oza_cxx_api.cpp -- the drop-in C++ API (<ozablas/...>) over the C ABI.
//
// Error mapping follows the reference: std::invalid_argument for a null
// executor or a bad slice count (src/core/workspace.cpp:24-25, 68-71),
// std::bad_alloc for allocation failures (src/core/executor.cpp:79-81),
// std::runtime_error for CUDA failures and for executors without a GPU
// backend (src/ozablas.cpp:42-45, 71-73).
#include <cstdlib>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>

#include "oza_capi.h"
#include "ozablas/core/executor.hpp"
#include "ozablas/core/workspace.hpp"
#include "ozablas/ozablas.hpp"

namespace ozablas {
namespace {

void check(oza_status_t st) {
    if (st == OZA_OK) return;
    std::string msg = oza_last_error_string();
    switch (st) {
        case OZA_INVALID_ARG: throw std::invalid_argument(msg);
        case OZA_OOM: throw std::bad_alloc();
        default: throw std::runtime_error(msg);
    }
}

const CudaExecutor& need_cuda(const std::shared_ptr<const Executor>& exec) {
    if (!exec) throw std::invalid_argument("OzaBLAS: Executor cannot be null.");
    auto* cuda = dynamic_cast<const CudaExecutor*>(exec.get());
    if (!cuda) throw std::runtime_error("OzaBLAS: No suitable hardware backend found for the provided Executor.");
    return *cuda;
}

oza_ws_info_t info_of(oza_workspace* ws) {
    oza_ws_info_t info;
    check(oza_ws_get_info(ws, &info));
    return info;
}

unsigned layout_flags(WorkspaceLayout layout) {
    return layout == WorkspaceLayout::Reference ? OZA_WS_REFERENCE_LAYOUT : 0u;
}

void* buf(oza_workspace* ws, int which) {
    void* p = nullptr;
    check(oza_ws_get_ptr(ws, which, &p));
    return p;
}

}  // namespace

// ------------------------------------------------------------- CpuExecutor
constexpr size_t kCpuAlign = 64;

void CpuExecutor::allocate(void** ptr, size_t bytes) const {
    size_t n = (bytes + kCpuAlign - 1) & ~(kCpuAlign - 1);
    *ptr = std::aligned_alloc(kCpuAlign, n ? n : kCpuAlign);
    if (!*ptr) throw std::bad_alloc();
}
void CpuExecutor::free(void* ptr) const { std::free(ptr); }
void CpuExecutor::copy_from_host(void* d, const void* s, size_t n) const { std::memcpy(d, s, n); }
void CpuExecutor::copy_to_host(void* d, const void* s, size_t n) const { std::memcpy(d, s, n); }
void CpuExecutor::copy_device_to_device(void* d, const void* s, size_t n) const { std::memcpy(d, s, n); }
void CpuExecutor::synchronize() const {}

// ------------------------------------------------------------- CudaExecutor
CudaExecutor::CudaExecutor(int device_id) : device_id_(device_id), handle_(nullptr) {
    oza_status_t st = oza_executor_create(device_id, &handle_);
    if (st != OZA_OK) throw std::runtime_error(std::string("CUDA: Failed to set device. ") + oza_last_error_string());
}
CudaExecutor::~CudaExecutor() { oza_executor_destroy(handle_); }
void CudaExecutor::allocate(void** ptr, size_t bytes) const {
    if (oza_executor_alloc(handle_, ptr, bytes) != OZA_OK) throw std::bad_alloc();
}
void CudaExecutor::free(void* ptr) const { oza_executor_free(handle_, ptr); }
void CudaExecutor::copy_from_host(void* d, const void* s, size_t n) const {
    if (oza_executor_copy(handle_, d, s, n, 1) != OZA_OK) throw std::runtime_error("CUDA: Memcpy HostToDevice failed.");
}
void CudaExecutor::copy_to_host(void* d, const void* s, size_t n) const {
    if (oza_executor_copy(handle_, d, s, n, 2) != OZA_OK) throw std::runtime_error("CUDA: Memcpy DeviceToHost failed.");
}
void CudaExecutor::copy_device_to_device(void* d, const void* s, size_t n) const {
    if (oza_executor_copy(handle_, d, s, n, 3) != OZA_OK)
        throw std::runtime_error("CUDA: Memcpy DeviceToDevice failed.");
}
void CudaExecutor::synchronize() const {
    if (oza_executor_synchronize(handle_) != OZA_OK) throw std::runtime_error("CUDA: Device synchronize failed.");
}
void* CudaExecutor::get_blas_handle() const { return oza_executor_blas_handle(handle_); }
void CudaExecutor::set_stream(void* stream) const { check(oza_executor_set_stream(handle_, stream)); }

HipExecutor::HipExecutor(int) { throw std::runtime_error("OzaBLAS was not compiled with HIP support."); }

// ------------------------------------------------------------- workspaces
WorkspaceScheme1::WorkspaceScheme1(std::shared_ptr<const Executor> exec, size_t M, size_t N, size_t K, int slices)
    : WorkspaceScheme1(std::move(exec), M, N, K, slices, WorkspaceLayout::Device) {}

WorkspaceScheme1::WorkspaceScheme1(std::shared_ptr<const Executor> exec, size_t M, size_t N, size_t K, int slices,
                                   WorkspaceLayout layout)
    : exec_(std::move(exec)), M_(M), N_(N), K_(K), slices_(slices) {
    if (!exec_) throw std::invalid_argument("OzaBLAS: Executor cannot be null.");
    if (slices_ < 1) throw std::invalid_argument("OzaBLAS: Slices must be >= 1.");
    const CudaExecutor& cu = need_cuda(exec_);
    check(oza_ws_create(cu.native(), OZA_SCHEME1, M, N, K, slices, layout_flags(layout), &ws_));
}
WorkspaceScheme1::~WorkspaceScheme1() { oza_ws_destroy(ws_); }
int32_t* WorkspaceScheme1::get_shift_A() const { return static_cast<int32_t*>(buf(ws_, OZA_BUF_SHIFT_A)); }
int32_t* WorkspaceScheme1::get_shift_B() const { return static_cast<int32_t*>(buf(ws_, OZA_BUF_SHIFT_B)); }
int8_t* WorkspaceScheme1::get_A_slices() const { return static_cast<int8_t*>(buf(ws_, OZA_BUF_A_SLICES)); }
int8_t* WorkspaceScheme1::get_B_slices() const { return static_cast<int8_t*>(buf(ws_, OZA_BUF_B_SLICES)); }
int32_t* WorkspaceScheme1::get_C_tc() const { return static_cast<int32_t*>(buf(ws_, OZA_BUF_C_TC)); }
size_t WorkspaceScheme1::get_Mp() const { return info_of(ws_).Mp; }
size_t WorkspaceScheme1::get_Np() const { return info_of(ws_).Np; }
size_t WorkspaceScheme1::get_Kp() const { return info_of(ws_).Kp; }

WorkspaceScheme2::WorkspaceScheme2(std::shared_ptr<const Executor> exec, size_t M, size_t N, size_t K, int slices)
    : WorkspaceScheme2(std::move(exec), M, N, K, slices, WorkspaceLayout::Device) {}

WorkspaceScheme2::WorkspaceScheme2(std::shared_ptr<const Executor> exec, size_t M, size_t N, size_t K, int slices,
                                   WorkspaceLayout layout)
    : exec_(std::move(exec)), M_(M), N_(N), K_(K), slices_(slices) {
    if (!exec_) throw std::invalid_argument("OzaBLAS: Executor cannot be null.");
    if (slices_ < 1 || slices_ > 20) throw std::invalid_argument("OzaBLAS: Scheme II supports between 1 and 20 slices.");
    const CudaExecutor& cu = need_cuda(exec_);
    check(oza_ws_create(cu.native(), OZA_SCHEME2, M, N, K, slices, layout_flags(layout), &ws_));
}
WorkspaceScheme2::~WorkspaceScheme2() { oza_ws_destroy(ws_); }
int32_t* WorkspaceScheme2::get_shift_A() const { return static_cast<int32_t*>(buf(ws_, OZA_BUF_SHIFT_A)); }
int32_t* WorkspaceScheme2::get_shift_B() const { return static_cast<int32_t*>(buf(ws_, OZA_BUF_SHIFT_B)); }
int8_t* WorkspaceScheme2::get_A_slices() const { return static_cast<int8_t*>(buf(ws_, OZA_BUF_A_SLICES)); }
int8_t* WorkspaceScheme2::get_B_slices() const { return static_cast<int8_t*>(buf(ws_, OZA_BUF_B_SLICES)); }
int32_t* WorkspaceScheme2::get_C_tc() const { return static_cast<int32_t*>(buf(ws_, OZA_BUF_C_TC)); }
size_t WorkspaceScheme2::get_Mp() const { return info_of(ws_).Mp; }
size_t WorkspaceScheme2::get_Np() const { return info_of(ws_).Np; }
size_t WorkspaceScheme2::get_Kp() const { return info_of(ws_).Kp; }

// ------------------------------------------------------------- entry points
static void run(oza_workspace* ws, const double* A, const double* B, double* C, OzaTimings* timings) {
    oza_timings_t t{};
    check(oza_gemm(ws, A, B, C, timings ? &t : nullptr));
    if (timings) {
        timings->step1_ms = t.step1_ms;
        timings->step2_ms = t.step2_ms;
        timings->step3_ms = t.step3_ms;
        timings->step4_ms = t.step4_ms;
        timings->total_ms = t.total_ms;
    }
}

void ozaki_scheme1_gemm(WorkspaceScheme1& ws, const double* A, const double* B, double* C, OzaTimings* timings) {
    need_cuda(ws.get_executor());
    run(ws.native(), A, B, C, timings);
}

void ozaki_scheme2_gemm(WorkspaceScheme2& ws, const double* A, const double* B, double* C, OzaTimings* timings) {
    need_cuda(ws.get_executor());
    run(ws.native(), A, B, C, timings);
}

}  // namespace ozablas
