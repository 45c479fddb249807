// <ozablas/core/executor.hpp> -- drop-in executor classes.
// Mirrors include/ozablas/core/executor.hpp:15-113 of IlyaNyrkov/ozablas:
// an abstract Executor, a host CpuExecutor (kept for API compatibility; the
// GEMM entry points reject it, as the reference's dispatcher does), the
// CudaExecutor that drives the sm_100a kernels, and a HipExecutor whose
// constructor throws because this build has no HIP backend.
#pragma once

#include <cstddef>
#include <memory>
#include <stdexcept>

struct oza_executor;

namespace ozablas {

class Executor {
public:
    virtual ~Executor() = default;
    virtual void allocate(void** ptr, size_t bytes) const = 0;
    virtual void free(void* ptr) const = 0;
    virtual void copy_from_host(void* device_dst, const void* host_src, size_t bytes) const = 0;
    virtual void copy_to_host(void* host_dst, const void* device_src, size_t bytes) const = 0;
    virtual void copy_device_to_device(void* dst, const void* src, size_t bytes) const = 0;
    virtual void synchronize() const = 0;
    /** A cuBLAS handle (cublasHandle_t as void*) for callers that want one;
     *  the Ozaki path itself never uses cuBLAS. */
    virtual void* get_blas_handle() const { return nullptr; }
};

class CpuExecutor : public Executor {
public:
    CpuExecutor() = default;
    ~CpuExecutor() override = default;
    void allocate(void** ptr, size_t bytes) const override;
    void free(void* ptr) const override;
    void copy_from_host(void* device_dst, const void* host_src, size_t bytes) const override;
    void copy_to_host(void* host_dst, const void* device_src, size_t bytes) const override;
    void copy_device_to_device(void* dst, const void* src, size_t bytes) const override;
    void synchronize() const override;
};

class CudaExecutor : public Executor {
public:
    /** Selects `device_id` (must be an sm_100 device). Throws std::runtime_error. */
    explicit CudaExecutor(int device_id = 0);
    ~CudaExecutor() override;
    CudaExecutor(const CudaExecutor&) = delete;
    CudaExecutor& operator=(const CudaExecutor&) = delete;

    void allocate(void** ptr, size_t bytes) const override;   // throws std::bad_alloc
    void free(void* ptr) const override;
    void copy_from_host(void* device_dst, const void* host_src, size_t bytes) const override;
    void copy_to_host(void* host_dst, const void* device_src, size_t bytes) const override;
    void copy_device_to_device(void* dst, const void* src, size_t bytes) const override;
    void synchronize() const override;
    void* get_blas_handle() const override;

    /** Extension: run subsequent work on a cudaStream_t (nullptr = default stream). */
    void set_stream(void* stream) const;
    int device() const { return device_id_; }
    oza_executor* native() const { return handle_; }

private:
    int device_id_;
    oza_executor* handle_;
};

class HipExecutor : public Executor {
public:
    explicit HipExecutor(int device_id = 0);   // always throws: no HIP backend in this build
    ~HipExecutor() override = default;
    void allocate(void**, size_t) const override {}
    void free(void*) const override {}
    void copy_from_host(void*, const void*, size_t) const override {}
    void copy_to_host(void*, const void*, size_t) const override {}
    void copy_device_to_device(void*, const void*, size_t) const override {}
    void synchronize() const override {}
};

}  // namespace ozablas
