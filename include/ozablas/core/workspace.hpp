// <ozablas/core/workspace.hpp> -- drop-in workspaces and OzaTimings.
// Mirrors include/ozablas/core/workspace.hpp:14-103 of IlyaNyrkov/ozablas.
//
// Layout note: by default the device buffers are laid out for the sm_100a
// kernels, not as in the reference.  Slices/residues are K-major and padded
// (zeros in the K padding; rows past M and N unwritten): get_A_slices() is
// int8 [S][Mp][Kp], get_B_slices() is int8 [S][Np][Kp] (B transposed), get_C_tc() is int32 [S][Mp][Np] with plane g
// holding group g (Scheme II: residue g; Scheme I: slice-sum group g+2; at large K
// a Scheme I group can span several planes, each an exact INT32 sum of some of its
// slice pairs: oza_ws_info_t::groups planes), and null for Scheme II, whose INT32
// products never reach memory.  The padded
// extents are get_Mp()/get_Np()/get_Kp().  Constructed with
// WorkspaceLayout::Reference, the getters return the reference's own layouts
// instead, refreshed by every GEMM call: A slices [S][M][K], B slices
// [S][K][N], C_tc [S][M][N] (Scheme II) or the last group [M][N] (Scheme I).
#pragma once

#include <cstddef>
#include <cstdint>
#include <memory>

#include "ozablas/core/executor.hpp"

struct oza_workspace;

namespace ozablas {

/** Layout of the intermediates the workspace getters expose (extension). */
enum class WorkspaceLayout {
    Device,      ///< the sm_100a kernels' padded K-major planes (default)
    Reference,   ///< also kept in the reference's layouts, returned by the getters
};

class WorkspaceScheme1 {
public:
    /** Throws std::invalid_argument (null executor, slices < 1), std::bad_alloc,
     *  std::runtime_error (executor is not a CudaExecutor or CUDA failure). */
    WorkspaceScheme1(std::shared_ptr<const Executor> exec, size_t M, size_t N, size_t K, int slices);
    WorkspaceScheme1(std::shared_ptr<const Executor> exec, size_t M, size_t N, size_t K, int slices,
                     WorkspaceLayout layout);
    ~WorkspaceScheme1();
    WorkspaceScheme1(const WorkspaceScheme1&) = delete;
    WorkspaceScheme1& operator=(const WorkspaceScheme1&) = delete;

    std::shared_ptr<const Executor> get_executor() const { return exec_; }
    size_t get_M() const { return M_; }
    size_t get_N() const { return N_; }
    size_t get_K() const { return K_; }
    int get_slices() const { return slices_; }
    int32_t* get_shift_A() const;
    int32_t* get_shift_B() const;
    int8_t* get_A_slices() const;
    int8_t* get_B_slices() const;
    int32_t* get_C_tc() const;
    size_t get_Mp() const;
    size_t get_Np() const;
    size_t get_Kp() const;
    oza_workspace* native() const { return ws_; }

private:
    std::shared_ptr<const Executor> exec_;
    size_t M_, N_, K_;
    int slices_;
    oza_workspace* ws_ = nullptr;
};

class WorkspaceScheme2 {
public:
    /** Throws std::invalid_argument (null executor, slices outside 1..20),
     *  std::bad_alloc, std::runtime_error. */
    WorkspaceScheme2(std::shared_ptr<const Executor> exec, size_t M, size_t N, size_t K, int slices);
    WorkspaceScheme2(std::shared_ptr<const Executor> exec, size_t M, size_t N, size_t K, int slices,
                     WorkspaceLayout layout);
    ~WorkspaceScheme2();
    WorkspaceScheme2(const WorkspaceScheme2&) = delete;
    WorkspaceScheme2& operator=(const WorkspaceScheme2&) = delete;

    std::shared_ptr<const Executor> get_executor() const { return exec_; }
    size_t get_M() const { return M_; }
    size_t get_N() const { return N_; }
    size_t get_K() const { return K_; }
    int get_slices() const { return slices_; }
    int32_t* get_shift_A() const;
    int32_t* get_shift_B() const;
    int8_t* get_A_slices() const;
    int8_t* get_B_slices() const;
    int32_t* get_C_tc() const;
    size_t get_Mp() const;
    size_t get_Np() const;
    size_t get_Kp() const;
    oza_workspace* native() const { return ws_; }

private:
    std::shared_ptr<const Executor> exec_;
    size_t M_, N_, K_;
    int slices_;
    oza_workspace* ws_ = nullptr;
};

struct OzaTimings {
    float step1_ms = 0.0f;   // exponent statistics
    float step2_ms = 0.0f;   // slicing / residues
    float step3_ms = 0.0f;   // INT8 tensor-core products
    float step4_ms = 0.0f;   // scaled sum / CRT reconstruction
    float total_ms = 0.0f;
};

}  // namespace ozablas
