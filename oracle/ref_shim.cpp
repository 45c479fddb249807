// ref_shim.cpp -- runs the reference's own step-1/2/4 kernel source on the CPU.
//
// TEST INFRASTRUCTURE ONLY (parity pinning).  This translation unit includes
// the unmodified OzaBLAS device headers from the reference source tree
//   src/pipeline/step1_statistics.hpp, step2_slicing.hpp, step4_reconstruction.hpp
// through a macro shim that turns CUDA/HIP kernel syntax into host C++, and
// exports one extern "C" launcher per kernel.  Each launcher emulates the
// reference's launch with one-thread blocks (blockDim = 1), which makes the
// in-block reductions of compute_row_shifts_A degenerate to a serial loop.
//
// Built by oracle/Makefile into oracle/_ref/libozaref_cpu.so; nothing from
// the reference is copied into this repository.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>

struct ShimDim3 { unsigned x = 0, y = 0, z = 0; };
static thread_local ShimDim3 blockIdx, threadIdx, blockDim;
static const int warpSize = 1;

#define __global__
#define __device__
#define __host__
#define __constant__
#define __shared__ static thread_local
// The reference reads its CRT tables from __constant__ arrays only when a GPU
// compiler macro is defined (step2_slicing.hpp:229-233, step4_reconstruction.hpp:72-77);
// the host fallbacks there are placeholders.  Defining __HIPCC__ selects the
// table branch; the shuffle it would use is never executed with warpSize == 1.
#define __HIPCC__ 1
template <class T> static inline T __shfl_down(T v, int) { return v; }
static inline void __syncthreads() {}
using std::max;

#include "pipeline/step1_statistics.hpp"
#include "pipeline/step2_slicing.hpp"
#include "pipeline/step4_reconstruction.hpp"

using namespace ozablas;

static void shim_upload_tables() {
    std::memcpy(OZA_c_moduli_all, crt::moduli_all, sizeof(crt::moduli_all));
    std::memcpy(OZA_c_M_prod_20, crt::M_prod_20, sizeof(crt::M_prod_20));
    std::memcpy(OZA_c_M_half_20, crt::M_half_20, sizeof(crt::M_half_20));
    std::memcpy(OZA_c_partial_moduli_20, crt::partial_moduli_20, sizeof(crt::partial_moduli_20));
    std::memcpy(OZA_c_mod_inv_20, crt::mod_inv_20, sizeof(crt::mod_inv_20));
}

static void set_block(unsigned bx, unsigned by) {
    blockIdx.x = bx; blockIdx.y = by; blockIdx.z = 0;
    threadIdx.x = threadIdx.y = threadIdx.z = 0;
    blockDim.x = blockDim.y = blockDim.z = 1;
}

extern "C" {

void ref_init_tables() { shim_upload_tables(); }

// Raw tables as the reference ships them, for table known-answer tests.
void ref_get_tables(uint8_t* moduli, uint64_t* Mprod, uint64_t* Mhalf, uint64_t* partial, uint64_t* inv) {
    std::memcpy(moduli, crt::moduli_all, sizeof(crt::moduli_all));
    std::memcpy(Mprod, crt::M_prod_20, sizeof(crt::M_prod_20));
    std::memcpy(Mhalf, crt::M_half_20, sizeof(crt::M_half_20));
    std::memcpy(partial, crt::partial_moduli_20, sizeof(crt::partial_moduli_20));
    std::memcpy(inv, crt::mod_inv_20, sizeof(crt::mod_inv_20));
}

int ref_scheme1_beta(int K) { return pipeline::calculate_scheme1_beta(K); }

// Host computation of K_param exactly as src/cuda/pipeline.cu:196-198 does it.
int ref_scheme2_kparam(int S, int K) {
    crt::uint256_t M(crt::M_prod_20[S - 1]);
    return pipeline::calculate_scheme2_k_param(crt::to_double_256(M), K);
}

void ref_row_shifts(const double* A, int rows, int cols, int offset, int32_t* shifts) {
    #pragma omp parallel for schedule(static)
    for (int r = 0; r < rows; ++r) { set_block(r, 0); pipeline::compute_row_shifts_A(A, rows, cols, offset, shifts); }
}

void ref_col_shifts(const double* B, int rows, int cols, int offset, int32_t* shifts) {
    #pragma omp parallel for schedule(static)
    for (int c = 0; c < cols; ++c) { set_block(c, 0); pipeline::compute_col_shifts_B(B, rows, cols, offset, shifts); }
}

void ref_slice2(const double* X, int rows, int cols, const int32_t* shifts, int per_row, int S, int8_t* out) {
    shim_upload_tables();
    #pragma omp parallel for schedule(static)
    for (int r = 0; r < rows; ++r)
        for (int c = 0; c < cols; ++c) {
            set_block(c, r);
            if (per_row) pipeline::slice_scheme2_A(X, shifts, rows, cols, S, out);
            else pipeline::slice_scheme2_B(X, shifts, rows, cols, S, out);
        }
}

// The reference casts NaN to int8 in Scheme I for an all-zero row (0 * inf);
// on the host that cast is undefined, on the GPU it yields 0.  The shim runs
// the kernel and then rewrites the slices of all-zero rows/columns to 0.
void ref_slice1(const double* X, int rows, int cols, const int32_t* neg_exp, int per_row, int S, int beta, int8_t* out) {
    #pragma omp parallel for schedule(static)
    for (int r = 0; r < rows; ++r)
        for (int c = 0; c < cols; ++c) {
            set_block(c, r);
            if (per_row) pipeline::slice_scheme1_A(X, neg_exp, rows, cols, S, beta, out);
            else pipeline::slice_scheme1_B(X, neg_exp, rows, cols, S, beta, out);
        }
    const size_t plane = (size_t)rows * cols;
    for (int r = 0; r < rows; ++r)
        for (int c = 0; c < cols; ++c) {
            int ne = per_row ? neg_exp[r] : neg_exp[c];
            if (ne == 1023) for (int s = 0; s < S; ++s) out[s * plane + (size_t)r * cols + c] = 0;
        }
}

void ref_reconstruct2(const int32_t* Ctc, const int32_t* sA, const int32_t* sB, int M, int N, int S, double* C) {
    shim_upload_tables();
    #pragma omp parallel for schedule(static)
    for (int r = 0; r < M; ++r)
        for (int c = 0; c < N; ++c) {
            set_block(c, r);
            if (S <= 7) pipeline::reconstruct_scheme2_leq7(Ctc, sA, sB, M, N, S, C);
            else pipeline::reconstruct_scheme2_gt7(Ctc, sA, sB, M, N, S, C);
        }
}

void ref_reconstruct1_group(const int32_t* Cg, const int32_t* negA, const int32_t* negB, int M, int N, int g, int beta, double* C) {
    #pragma omp parallel for schedule(static)
    for (int r = 0; r < M; ++r)
        for (int c = 0; c < N; ++c) {
            set_block(c, r);
            pipeline::reconstruct_scheme1_group(Cg, negA, negB, M, N, g, beta, C);
        }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Whole CPU pipelines over the reference kernels.  The reference has no CPU
// GEMM (its step 3 is cuBLAS, src/cuda/pipeline.cu:117-124, :228-235), so
// step 3 here is a plain exact INT8 x INT8 -> INT32 loop of this file's own.
// These are the CPU baseline that bench.py times as the reference arm.
// ---------------------------------------------------------------------------
static void cpu_gemm_i8(const int8_t* A, const int8_t* Bt, int M, int N, int K, int32_t* C, bool acc) {
    #pragma omp parallel for schedule(dynamic, 4)
    for (int i = 0; i < M; ++i) {
        const int8_t* a = A + (size_t)i * K;
        for (int j = 0; j < N; ++j) {
            const int8_t* b = Bt + (size_t)j * K;
            int32_t s = 0;
            for (int k = 0; k < K; ++k) s += (int16_t)a[k] * (int16_t)b[k];
            size_t o = (size_t)i * N + j;
            C[o] = acc ? C[o] + s : s;
        }
    }
}

static void transpose_i8(const int8_t* B, int K, int N, int8_t* Bt) {
    #pragma omp parallel for schedule(static)
    for (int j = 0; j < N; ++j)
        for (int k = 0; k < K; ++k) Bt[(size_t)j * K + k] = B[(size_t)k * N + j];
}

extern "C" {

// Scheme II, src/cuda/pipeline.cu:173-265 with the kernels run on the host.
// Buffers are caller-provided: shifts (M, N), slices (S*M*K, S*K*N),
// Ctc (S*M*N), Bt scratch (K*N).
void ref_cpu_scheme2_gemm(const double* A, const double* B, double* C, int M, int N, int K, int S,
                          int32_t* sA, int32_t* sB, int8_t* As, int8_t* Bs, int32_t* Ctc, int8_t* Bt) {
    int kp = ref_scheme2_kparam(S, K);
    ref_row_shifts(A, M, K, kp, sA);
    ref_col_shifts(B, K, N, kp, sB);
    ref_slice2(A, M, K, sA, 1, S, As);
    ref_slice2(B, K, N, sB, 0, S, Bs);
    for (int s = 0; s < S; ++s) {
        transpose_i8(Bs + (size_t)s * K * N, K, N, Bt);
        cpu_gemm_i8(As + (size_t)s * M * K, Bt, M, N, K, Ctc + (size_t)s * M * N, false);
    }
    ref_reconstruct2(Ctc, sA, sB, M, N, S, C);
}

// Scheme I, src/cuda/pipeline.cu:40-167.  Ctc holds one M*N group buffer.
void ref_cpu_scheme1_gemm(const double* A, const double* B, double* C, int M, int N, int K, int S,
                          int32_t* sA, int32_t* sB, int8_t* As, int8_t* Bs, int32_t* Ctc, int8_t* Bt) {
    int beta = pipeline::calculate_scheme1_beta(K);
    std::memset(C, 0, sizeof(double) * (size_t)M * N);
    ref_row_shifts(A, M, K, 0, sA);
    ref_col_shifts(B, K, N, 0, sB);
    ref_slice1(A, M, K, sA, 1, S, beta, As);
    ref_slice1(B, K, N, sB, 0, S, beta, Bs);
    for (int g = 2; g <= S + 1; ++g) {
        bool first = true;
        for (int s = 1; s <= g - 1; ++s) {
            int t = g - s;
            if (s > S || t > S) continue;
            transpose_i8(Bs + (size_t)(t - 1) * K * N, K, N, Bt);
            cpu_gemm_i8(As + (size_t)(s - 1) * M * K, Bt, M, N, K, Ctc, !first);
            first = false;
        }
        ref_reconstruct1_group(Ctc, sA, sB, M, N, g, beta, C);
    }
}

}  // extern "C"
