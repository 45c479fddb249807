// oza_tune.cu -- accuracy tools: a double-double reference GEMM on a sampled
// block, the sampled maximum relative error, and the slice-count autotuner.
//
// The Ozaki result for a block of rows I and columns J of C depends only on
// the rows I of A and the columns J of B: the step-1 shifts of a row of A (a
// column of B) are taken over that row (column) alone.  So the pipeline run on
// the gathered block A[I,:] x B[:,J] returns exactly the (I, J) entries of the
// full run, and its error against a double-double reference of the same block
// measures the full run's error on those entries.  The autotuner uses this to
// pick the smallest slice count whose sampled error meets a target.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <random>
#include <string>
#include <vector>

#include "oza_capi.h"
#include "oza_kernels.h"

namespace oza {
namespace {

// Error-free transformations (Knuth two-sum, FMA two-product).
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
    s = __dadd_rn(a, b);
    const double bb = __dsub_rn(s, a);
    e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
}

__device__ __forceinline__ void dd_add(double& hi, double& lo, double bh, double bl) {
    double s, e;
    two_sum(hi, bh, s, e);
    e = __dadd_rn(e, __dadd_rn(lo, bl));
    hi = __dadd_rn(s, e);
    lo = __dsub_rn(e, __dsub_rn(hi, s));
}

// One warp per output entry of an r x c block: C[i][j] = sum_k A[i][k] B[k][j]
// in double-double (products split exactly with FMA), rounded to double.
// A is r x K (row-major), B is K x c (row-major).
__global__ void __launch_bounds__(256) k_dd_block_gemm(const double* __restrict__ A, const double* __restrict__ B,
                                                       int r, int c, long long K, double* __restrict__ C) {
    const int lane = threadIdx.x & 31;
    const long long w = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (w >= (long long)r * c) return;
    const int i = (int)(w / c), j = (int)(w - (long long)i * c);
    double hi = 0.0, lo = 0.0;
    for (long long k = lane; k < K; k += 32) {
        const double a = A[(size_t)i * K + k], b = B[(size_t)k * c + j];
        const double p = __dmul_rn(a, b);
        const double pe = __fma_rn(a, b, -p);
        dd_add(hi, lo, p, pe);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double oh = __shfl_xor_sync(0xFFFFFFFFu, hi, o);
        const double ol = __shfl_xor_sync(0xFFFFFFFFu, lo, o);
        dd_add(hi, lo, oh, ol);
    }
    if (lane == 0) C[w] = __dadd_rn(hi, lo);
}

// Gather rows `rows` of A (M x K) into Ab (r x K) and columns `cols` of B (K x N)
// into Bb (K x c).
__global__ void k_gather_rows(const double* __restrict__ A, long long K, const long long* __restrict__ rows, int r,
                              double* __restrict__ Ab) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < (long long)r * K;
         t += (long long)gridDim.x * blockDim.x) {
        const long long i = t / K, k = t - i * K;
        Ab[t] = A[rows[i] * K + k];
    }
}

__global__ void k_gather_cols(const double* __restrict__ B, long long K, long long N, const long long* __restrict__ cols,
                              int c, double* __restrict__ Bb) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < (long long)c * K;
         t += (long long)gridDim.x * blockDim.x) {
        const long long k = t / c, j = t - k * c;
        Bb[t] = B[k * N + cols[j]];
    }
}

}  // namespace

cudaError_t launch_dd_block_gemm(const double* A, const double* B, int r, int c, size_t K, double* C,
                                 cudaStream_t st) {
    const long long warps = (long long)r * c;
    if (warps == 0) return cudaSuccess;
    k_dd_block_gemm<<<(unsigned)((warps + 7) / 8), 256, 0, st>>>(A, B, r, c, (long long)K, C);
    return cudaGetLastError();
}

cudaError_t launch_gather_block(const double* A, const double* B, size_t M, size_t N, size_t K,
                                const long long* rows, int r, const long long* cols, int c, double* Ab, double* Bb,
                                cudaStream_t st) {
    (void)M;
    k_gather_rows<<<592, 256, 0, st>>>(A, (long long)K, rows, r, Ab);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_gather_cols<<<592, 256, 0, st>>>(B, (long long)K, (long long)N, cols, c, Bb);
    return cudaGetLastError();
}

}  // namespace oza
