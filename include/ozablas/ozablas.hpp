// <ozablas/ozablas.hpp> -- drop-in public API of the B200-native build.
// Same entry points as the reference header include/ozablas/ozablas.hpp:20,31
// of IlyaNyrkov/ozablas; implemented in ozablas_b200/csrc/oza_cxx_api.cpp over
// the C ABI of <oza_capi.h>.
#pragma once

namespace ozablas {

class WorkspaceScheme1;
class WorkspaceScheme2;
struct OzaTimings;

/**
 * C = A * B with Ozaki Scheme I (sum and scale).  A (M x K), B (K x N) and
 * C (M x N) are row-major FP64 device buffers of the workspace's executor
 * device.  Asynchronous unless `timings` is given.
 * Throws std::runtime_error on a CUDA failure.
 */
void ozaki_scheme1_gemm(WorkspaceScheme1& ws, const double* A, const double* B, double* C,
                        OzaTimings* timings = nullptr);

/**
 * C = A * B with Ozaki Scheme II (Chinese remainder theorem over `slices`
 * moduli).  Same conventions as ozaki_scheme1_gemm.
 */
void ozaki_scheme2_gemm(WorkspaceScheme2& ws, const double* A, const double* B, double* C,
                        OzaTimings* timings = nullptr);

}  // namespace ozablas
