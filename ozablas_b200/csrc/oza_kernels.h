// oza_kernels.h -- host-side launch wrappers of the sm_100a kernels
// (internal to liboza_b200; the public boundary is include/oza_capi.h).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace oza {

constexpr int kMaxSlicesHost = 20;

// Tile geometry of the INT8 tensor-core GEMM and the padding it imposes on
// the workspace layouts.
constexpr int kTileM = 128;   // rows of A per CTA tile (UMMA M)
constexpr int kTileN = 256;   // rows of B^T per CTA tile (UMMA N)
constexpr int kTileK = 128;   // bytes of K per pipeline stage (one 128B swizzle row)

inline size_t round_up(size_t x, size_t m) { return (x + m - 1) / m * m; }

// Which (A-plane, B-plane) products are summed into each INT32 group.
// Scheme II: group s = A_s * B_s.  Scheme I: group g (plane g-2) sums
// A_s * B_t over s + t = g (1-based slice indices), s, t <= S.
// Accumulation units of the GEMM: Scheme II one per modulus; Scheme I one per
// group g = s + t, split into consecutive sub-groups where the group's INT32
// sum could overflow (more than (2^31 - 1) / (K 2^(2 beta - 2)) pairs: each
// slice product is at most 2^(2 beta - 2) in magnitude), so every INT32
// accumulator stays exact.  Each unit is one INT32 (or coefficient) plane.
constexpr int kMaxUnits = 80;   // Scheme I, S = 20, at least 3 pairs per unit: 77
struct PairList {
    int num_groups;                      // units
    int start[kMaxUnits + 1];            // pairs of unit u: [start[u], start[u + 1])
    int first_unit[kMaxSlicesHost + 1];  // Scheme I: units of group g: [first_unit[g], first_unit[g + 1])
    uint8_t a[kMaxSlicesHost * (kMaxSlicesHost + 1) / 2];
    uint8_t b[kMaxSlicesHost * (kMaxSlicesHost + 1) / 2];
};
PairList make_pairs(int scheme, int slices, size_t K);

// Upload the per-modulus and CRT constants to the current device.
cudaError_t upload_tables();

// Step 1.
cudaError_t launch_stats_rows(const double* A, size_t rows, size_t cols, int offset, int32_t* shift,
                              int sms, cudaStream_t st);
cudaError_t launch_stats_cols(const double* B, size_t rows, size_t cols, unsigned long long* colmax, int sms,
                              cudaStream_t st);

// Step 2.  scheme 1: slices with width beta from shifts (offset 0);
// scheme 2: symmetric residues of rint(ldexp(x, shift)).
// Rows: A (rows x cols, row-major) -> out[s][rows_p][cols_p].
// plane_rows: rows between planes of `out` (0: rows_p), so a row chunk can be
// sliced into its place in full-size planes.
// err: device error word; with it, Scheme II with S <= 16 forms the digit
// products on the tensor cores (a bounded wait that expires records
// kErrWaitTimeout there), without it on the CUDA cores.
cudaError_t launch_slice_rows(int scheme, const double* A, size_t rows, size_t cols, const int32_t* shift,
                              int S, int beta, int k_param, int8_t* out, size_t rows_p, size_t cols_p, int sms,
                              cudaStream_t st, size_t plane_rows = 0, int* err = nullptr);
// Columns: B (K x N, row-major) -> out[s][Np][Kp] (transposed, K-major); also
// writes shift[n] = offset - max exponent of column n.
cudaError_t launch_slice_cols(int scheme, const double* B, size_t K, size_t N, const unsigned long long* colmax,
                              int offset, int S, int beta, int32_t* shift, int8_t* out, size_t Np, size_t Kp,
                              cudaStream_t st, int* err = nullptr);
// Process-wide choice of the Scheme II residue slicer: 0 (default) tensor-core
// digit products where S <= 16, 1 CUDA cores only.  Both give identical planes.
void set_residue_slicer(int mode);
int residue_slicer();

// Step 3.
struct GemmPlan {
    const int8_t* a_planes;   // [planes][Mp][Kp]
    const int8_t* b_planes;   // [planes][Np][Kp]
    int planes;
    size_t Mp, Np, Kp;
    size_t M = 0, N = 0;      // real extents (0: Mp, Np); the epilogue skips whole padding quadrants and chunks
    PairList pairs;
    int* err;                 // device error word
    int sms;
    // epilogue output: INT32 group planes, or (Scheme II) CRT coefficient bytes
    int32_t* ctc;             // [groups][Mp][Np], used when coef == nullptr
    uint8_t* coef;            // [S][Mp][Np]
    int m_tile_begin = 0;     // restrict the launch to m-tiles [begin, begin + count) (count 0: to the end)
    int m_tile_count = 0;
    // Tuning (0: defaults): m-tiles per rasterisation band.
    int band = 0;
    uint32_t wait_hint_ns = 0;   // mbarrier suspend-time hint of the kernel's waits (0: poll)
};
cudaError_t launch_gemm_i8(const GemmPlan& plan, cudaStream_t st);

// Step 4.
cudaError_t launch_reconstruct2(const int32_t* ctc, size_t Mp, size_t Np, size_t M, size_t N, int S,
                                const int32_t* shiftA, const int32_t* shiftB, double* C, cudaStream_t st);
// Scheme II step 4 from the GEMM's coefficient byte planes.
cudaError_t launch_crt_coef(const uint8_t* coef, size_t Mp, size_t Np, size_t M, size_t N, int S,
                            const int32_t* shiftA, const int32_t* shiftB, double* C, int sms, cudaStream_t st);
cudaError_t launch_reconstruct1(const int32_t* ctc, size_t Mp, size_t Np, size_t M, size_t N, int S, int beta,
                                const int32_t* negA, const int32_t* negB, double* C, int sms, cudaStream_t st,
                                const PairList* units = nullptr);

// Grouped Scheme II: many independent GEMMs, each stage one launch (the
// slicers and the CRT one per slice-count class).  Buffers as in a Scheme II
// workspace, per problem; colmax of all problems is one contiguous array.
struct GroupProblem {
    const double* A;
    const double* B;
    double* C;
    size_t M, N, K, Mp, Np, Kp;
    int S, k_param;
    int32_t* shiftA;
    int32_t* shiftB;
    unsigned long long* colmax;
    int8_t* a_planes;   // [S][Mp][Kp]
    int8_t* b_planes;   // [S][Np][Kp]
    uint8_t* coef;      // [S][Mp][Np]
};
struct GroupPlan;   // device tables: problems, per-stage block maps, GEMM work units, tensor maps
cudaError_t group_plan_create(const GroupProblem* probs, int count, int* err, GroupPlan** out);
// The same tables without device memory: a host image of group_plan_table_bytes()
// (group_plan_image) that the caller copies to device memory it owns, then binds.
cudaError_t group_plan_build(const GroupProblem* probs, int count, int* err, GroupPlan** out);
const void* group_plan_image(const GroupPlan* p);
void group_plan_bind(GroupPlan* p, void* dev_tables);
void group_plan_destroy(GroupPlan* p);
// New A/B/C pointers for the next launches (stream-ordered upload when changed).
cudaError_t group_plan_set_matrices(GroupPlan* p, const double* const* A, const double* const* B,
                                    double* const* C, cudaStream_t st);
// Steps 1-4 of every problem; ev (optional) = 5 events bracketing the steps.
cudaError_t group_plan_launch(GroupPlan* p, unsigned long long* colmax, size_t colmax_count, int sms,
                              cudaStream_t st, cudaEvent_t* ev);
size_t group_plan_units(const GroupPlan* p);
size_t group_plan_table_bytes(const GroupPlan* p);
int group_plan_launches(const GroupPlan* p);   // kernel launches per call

// Copies of the intermediates in the reference's layouts: A slices [S][M][K],
// B slices [S][K][N] (from the K-major B^T planes) and INT32 groups
// [c_count][M][N] (groups c_first.. of the [groups][Mp][Np] planes).
cudaError_t launch_to_reference_layout(const int8_t* a_planes, const int8_t* b_planes, const int32_t* ctc, int S,
                                      int groups, size_t M, size_t N, size_t K, size_t Mp, size_t Np, size_t Kp,
                                      int8_t* a_ref, int8_t* b_ref, int32_t* c_ref, int c_first, int c_count,
                                      bool sum_planes, cudaStream_t st);

// One bounded wait on an mbarrier that nothing arrives on (self-test of the
// wait bound): *gerr receives the device error code, *status 1 if it returned early.
cudaError_t launch_wait_probe(int* gerr, unsigned long long limit_ns, int* status, cudaStream_t st);

// Sets the text returned by oza_last_error_string() on this thread.
void set_last_error(const char* msg);

}  // namespace oza
