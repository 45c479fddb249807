/*
 * oza_capi.h -- C ABI of the B200-native Ozaki Scheme I / II FP64 GEMM.
 *
 * Plain C: opaque handles, device pointers and sizes; no CUDA or C++ types in
 * any signature.  The C++ drop-in API (<ozablas/ozablas.hpp>,
 * <ozablas/core/executor.hpp>, <ozablas/core/workspace.hpp>) is implemented on
 * top of these entry points, and the Python bindings (ozablas_b200) load them
 * with ctypes.  Each entry point names the reference interface it replaces
 * (paths relative to the IlyaNyrkov/ozablas source tree).
 *
 * Conventions (same as the reference, include/ozablas/ozablas.hpp:13-31):
 *   A is M x K, B is K x N, C is M x N, all row-major FP64 device buffers with
 *   leading dimensions K, N, N.  C is fully overwritten.  No alpha, beta or
 *   transposes.  Work is issued on the executor's stream (default: the legacy
 *   default stream, as in the reference); the call returns asynchronously
 *   unless a timings struct is passed, in which case it waits for the result.
 *   Inputs must be finite.
 */
#ifndef OZA_CAPI_H
#define OZA_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum oza_status {
    OZA_OK = 0,
    OZA_INVALID_ARG = 1,   /* -> std::invalid_argument in the C++ layer      */
    OZA_OOM = 2,           /* -> std::bad_alloc                                */
    OZA_CUDA_ERROR = 3,    /* -> std::runtime_error                            */
    OZA_TIMEOUT = 4,       /* a bounded device-side wait expired               */
    OZA_UNSUPPORTED = 5    /* valid request this build cannot serve            */
} oza_status_t;

typedef struct oza_executor* oza_exec_t;
typedef struct oza_workspace* oza_ws_t;

/* Per-step device times in milliseconds.
 * Reference: struct OzaTimings, include/ozablas/core/workspace.hpp:97-103. */
typedef struct oza_timings {
    float step1_ms;  /* exponent statistics                         */
    float step2_ms;  /* slicing / residues                          */
    float step3_ms;  /* INT8 tensor-core products                   */
    float step4_ms;  /* scaled sum / CRT reconstruction             */
    float total_ms;
} oza_timings_t;

/* Schemes. */
#define OZA_SCHEME1 1  /* sum-and-scale slices */
#define OZA_SCHEME2 2  /* CRT residues          */

/* Workspace flags. */
#define OZA_WS_MATERIALIZE 0x1u  /* keep every intermediate (slices, INT32 products) in
                                    the workspace buffers, for inspection and parity */
#define OZA_WS_REFERENCE_LAYOUT 0x2u  /* implies MATERIALIZE; after each GEMM also copy the
                                    intermediates into buffers laid out as the reference's
                                    workspace getters return them (see OZA_BUF_*), which
                                    oza_ws_get_ptr then returns; for inspection and for code
                                    that reads the reference's buffers (costs a copy per call) */

/* Buffers exposed by oza_ws_get_ptr (reference getters workspace.hpp:174-178).
 * Default layouts (those the sm_100a kernels use), and with
 * OZA_WS_REFERENCE_LAYOUT the reference's own (workspace.cpp:21-126,
 * pipeline.cu:40-265):                                 reference layout:
 *   OZA_BUF_A_SLICES  int8 [S][Mp][Kp] K-major, padded  int8 [S][M][K]
 *   OZA_BUF_B_SLICES  int8 [S][Np][Kp] (B transposed)   int8 [S][K][N]
 *   OZA_BUF_C_TC      int32[G][Mp][Np] (MATERIALIZE)    Scheme II: int32 [S][M][N];
 *                                                       Scheme I: int32 [M][N], the
 *                                                       last group (g = S + 1), as the
 *                                                       reference's buffer holds it */
#define OZA_BUF_SHIFT_A  0  /* int32[M]                                      */
#define OZA_BUF_SHIFT_B  1  /* int32[N]                                      */
#define OZA_BUF_A_SLICES 2
#define OZA_BUF_B_SLICES 3
#define OZA_BUF_C_TC     4

/* Workspace geometry (padded extents of the buffers above). */
typedef struct oza_ws_info {
    int scheme, slices;
    size_t M, N, K;
    size_t Mp, Np, Kp;     /* padded extents used by the device layouts   */
    int groups;            /* INT32 product planes: S (II); Scheme I one per group g=2..S+1,
                              more where a group is split into several exact INT32 sums
                              (at most (2^31 - 1) / (K 2^(2 beta - 2)) slice pairs each) */
    int k_param;           /* Scheme II: K_param of step 1; Scheme I: 0   */
    int beta;              /* Scheme I: slice width beta; Scheme II: 0    */
    unsigned flags;
    size_t bytes;          /* device bytes held by the workspace          */
} oza_ws_info_t;

/* ---- errors -------------------------------------------------------------- */
/* Thread-local text of the last failure of any entry point on this thread. */
const char* oza_last_error_string(void);

/* ---- executor ------------------------------------------------------------ */
/* Reference: CudaExecutor::CudaExecutor(int), src/core/executor.cpp:61-70. */
oza_status_t oza_executor_create(int device, oza_exec_t* out);
/* Reference: CudaExecutor::~CudaExecutor, executor.cpp:72-76. */
oza_status_t oza_executor_destroy(oza_exec_t ex);
/* Reference: Executor::allocate / free, executor.hpp:19-24 (executor.cpp:78-86). */
oza_status_t oza_executor_alloc(oza_exec_t ex, void** ptr, size_t bytes);
oza_status_t oza_executor_free(oza_exec_t ex, void* ptr);
/* kind: 1 host->device, 2 device->host, 3 device->device.
 * Reference: copy_from_host / copy_to_host / copy_device_to_device, executor.cpp:88-104. */
oza_status_t oza_executor_copy(oza_exec_t ex, void* dst, const void* src, size_t bytes, int kind);
/* Reference: Executor::synchronize, executor.cpp:106-110. */
oza_status_t oza_executor_synchronize(oza_exec_t ex);
/* Extension (no reference counterpart): issue work on a caller cudaStream_t
 * (passed as void*; NULL = legacy default stream). */
oza_status_t oza_executor_set_stream(oza_exec_t ex, void* stream);
oza_status_t oza_executor_device(oza_exec_t ex, int* device);
/* Reference: Executor::get_blas_handle, executor.hpp:35 -- a cuBLAS handle
 * created on first use (the GEMM path itself never calls cuBLAS); NULL if
 * libcublas cannot be loaded. */
void* oza_executor_blas_handle(oza_exec_t ex);

/* ---- workspace ----------------------------------------------------------- */
/* Reference: WorkspaceScheme1/2 constructors, src/core/workspace.cpp:21-47, 65-114.
 * Scheme I requires slices >= 1, Scheme II 1 <= slices <= 20. */
oza_status_t oza_ws_create(oza_exec_t ex, int scheme, size_t M, size_t N, size_t K, int slices,
                           unsigned flags, oza_ws_t* out);
/* Reference: ~WorkspaceScheme1/2, workspace.cpp:49-56, 117-124. */
oza_status_t oza_ws_destroy(oza_ws_t ws);
/* Reference: get_shift_A/B, get_A_slices/get_B_slices, get_C_tc (workspace.hpp:174-178). */
oza_status_t oza_ws_get_ptr(oza_ws_t ws, int which, void** ptr);
oza_status_t oza_ws_get_info(oza_ws_t ws, oza_ws_info_t* info);

/* ---- the GEMM ------------------------------------------------------------ */
/* C = A * B by the workspace's scheme.
 * Reference: ozablas::ozaki_scheme1_gemm / ozaki_scheme2_gemm
 * (include/ozablas/ozablas.hpp:20,31; src/ozablas.cpp:22-74; src/cuda/pipeline.cu:40-265).
 * timings may be NULL (asynchronous call). */
oza_status_t oza_gemm(oza_ws_t ws, const double* A, const double* B, double* C, oza_timings_t* timings);

/* Device error word of the last launch sequence on this workspace: 0 = none,
 * otherwise a bounded wait expired inside a kernel (the call then returned
 * OZA_TIMEOUT). */
oza_status_t oza_ws_device_error(oza_ws_t ws, int* code);

/* ---- allocation-free GEMM ------------------------------------------------- */
/* No counterpart in the reference.  For callers that cannot allocate device
 * memory -- code running while a stream is being captured into a CUDA graph,
 * code inside an application's own allocator or memory-pool callback, paths
 * that cannot afford the synchronisation cudaMalloc/cudaFree may imply --
 * C = A * B by `scheme` with `slices` slices/moduli, with every intermediate
 * in a fixed device array of OZA_NOALLOC_SCRATCH_BYTES that the library holds
 * on each GPU it is loaded on until the process exits.  A, B, C as for
 * oza_gemm (row-major FP64 device buffers on the current device); work is
 * issued on `stream` (NULL = legacy default stream) and the call returns
 * asynchronously.  Problems whose intermediates do not fit in the array are
 * rejected with OZA_UNSUPPORTED and a message giving the bytes needed.  No
 * cudaMalloc/cudaFree or other allocating call is made.  The first call on a
 * device looks up the array's device address and uploads the CRT tables, so
 * make it before any stream capture.  All calls share the one array: calls
 * whose work overlaps on the GPU race; issue them on one stream. */
#define OZA_NOALLOC_SCRATCH_BYTES (64u << 20)
oza_status_t oza_gemm_noalloc(int scheme, int slices, size_t M, size_t N, size_t K, const double* A,
                              const double* B, double* C, void* stream);
/* Device error word of the allocation-free GEMM on the current device: waits
 * for `stream`, then *code = 1 if a bounded device-side wait expired in any
 * oza_gemm_noalloc call since the previous query (its C is then not valid),
 * else 0; the word is cleared.  Allocates nothing.  The array's address is
 * looked up once per device and kept for the process: cudaDeviceReset between
 * calls is not supported.  No counterpart in the reference. */
oza_status_t oza_noalloc_device_error(void* stream, int* code);
/* Self-test of that report, without a GPU fault: one kernel waits, through the
 * GEMM kernels' bounded mbarrier wait, on a barrier nothing arrives on, with
 * the array's error word as its error word; after limit_s (0 < limit_s <= 5)
 * it gives up and sets the word, so the next oza_noalloc_device_error reports
 * 1.  Synchronous on `stream`.  No counterpart in the reference. */
oza_status_t oza_noalloc_selftest_wait_timeout(double limit_s, void* stream);

/* Self-test of failure detection: one kernel waits, through the same bounded
 * mbarrier wait as the GEMM kernels, on a barrier that nothing arrives on.
 * The wait gives up after limit_s (0 < limit_s <= 5) and the kernel returns;
 * *code receives the device error code (1: a wait expired), *elapsed_s
 * (optional) the kernel's device time.  The context stays usable.
 * Extension: the reference has no device-side wait. */
oza_status_t oza_selftest_wait_timeout(oza_exec_t ex, double limit_s, int* code, double* elapsed_s);

/* ---- GEMM tuning ------------------------------------------------------------ */
/* Step-3 kernel configuration of a workspace (0 fields: library defaults).
 *   band         m-tiles (128 rows each) per rasterisation band of the GEMM's
 *                output tiles (default: Scheme II the m-tiles of 32 MiB of one
 *                A plane, at least 16; Scheme I 16)
 *   wait_hint_ns suspend-time hint of the kernel's mbarrier waits (0: poll)
 *   overlap_chunks  Scheme II fused path, calls without timings: >= 2 splits
 *                the GEMM into that many row chunks and overlaps A's slicing
 *                and each chunk's reconstruction with the GEMM on two more
 *                streams; 1: the steps in order; 0: 2 chunks for 8 to 47 row
 *                tiles of 128 when 2 M N K >= 2^33, else 1 (and B's steps 1-2
 *                on a second stream when M K + K N >= 2^26).  Calls with
 *                timings run the steps in order.
 * Results do not depend on the configuration (bit-identical).
 * Extension: the reference's step 3 is cuBLAS with its own heuristics. */
typedef struct {
    int band;
    int wait_hint_ns;
    int overlap_chunks;
} oza_gemm_config_t;

oza_status_t oza_ws_set_gemm_config(oza_ws_t ws, const oza_gemm_config_t* cfg); /* NULL: defaults */
/* Process-wide choice of the Scheme II step-2 residue slicer.  The tensor-core
 * slicer forms the digit products (sum_i d_i (256^i mod m)) with tcgen05 INT8
 * MMAs (S <= 16), the CUDA-core slicer with dp4a.  OZA_SLICER_AUTO (default)
 * takes the tensor cores from S = 12 to 16, where they are as fast or faster,
 * and dp4a below (at S <= 6 the MMA rounds' fixed cost outweighs the dp4a
 * work they save); OZA_SLICER_TENSOR forces the tensor cores for every
 * S <= 16; OZA_SLICER_CUDA_CORES forces dp4a.  The residue planes are
 * identical; the choice only changes speed.  Applies to calls issued
 * afterwards.  Extension: the reference has one CUDA-core slicer
 * (src/pipeline/step2_slicing.hpp:110-206). */
#define OZA_SLICER_AUTO 0
#define OZA_SLICER_CUDA_CORES 1
#define OZA_SLICER_TENSOR 2
oza_status_t oza_set_residue_slicer(int mode);
int oza_get_residue_slicer(void);
oza_status_t oza_ws_get_gemm_config(oza_ws_t ws, oza_gemm_config_t* cfg);
/* Times every configuration on this workspace with these device inputs
 * (step 3 device time, best of 2 after a warm-up), keeps the fastest on the
 * workspace and returns it.  C is overwritten. */
oza_status_t oza_autotune_gemm(oza_ws_t ws, const double* A, const double* B, double* C, oza_gemm_config_t* best,
                               float* best_step3_ms);

/* C = A * B with A, B, C in HOST memory (row-major; pinned for overlap),
 * synchronous.  Scheme II (fused path) and Scheme I: the copies are
 * pipelined with the compute in row chunks of A -- B is copied and sliced
 * while A's chunks arrive, each chunk is sliced, multiplied and
 * reconstructed as it lands, and its rows of C are copied back while the next
 * chunk runs.  Materialised Scheme II and reference-layout workspaces copy
 * in, compute, copy out.  Device staging for A, B and C is
 * allocated in the workspace on the first call.  timings->total_ms is the
 * device time from the first copy to the last; the step fields are 0.
 * Results are bit-identical to oza_gemm.
 * Extension: the reference takes device buffers only (include/ozablas/ozablas.hpp:20,31). */
oza_status_t oza_gemm_host(oza_ws_t ws, const double* A, const double* B, double* C, oza_timings_t* timings);

/* ---- grouped Scheme II GEMM ------------------------------------------------ */
/* Many independent row-major FP64 GEMMs C_i = A_i (M_i x K_i) * B_i (K_i x N_i),
 * each with its own slice count, run as one launch per stage: step 1 and 2
 * over all problems, one persistent tcgen05 GEMM over every problem's work
 * units, one CRT launch (stages 2 and 4 once per distinct slice count).  The
 * sequence is captured into a CUDA graph on the first call and replayed.
 * Results are bit-identical to oza_gemm on each problem alone.
 * Extension: the reference runs one GEMM per call (include/ozablas/ozablas.hpp:31). */
typedef struct oza_group* oza_group_t;

#define OZA_GROUP_NO_GRAPH 0x2u /* launch the stages directly instead of replaying a graph */

typedef struct {
    size_t count;  /* problems */
    size_t units;  /* GEMM work units (problem, m-tile, n-tile, modulus) */
    size_t bytes;  /* device memory held */
    int launches;  /* kernel launches per call */
    int graph;     /* 1 if calls replay a CUDA graph */
} oza_group_info_t;

/* M, N, K, slices: arrays of `count` entries; every dimension >= 1, slices
 * 1..20.  Only Scheme II is grouped (OZA_UNSUPPORTED otherwise). */
oza_status_t oza_group_create(oza_exec_t ex, int scheme, size_t count, const size_t* M, const size_t* N,
                              const size_t* K, const int* slices, unsigned flags, oza_group_t* out);
oza_status_t oza_group_destroy(oza_group_t g);
/* A, B, C: host arrays of `count` device pointers.  Asynchronous on the
 * executor's stream unless timings is non-null (then the stages run without
 * the graph, bracketed by events, and the call synchronises). */
oza_status_t oza_group_gemm(oza_group_t g, const double* const* A, const double* const* B, double* const* C,
                            oza_timings_t* timings);
oza_status_t oza_group_get_info(oza_group_t g, oza_group_info_t* info);
oza_status_t oza_group_device_error(oza_group_t g, int* code);

/* ---- request loop ---------------------------------------------------------- */
/* A server for streams of independent FP64 GEMMs with continuous
 * batching.  Requests are admitted in arrival order while their workspaces fit
 * in a device arena of `workspace_budget` bytes (allocated at creation) and one
 * of `max_inflight` stream slots is free; the Scheme II requests admitted
 * together run as one grouped batch (the oza_group kernels), a Scheme I
 * request as a batch of its own.  Batches on different slots overlap on the
 * device.  Each result is bit-identical to oza_gemm on the same request alone.
 * Extension: the reference has no request loop. */
typedef struct oza_server* oza_server_t;

typedef struct {
    size_t workspace_budget; /* bytes of device memory for request workspaces */
    int max_inflight;        /* batches on the GPU at once (1..16) */
    int max_batch;           /* requests per batch */
} oza_server_config_t;

typedef struct {
    double submit_s, admit_s, done_s; /* host clock, seconds since server creation */
    int slices;
    int batch_size;                   /* requests in the batch that ran it */
    int status;                       /* oza_status_t of the request */
    size_t workspace_bytes;
} oza_request_stats_t;

typedef struct {
    size_t submitted, admitted, completed, queued, batches;
    int max_batch_seen;
    size_t arena_used, arena_peak, workspace_budget;
} oza_server_stats_t;

oza_status_t oza_server_create(oza_exec_t ex, const oza_server_config_t* cfg, oza_server_t* out);
/* Runs every queued request to completion, then frees the server. */
oza_status_t oza_server_destroy(oza_server_t s);
/* Queue C = A * B (row-major device buffers, valid until the request
 * completes) by `scheme` (OZA_SCHEME2: batched with other Scheme II requests;
 * OZA_SCHEME1: run as a batch of its own) with `slices` slices/moduli, e.g.
 * as oza_scheme_for_target chooses them.  OZA_OOM if the request alone
 * exceeds the budget. */
oza_status_t oza_server_submit(oza_server_t s, int scheme, size_t M, size_t N, size_t K, const double* A,
                               const double* B, double* C, int slices, uint64_t* id);
/* Wait for a request (timeout_s < 0: no limit; OZA_TIMEOUT if it expires) and
 * release its record; stats (optional) receives its timestamps. */
oza_status_t oza_server_wait(oza_server_t s, uint64_t id, double timeout_s, oza_request_stats_t* stats);
oza_status_t oza_server_get_stats(oza_server_t s, oza_server_stats_t* out);
/* Workspace bytes one request takes from the arena (0 for invalid sizes). */
size_t oza_server_request_bytes(int scheme, size_t M, size_t N, size_t K, int slices);

/* ---- accuracy tools ------------------------------------------------------- */
/* Maximum relative error of C (M x N, device) against a double-double
 * reference of the same entries, over a seeded sample of `block` rows x `block`
 * columns (relative error falls back to absolute where the reference is 0).
 * Extension: the reference measures accuracy with its FP128 CPU oracle and
 * compute_errors (utils/matrix_reference.hpp:22-50, utils/matrix_compare.hpp:24-65). */
oza_status_t oza_block_error(oza_exec_t ex, const double* A, const double* B, const double* C, size_t M, size_t N,
                             size_t K, int block, unsigned seed, double* max_rel_err);

/* Accuracy-target knob: the smallest slice count (1..20) whose result meets
 * `target_rel_err` on a seeded block sample of this A and B (the pipeline run
 * on the gathered rows and columns reproduces those entries of the full run
 * exactly).  Returns OZA_UNSUPPORTED with slices = 20 if even 20 misses.
 * Extension: the reference leaves the choice of `slices` to the caller
 * (its precision benchmarks sweep it, precision_benchmarks/02_...:146-178). */
oza_status_t oza_autotune_slices(oza_exec_t ex, int scheme, size_t M, size_t N, size_t K, const double* A,
                                 const double* B, double target_rel_err, int block, unsigned seed, int* slices,
                                 double* achieved_err);

/* The accuracy knob's choice of scheme as well: Scheme II (S INT8 GEMMs for
 * S moduli) or Scheme I (S (S + 1) / 2 GEMMs for S slices), whichever meets
 * `target_rel_err` with fewer INT8 GEMMs on two independent seeded block
 * samples (`seed` and a second seed derived from it; the count must meet the
 * target on both; Scheme II at its 20-modulus cap on four more) --
 * Scheme I where Scheme II's 20 moduli miss the target (wide exponent ranges,
 * deep K) or where K exceeds Scheme II's INT32-exact bound.  Returns
 * OZA_UNSUPPORTED, with the scheme whose 20-slice error is lower, if neither
 * reaches it.  Extension: the reference leaves scheme and slices to the caller. */
oza_status_t oza_autotune_scheme(oza_exec_t ex, size_t M, size_t N, size_t K, const double* A, const double* B,
                                 double target_rel_err, int block, unsigned seed, int* scheme, int* slices,
                                 double* achieved_err);

/* As oza_autotune_scheme, with the target given block by block by another
 * result of the same product: C_ref (M x N device, row-major; e.g. native
 * DGEMM's C).  A count is accepted when, on every sampled block, its maximum
 * relative error is at most `factor` times C_ref's on that block (blocks
 * where C_ref is exact count it as one unit roundoff).  *achieved_ratio: the
 * largest sampled error / (factor x C_ref's), <= 1 when met.  Extension: the
 * reference leaves scheme and slices to the caller. */
oza_status_t oza_autotune_scheme_like(oza_exec_t ex, size_t M, size_t N, size_t K, const double* A, const double* B,
                                      const double* C_ref, double factor, int block, unsigned seed, int* scheme,
                                      int* slices, double* achieved_ratio);

/* Slice count for a maximum-relative-error target without running anything:
 * a table measured on B200 (ozablas_b200/calibrate_slices.py) for K = 128 ..
 * 65536 and inputs (U - 0.5) * exp(phi * N(0,1)), phi = 0.5 .. 4, errors over
 * 256 x 256 outputs against a double-double reference; the monotone envelope
 * over K' <= K and phi' <= phi is taken.  Returns 1..20, 21 if 20 slices did
 * not reach the target at the calibrated points, 0 for invalid arguments.
 * Extension: the reference leaves `slices` to the caller. */
int oza_slices_for_target(double target_rel_err, size_t K, double phi);
/* Scheme and slice count for a target without running anything, from the same
 * calibration for both schemes: returns OZA_SCHEME2 or OZA_SCHEME1 (the one
 * reaching the target with fewer INT8 GEMMs; Scheme II on a tie), *slices its
 * count; Scheme I with *slices = 21 if neither reaches the target with 20.
 * 0 for invalid arguments.  Extension: the reference leaves the choice to the
 * caller. */
int oza_scheme_for_target(double target_rel_err, size_t K, double phi, int* slices);

/* Estimate of phi, the exponent spread the two lookups above take, from the
 * data: on `block` sampled rows of A and columns of B (device, row-major),
 * the variance of ln|x| about each row's and column's own mean, pooled over
 * nonzero finite entries, is 1 + phi^2 for (U - 0.5) exp(phi N(0,1)) inputs
 * (the family the tables were calibrated on).  Row and column scaling, which
 * the step-1 shifts absorb, does not change it.  Extension. */
oza_status_t oza_estimate_phi(oza_exec_t ex, size_t M, size_t N, size_t K, const double* A, const double* B,
                              int block, unsigned seed, double* phi);

/* ---- host utilities ------------------------------------------------------- */
/* Seeded test matrix (U - 0.5) * exp(phi * N(0,1)) with U in (0,1], drawn from
 * std::mt19937(seed) in row-major order.
 * Reference: matrix_utils::generation::generate_ozaki_matrix, utils/matrix_gen.hpp:15-34. */
oza_status_t oza_generate_matrix(int rows, int cols, double phi, int seed, double* out);

/* Scheme parameters computed on the host.
 * Reference: calculate_scheme1_beta / calculate_scheme2_k_param,
 * src/pipeline/step1_statistics.hpp:12-20 (K_param with M as in pipeline.cu:196-198). */
int oza_scheme1_beta(size_t K);
int oza_scheme2_k_param(int slices, size_t K);

/* Library version string. */
const char* oza_version(void);

#ifdef __cplusplus
}
#endif

#endif /* OZA_CAPI_H */
