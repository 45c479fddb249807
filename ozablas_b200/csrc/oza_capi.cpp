// oza_capi.cpp -- host side of the C ABI declared in include/oza_capi.h:
// executor (device, stream, allocations), workspaces (padded device layouts)
// and the stage orchestration of Scheme I / Scheme II.
//
// Orchestration follows the reference's four steps (src/cuda/pipeline.cu:40-265)
// with its observable contract: per-step OzaTimings measured with CUDA events,
// asynchronous unless timings are requested, C fully overwritten.
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <random>
#include <string>
#include <vector>

#include "oza_capi.h"
#include "oza_internal.h"
#include "oza_kernels.h"

using oza::DeviceGuard;

namespace {

thread_local std::string g_last_error;

oza_status_t fail(oza_status_t st, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return st;
}

oza_status_t cuda_fail(cudaError_t e, const char* what) {
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return fail(OZA_OOM, "%s: %s", what, cudaGetErrorString(e));
    }
    return fail(OZA_CUDA_ERROR, "%s: %s", what, cudaGetErrorString(e));
}

#define OZA_CUDA_TRY(call, what)                   \
    do {                                           \
        cudaError_t e__ = (call);                  \
        if (e__ != cudaSuccess) return cuda_fail(e__, what); \
    } while (0)

}  // namespace

void oza::set_last_error(const char* msg) { g_last_error = msg ? msg : ""; }

oza_status_t oza::check_problem(const char* who, int scheme, size_t M, size_t N, size_t K, int slices) {
    if (scheme != OZA_SCHEME1 && scheme != OZA_SCHEME2) return fail(OZA_INVALID_ARG, "%s: unknown scheme %d", who, scheme);
    // Messages of the reference's workspace constructors (src/core/workspace.cpp:24-25, 68-71).
    if (scheme == OZA_SCHEME1 && slices < 1) return fail(OZA_INVALID_ARG, "OzaBLAS: Slices must be >= 1.");
    if (scheme == OZA_SCHEME2 && (slices < 1 || slices > 20))
        return fail(OZA_INVALID_ARG, "OzaBLAS: Scheme II supports between 1 and 20 slices.");
    if (scheme == OZA_SCHEME1 && slices > 20)
        return fail(OZA_UNSUPPORTED, "OzaBLAS: Scheme I is built for at most 20 slices (got %d)", slices);
    const size_t Mp = oza::round_up(M, oza::kTileM), Np = oza::round_up(N, oza::kTileN);
    const size_t Kp = oza::round_up(K, oza::kTileK);
    if ((double)slices * (double)Mp >= 2147483648.0 || (double)slices * (double)Np >= 2147483648.0 ||
        Kp >= (1ull << 31))
        return fail(OZA_UNSUPPORTED, "OzaBLAS: problem too large for one workspace (M=%zu N=%zu K=%zu S=%d)", M, N, K,
                    slices);
    if (scheme == OZA_SCHEME2 && (double)K * 125.0 * 125.0 >= 2147483648.0)
        return fail(OZA_UNSUPPORTED, "OzaBLAS: K=%zu exceeds the INT32-exact bound of Scheme II (K <= 137438)", K);
    return OZA_OK;
}


struct oza_workspace {
    oza_executor* ex = nullptr;
    int scheme = 0, S = 0;
    size_t M = 0, N = 0, K = 0, Mp = 0, Np = 0, Kp = 0;
    int groups = 0, k_param = 0, beta = 0;
    unsigned flags = 0;
    size_t bytes = 0;
    int32_t* shiftA = nullptr;
    int32_t* shiftB = nullptr;
    unsigned long long* colmax = nullptr;
    int8_t* aplanes = nullptr;
    int8_t* bplanes = nullptr;
    int32_t* ctc = nullptr;          // INT32 group planes (materialised / Scheme I)
    uint8_t* coef = nullptr;         // Scheme II CRT coefficient bytes [S][Mp][Np]
    // OZA_WS_REFERENCE_LAYOUT: the intermediates in the reference's layouts
    int8_t* a_ref = nullptr;         // [S][M][K]
    int8_t* b_ref = nullptr;         // [S][K][N]
    int32_t* c_ref = nullptr;        // Scheme II [S][M][N]; Scheme I [M][N] (last group)
    bool fused = false;
    int* err = nullptr;
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    oza::PairList pairs{};
    oza_gemm_config_t cfg{0, 0, 0};  // GEMM tuning (0: library defaults)
    // oza_gemm_host: device staging of A, B, C, copy streams and chunk events,
    // made on first use.
    struct HostPipe {
        double* dA = nullptr;
        double* dB = nullptr;
        double* dC = nullptr;
        cudaStream_t cin = nullptr, cout = nullptr;
        cudaEvent_t t0 = nullptr, t1 = nullptr, b_in = nullptr, out_done = nullptr;
        static constexpr int kMaxChunks = 32;
        cudaEvent_t a_in[kMaxChunks] = {}, done[kMaxChunks] = {};
    } hp;
    // Overlapped device path: slicer and reconstruction streams, chunk events.
    struct Overlap {
        static constexpr int kMaxChunks = 16;
        cudaStream_t s_slice = nullptr, s_crt = nullptr;
        cudaEvent_t start = nullptr, end = nullptr;
        cudaEvent_t a_done[kMaxChunks] = {}, g_done[kMaxChunks] = {};
    } ov;
};

namespace {


void overlap_release(oza_workspace* ws);

void ws_release(oza_workspace* ws) {
    overlap_release(ws);
    auto& h = ws->hp;
    if (h.cin) cudaStreamSynchronize(h.cin);
    if (h.cout) cudaStreamSynchronize(h.cout);
    void* bufs[] = {ws->shiftA, ws->shiftB, ws->colmax, ws->aplanes, ws->bplanes, ws->ctc, ws->coef, ws->err,
                    ws->a_ref, ws->b_ref, ws->c_ref, h.dA, h.dB, h.dC};
    for (void* p : bufs)
        if (p) cudaFree(p);
    for (auto& e : ws->ev)
        if (e) cudaEventDestroy(e);
    cudaEvent_t evs[] = {h.t0, h.t1, h.b_in, h.out_done};
    for (cudaEvent_t e : evs)
        if (e) cudaEventDestroy(e);
    for (int i = 0; i < oza_workspace::HostPipe::kMaxChunks; ++i) {
        if (h.a_in[i]) cudaEventDestroy(h.a_in[i]);
        if (h.done[i]) cudaEventDestroy(h.done[i]);
    }
    if (h.cin) cudaStreamDestroy(h.cin);
    if (h.cout) cudaStreamDestroy(h.cout);
}


void overlap_release(oza_workspace* ws) {
    auto& o = ws->ov;
    if (o.s_slice) cudaStreamSynchronize(o.s_slice);
    if (o.s_crt) cudaStreamSynchronize(o.s_crt);
    cudaEvent_t evs[] = {o.start, o.end};
    for (cudaEvent_t e : evs)
        if (e) cudaEventDestroy(e);
    for (int i = 0; i < oza_workspace::Overlap::kMaxChunks; ++i) {
        if (o.a_done[i]) cudaEventDestroy(o.a_done[i]);
        if (o.g_done[i]) cudaEventDestroy(o.g_done[i]);
    }
    if (o.s_slice) cudaStreamDestroy(o.s_slice);
    if (o.s_crt) cudaStreamDestroy(o.s_crt);
}

// The second stream and its two events (the two-stream steps 1-2), and with
// `chunks` > 0 the reconstruction stream and the events of that many row
// chunks: each object made on first use and kept with the workspace.
cudaError_t overlap_init(oza_workspace* ws, int chunks) {
    auto& o = ws->ov;
    cudaError_t e = cudaSuccess;
    if (!o.s_slice) e = cudaStreamCreateWithFlags(&o.s_slice, cudaStreamNonBlocking);
    if (e == cudaSuccess && !o.start) e = cudaEventCreateWithFlags(&o.start, cudaEventDisableTiming);
    if (e == cudaSuccess && !o.end) e = cudaEventCreateWithFlags(&o.end, cudaEventDisableTiming);
    if (chunks > 0) {
        if (e == cudaSuccess && !o.s_crt) e = cudaStreamCreateWithFlags(&o.s_crt, cudaStreamNonBlocking);
        const int n = std::min(chunks, (int)oza_workspace::Overlap::kMaxChunks);
        for (int i = 0; i < n && e == cudaSuccess; ++i) {
            if (!o.a_done[i]) e = cudaEventCreateWithFlags(&o.a_done[i], cudaEventDisableTiming);
            if (e == cudaSuccess && !o.g_done[i]) e = cudaEventCreateWithFlags(&o.g_done[i], cudaEventDisableTiming);
        }
    }
    return e;
}

// Scheme II fused path with the stages overlapped across streams, always on
// the one-CTA GEMM kernel: B is sliced on the executor's stream while A's row
// chunks are sliced on a second stream; the GEMM runs chunk by chunk on the
// executor's stream; each chunk's CRT runs on a third stream while the next
// chunk's GEMM runs.  Same kernels, same results as the sequential steps.
oza_status_t gemm_overlapped(oza_workspace* ws, const double* A, const double* B, double* C, int chunks) {
    oza_executor* ex = ws->ex;
    auto& o = ws->ov;
    cudaStream_t st = ex->stream;
    const size_t M = ws->M, N = ws->N, K = ws->K;
    const int offset = ws->k_param;
    const size_t tile_m = oza::kTileM;
    const int mt_all = (int)((M + tile_m - 1) / tile_m);
    const int R0 = std::min(std::min(chunks, (int)oza_workspace::Overlap::kMaxChunks), mt_all);
    const int q = (mt_all + R0 - 1) / R0;
    const int R = (mt_all + q - 1) / q;
    OZA_CUDA_TRY(cudaEventRecord(o.start, st), "CUDA: event record");
    OZA_CUDA_TRY(cudaStreamWaitEvent(o.s_slice, o.start, 0), "CUDA: stream wait");
    OZA_CUDA_TRY(cudaStreamWaitEvent(o.s_crt, o.start, 0), "CUDA: stream wait");
    OZA_CUDA_TRY(oza::launch_stats_cols(B, K, N, ws->colmax, ex->sms, st), "step1 cols");
    OZA_CUDA_TRY(oza::launch_slice_cols(ws->scheme, B, K, N, ws->colmax, offset, ws->S, ws->beta, ws->shiftB,
                                        ws->bplanes, ws->Np, ws->Kp, st, ws->err),
                 "step2 cols");
    for (int c = 0; c < R; ++c) {
        const size_t r0 = (size_t)c * q * tile_m;
        const size_t rows_p = std::min((size_t)q * tile_m, (size_t)mt_all * tile_m - r0);
        const size_t rows = std::min(M, r0 + rows_p) - r0;
        OZA_CUDA_TRY(oza::launch_stats_rows(A + r0 * K, rows, K, offset, ws->shiftA + r0, ex->sms, o.s_slice),
                     "step1 rows");
        OZA_CUDA_TRY(oza::launch_slice_rows(ws->scheme, A + r0 * K, rows, K, ws->shiftA + r0, ws->S, ws->beta, offset,
                                            ws->aplanes + r0 * ws->Kp, rows_p, ws->Kp, ex->sms, o.s_slice, ws->Mp,
                                            ws->err),
                     "step2 rows");
        OZA_CUDA_TRY(cudaEventRecord(o.a_done[c], o.s_slice), "CUDA: event record");
    }
    for (int c = 0; c < R; ++c) {
        const size_t r0 = (size_t)c * q * tile_m;
        const size_t rows_p = std::min((size_t)q * tile_m, (size_t)mt_all * tile_m - r0);
        const size_t rows = std::min(M, r0 + rows_p) - r0;
        OZA_CUDA_TRY(cudaStreamWaitEvent(st, o.a_done[c], 0), "CUDA: stream wait");
        oza::GemmPlan plan;
        plan.a_planes = ws->aplanes;
        plan.b_planes = ws->bplanes;
        plan.planes = ws->S;
        plan.Mp = ws->Mp;
        plan.Np = ws->Np;
        plan.Kp = ws->Kp;
        plan.M = ws->M;
        plan.N = ws->N;
        plan.pairs = ws->pairs;
        plan.err = ws->err;
        plan.sms = ex->sms;
        plan.ctc = nullptr;
        plan.coef = ws->coef;
        plan.m_tile_begin = c * q;
        plan.m_tile_count = std::min(q, mt_all - c * q);
        plan.band = ws->cfg.band;
        plan.wait_hint_ns = (uint32_t)ws->cfg.wait_hint_ns;
        OZA_CUDA_TRY(oza::launch_gemm_i8(plan, st), "step3 gemm");
        OZA_CUDA_TRY(cudaEventRecord(o.g_done[c], st), "CUDA: event record");
        OZA_CUDA_TRY(cudaStreamWaitEvent(o.s_crt, o.g_done[c], 0), "CUDA: stream wait");
        OZA_CUDA_TRY(oza::launch_crt_coef(ws->coef + r0 * ws->Np, ws->Mp, ws->Np, rows, N, ws->S, ws->shiftA + r0,
                                          ws->shiftB, C + r0 * N, ex->sms, o.s_crt),
                     "step4 crt");
    }
    OZA_CUDA_TRY(cudaEventRecord(o.end, o.s_crt), "CUDA: event record");
    OZA_CUDA_TRY(cudaStreamWaitEvent(st, o.end, 0), "CUDA: stream wait");
    return OZA_OK;
}

cudaError_t host_pipe_init(oza_workspace* ws) {
    auto& h = ws->hp;
    if (h.dC) return cudaSuccess;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&h.dA), ws->M * ws->K * sizeof(double) + 16);
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&h.dB), ws->K * ws->N * sizeof(double) + 16);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h.cin, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h.cout, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&h.t0);
    if (e == cudaSuccess) e = cudaEventCreate(&h.t1);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h.b_in, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h.out_done, cudaEventDisableTiming);
    for (int i = 0; i < oza_workspace::HostPipe::kMaxChunks && e == cudaSuccess; ++i) {
        e = cudaEventCreateWithFlags(&h.a_in[i], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h.done[i], cudaEventDisableTiming);
    }
    // dC last: its presence marks a complete set-up.
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&h.dC), ws->M * ws->N * sizeof(double) + 16);
    return e;
}

}  // namespace

extern "C" {

const char* oza_last_error_string(void) { return g_last_error.c_str(); }

const char* oza_version(void) { return "ozablas_b200 0.1 (sm_100a)"; }

// ---------------------------------------------------------------- executor
oza_status_t oza_executor_create(int device, oza_exec_t* out) {
    if (!out) return fail(OZA_INVALID_ARG, "oza_executor_create: null output handle");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess) return cuda_fail(e, "CUDA: no usable device");
    if (device < 0 || device >= count) return fail(OZA_INVALID_ARG, "CUDA: device %d out of range (%d)", device, count);
    OZA_CUDA_TRY(cudaSetDevice(device), "CUDA: Failed to set device");
    int major = 0, minor = 0, sms = 0;
    OZA_CUDA_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device), "CUDA: attribute");
    OZA_CUDA_TRY(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device), "CUDA: attribute");
    OZA_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "CUDA: attribute");
    if (major != 10 || minor != 0)
        return fail(OZA_UNSUPPORTED, "device %d is sm_%d%d; this build targets sm_100a (B200) only", device, major,
                    minor);
    auto* ex = new (std::nothrow) oza_executor();
    if (!ex) return fail(OZA_OOM, "oza_executor_create: host allocation failed");
    ex->device = device;
    ex->sms = sms;
    *out = ex;
    return OZA_OK;
}

oza_status_t oza_executor_destroy(oza_exec_t ex) {
    if (!ex) return OZA_OK;
    if (ex->blas) {
        void* lib = dlopen("libcublas.so.12", RTLD_NOW | RTLD_NOLOAD);
        if (lib) {
            auto destroy = reinterpret_cast<int (*)(void*)>(dlsym(lib, "cublasDestroy_v2"));
            if (destroy) destroy(ex->blas);
        }
    }
    delete ex;
    return OZA_OK;
}

oza_status_t oza_executor_alloc(oza_exec_t ex, void** ptr, size_t bytes) {
    if (!ex || !ptr) return fail(OZA_INVALID_ARG, "oza_executor_alloc: null argument");
    DeviceGuard g(ex->device);
    *ptr = nullptr;
    cudaError_t e = cudaMalloc(ptr, bytes ? bytes : 1);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(OZA_OOM, "CUDA: allocation of %zu bytes failed (%s)", bytes, cudaGetErrorString(e));
    }
    return OZA_OK;
}

oza_status_t oza_executor_free(oza_exec_t ex, void* ptr) {
    if (!ex) return fail(OZA_INVALID_ARG, "oza_executor_free: null executor");
    if (!ptr) return OZA_OK;
    DeviceGuard g(ex->device);
    OZA_CUDA_TRY(cudaFree(ptr), "CUDA: free failed");
    return OZA_OK;
}

oza_status_t oza_executor_copy(oza_exec_t ex, void* dst, const void* src, size_t bytes, int kind) {
    if (!ex || (!dst && bytes) || (!src && bytes)) return fail(OZA_INVALID_ARG, "oza_executor_copy: null argument");
    cudaMemcpyKind k;
    const char* what;
    switch (kind) {
        case 1: k = cudaMemcpyHostToDevice; what = "CUDA: Memcpy HostToDevice failed"; break;
        case 2: k = cudaMemcpyDeviceToHost; what = "CUDA: Memcpy DeviceToHost failed"; break;
        case 3: k = cudaMemcpyDeviceToDevice; what = "CUDA: Memcpy DeviceToDevice failed"; break;
        default: return fail(OZA_INVALID_ARG, "oza_executor_copy: kind %d", kind);
    }
    if (!bytes) return OZA_OK;
    DeviceGuard g(ex->device);
    OZA_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, k, ex->stream), what);
    OZA_CUDA_TRY(cudaStreamSynchronize(ex->stream), what);
    return OZA_OK;
}

oza_status_t oza_executor_synchronize(oza_exec_t ex) {
    if (!ex) return fail(OZA_INVALID_ARG, "oza_executor_synchronize: null executor");
    DeviceGuard g(ex->device);
    OZA_CUDA_TRY(cudaDeviceSynchronize(), "CUDA: Device synchronize failed");
    return OZA_OK;
}

oza_status_t oza_executor_set_stream(oza_exec_t ex, void* stream) {
    if (!ex) return fail(OZA_INVALID_ARG, "oza_executor_set_stream: null executor");
    ex->stream = static_cast<cudaStream_t>(stream);
    return OZA_OK;
}

oza_status_t oza_executor_device(oza_exec_t ex, int* device) {
    if (!ex || !device) return fail(OZA_INVALID_ARG, "oza_executor_device: null argument");
    *device = ex->device;
    return OZA_OK;
}

void* oza_executor_blas_handle(oza_exec_t ex) {
    if (!ex) return nullptr;
    std::lock_guard<std::mutex> lk(ex->blas_mu);
    if (ex->blas) return ex->blas;
    void* lib = dlopen("libcublas.so.12", RTLD_NOW | RTLD_GLOBAL);
    if (!lib) return nullptr;
    auto create = reinterpret_cast<int (*)(void**)>(dlsym(lib, "cublasCreate_v2"));
    if (!create) return nullptr;
    DeviceGuard g(ex->device);
    void* h = nullptr;
    if (create(&h) != 0) return nullptr;
    ex->blas = h;
    return h;
}

// ---------------------------------------------------------------- workspace
oza_status_t oza_ws_create(oza_exec_t ex, int scheme, size_t M, size_t N, size_t K, int slices, unsigned flags,
                           oza_ws_t* out) {
    if (!out) return fail(OZA_INVALID_ARG, "oza_ws_create: null output handle");
    *out = nullptr;
    if (!ex) return fail(OZA_INVALID_ARG, "OzaBLAS: Executor cannot be null.");
    if (flags & ~(OZA_WS_MATERIALIZE | OZA_WS_REFERENCE_LAYOUT))
        return fail(OZA_INVALID_ARG, "oza_ws_create: unknown flags 0x%x", flags);
    if (flags & OZA_WS_REFERENCE_LAYOUT) flags |= OZA_WS_MATERIALIZE;
    {
        const oza_status_t chk = oza::check_problem("oza_ws_create", scheme, M, N, K, slices);
        if (chk != OZA_OK) return chk;
    }

    auto* ws = new (std::nothrow) oza_workspace();
    if (!ws) return fail(OZA_OOM, "oza_ws_create: host allocation failed");
    ws->ex = ex;
    ws->scheme = scheme;
    ws->S = slices;
    ws->M = M;
    ws->N = N;
    ws->K = K;
    ws->Mp = oza::round_up(M, oza::kTileM);
    ws->Np = oza::round_up(N, oza::kTileN);
    ws->Kp = oza::round_up(K, oza::kTileK);
    ws->flags = flags;
    ws->pairs = oza::make_pairs(scheme, slices, K);
    ws->groups = ws->pairs.num_groups;   // INT32 planes: Scheme I groups may split at large K
    if (scheme == OZA_SCHEME2) ws->k_param = K ? oza_scheme2_k_param(slices, K) : 0;
    else ws->beta = K ? oza_scheme1_beta(K) : 1;

    DeviceGuard g(ex->device);
    cudaError_t e = oza::upload_tables();
    if (e != cudaSuccess) {
        delete ws;
        return cuda_fail(e, "CUDA: constant table upload failed");
    }
    // Scheme II without MATERIALIZE reduces the INT32 residue products to their
    // one-byte CRT coefficients inside the GEMM epilogue: byte planes replace
    // the INT32 planes (a quarter of the memory and traffic).
    ws->fused = (scheme == OZA_SCHEME2) && !(flags & OZA_WS_MATERIALIZE);
    const size_t ctc_bytes = ws->fused ? 0 : (size_t)ws->groups * ws->Mp * ws->Np * sizeof(int32_t) + 16;
    const size_t coef_bytes = ws->fused ? (size_t)slices * ws->Mp * ws->Np + 16 : 0;
    const bool ref_layout = (flags & OZA_WS_REFERENCE_LAYOUT) != 0;
    const size_t S_ = (size_t)slices;
    const size_t ref_c_planes = scheme == OZA_SCHEME2 ? S_ : 1;
    struct Req {
        void** p;
        size_t bytes;
    } reqs[] = {
        {(void**)&ws->shiftA, (M ? M : 1) * sizeof(int32_t)},
        {(void**)&ws->shiftB, (N ? N : 1) * sizeof(int32_t)},
        {(void**)&ws->colmax, (N ? N : 1) * sizeof(unsigned long long)},
        {(void**)&ws->aplanes, (size_t)slices * ws->Mp * ws->Kp + 16},
        {(void**)&ws->bplanes, (size_t)slices * ws->Np * ws->Kp + 16},
        {(void**)&ws->ctc, ctc_bytes},
        {(void**)&ws->coef, coef_bytes},
        {(void**)&ws->err, sizeof(int)},
        {(void**)&ws->a_ref, ref_layout ? S_ * M * K + 16 : 0},
        {(void**)&ws->b_ref, ref_layout ? S_ * K * N + 16 : 0},
        {(void**)&ws->c_ref, ref_layout ? ref_c_planes * M * N * sizeof(int32_t) + 16 : 0},
    };
    for (auto& r : reqs) {
        if (r.bytes == 0) continue;
        e = cudaMalloc(r.p, r.bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            ws_release(ws);
            delete ws;
            return fail(OZA_OOM, "OzaBLAS: workspace allocation of %zu bytes failed", r.bytes);
        }
        ws->bytes += r.bytes;
    }
    e = cudaMemset(ws->err, 0, sizeof(int));
    for (auto& ev : ws->ev)
        if (e == cudaSuccess) e = cudaEventCreate(&ev);
    if (e != cudaSuccess) {
        ws_release(ws);
        delete ws;
        return cuda_fail(e, "CUDA: workspace setup failed");
    }
    *out = ws;
    return OZA_OK;
}

oza_status_t oza_ws_destroy(oza_ws_t ws) {
    if (!ws) return OZA_OK;
    DeviceGuard g(ws->ex->device);
    ws_release(ws);
    delete ws;
    return OZA_OK;
}

oza_status_t oza_ws_get_ptr(oza_ws_t ws, int which, void** ptr) {
    if (!ws || !ptr) return fail(OZA_INVALID_ARG, "oza_ws_get_ptr: null argument");
    switch (which) {
        case OZA_BUF_SHIFT_A: *ptr = ws->shiftA; break;
        case OZA_BUF_SHIFT_B: *ptr = ws->shiftB; break;
        case OZA_BUF_A_SLICES: *ptr = ws->a_ref ? (void*)ws->a_ref : (void*)ws->aplanes; break;
        case OZA_BUF_B_SLICES: *ptr = ws->b_ref ? (void*)ws->b_ref : (void*)ws->bplanes; break;
        case OZA_BUF_C_TC: *ptr = ws->c_ref ? (void*)ws->c_ref : (void*)ws->ctc; break;
        default: return fail(OZA_INVALID_ARG, "oza_ws_get_ptr: unknown buffer %d", which);
    }
    return OZA_OK;
}

oza_status_t oza_ws_get_info(oza_ws_t ws, oza_ws_info_t* info) {
    if (!ws || !info) return fail(OZA_INVALID_ARG, "oza_ws_get_info: null argument");
    info->scheme = ws->scheme;
    info->slices = ws->S;
    info->M = ws->M;
    info->N = ws->N;
    info->K = ws->K;
    info->Mp = ws->Mp;
    info->Np = ws->Np;
    info->Kp = ws->Kp;
    info->groups = ws->groups;
    info->k_param = ws->k_param;
    info->beta = ws->beta;
    info->flags = ws->flags;
    info->bytes = ws->bytes;
    return OZA_OK;
}

oza_status_t oza_ws_device_error(oza_ws_t ws, int* code) {
    if (!ws || !code) return fail(OZA_INVALID_ARG, "oza_ws_device_error: null argument");
    DeviceGuard g(ws->ex->device);
    OZA_CUDA_TRY(cudaStreamSynchronize(ws->ex->stream), "CUDA: synchronize failed");
    OZA_CUDA_TRY(cudaMemcpy(code, ws->err, sizeof(int), cudaMemcpyDeviceToHost), "CUDA: error word read failed");
    return OZA_OK;
}

// ---------------------------------------------------------------- GEMM
oza_status_t oza_gemm(oza_ws_t ws, const double* A, const double* B, double* C, oza_timings_t* timings) {
    if (!ws) return fail(OZA_INVALID_ARG, "oza_gemm: null workspace");
    if (ws->M == 0 || ws->N == 0) {
        if (timings) std::memset(timings, 0, sizeof(*timings));
        return OZA_OK;
    }
    if (!C || (ws->K && (!A || !B))) return fail(OZA_INVALID_ARG, "oza_gemm: null matrix pointer");
    oza_executor* ex = ws->ex;
    DeviceGuard g(ex->device);
    if (!g.ok) return fail(OZA_CUDA_ERROR, "CUDA: Failed to set device %d", ex->device);
    cudaStream_t st = ex->stream;
    const size_t M = ws->M, N = ws->N, K = ws->K;

    if (!timings && K && ws->fused) {
        // Overlapped stages on the one-CTA kernel, by default in 2 row chunks
        // for 8..47 row tiles: +6% at 2048^3, +3.7% at 1024x1024x65536, +1.7%
        // at 4096^3 over the steps in order.  From 48 tiles the GEMM dominates
        // and a single full launch is faster per clock than chunk launches
        // sharing the SMs with the slicer: at 8192^3 the steps in order run at
        // 132.5 TFLOP/s against 127-129 with 2 to 4 chunks.  Below 2^33 FP64
        // flops (2 M N K) the extra streams' synchronisation costs more than
        // the overlap gains: the steps in order.
        int chunks = ws->cfg.overlap_chunks;
        if (chunks == 0) {
            const size_t tiles = (M + oza::kTileM - 1) / oza::kTileM;
            const double flops = 2.0 * (double)M * (double)N * (double)K;
            chunks = (tiles >= 8 && tiles < 48 && flops >= 0x1p33) ? 2 : 1;
        }
        if (chunks >= 2) {
            OZA_CUDA_TRY(overlap_init(ws, chunks), "oza_gemm: overlap streams");
            return gemm_overlapped(ws, A, B, C, chunks);
        }
    }
    // Untimed calls with the default configuration run B's statistics and
    // slicer on a second stream beside A's: the HBM-bound statistics of one
    // operand overlap the issue-bound slicer of the other.  The GEMM waits
    // for both.  Only where steps 1-2 are long enough to pay for the second
    // stream's synchronisation: M K + K N of at least 2^26 elements (8192^3:
    // -2.1% per call); smaller calls, and calls with timings, keep the four
    // steps in order.
    const bool dual = !timings && K && ws->cfg.overlap_chunks == 0 &&
                      (double)M * (double)K + (double)K * (double)N >= 0x1p26;
    cudaStream_t sb = st;
    if (dual) {
        OZA_CUDA_TRY(overlap_init(ws, 0), "oza_gemm: second stream");
        sb = ws->ov.s_slice;
        OZA_CUDA_TRY(cudaEventRecord(ws->ov.start, st), "CUDA: event record");
        OZA_CUDA_TRY(cudaStreamWaitEvent(sb, ws->ov.start, 0), "CUDA: stream wait");
    }
    if (timings) OZA_CUDA_TRY(cudaEventRecord(ws->ev[0], st), "CUDA: event record");
    if (K == 0) {
        // Empty inner dimension: the product is exactly zero.
        OZA_CUDA_TRY(cudaMemsetAsync(C, 0, M * N * sizeof(double), st), "CUDA: memset");
        for (int i = 1; i < 5 && timings; ++i) OZA_CUDA_TRY(cudaEventRecord(ws->ev[i], st), "CUDA: event record");
    } else {
        const int offset = ws->scheme == OZA_SCHEME2 ? ws->k_param : 0;
        // step 1
        OZA_CUDA_TRY(oza::launch_stats_rows(A, M, K, offset, ws->shiftA, ex->sms, st), "step1 rows");
        OZA_CUDA_TRY(oza::launch_stats_cols(B, K, N, ws->colmax, ex->sms, sb), "step1 cols");
        if (timings) OZA_CUDA_TRY(cudaEventRecord(ws->ev[1], st), "CUDA: event record");
        // step 2
        OZA_CUDA_TRY(oza::launch_slice_rows(ws->scheme, A, M, K, ws->shiftA, ws->S, ws->beta, offset, ws->aplanes, ws->Mp,
                                            ws->Kp, ex->sms, st, 0, ws->err),
                     "step2 rows");
        OZA_CUDA_TRY(oza::launch_slice_cols(ws->scheme, B, K, N, ws->colmax, offset, ws->S, ws->beta, ws->shiftB,
                                            ws->bplanes, ws->Np, ws->Kp, sb, ws->err),
                     "step2 cols");
        if (dual) {
            OZA_CUDA_TRY(cudaEventRecord(ws->ov.end, sb), "CUDA: event record");
            OZA_CUDA_TRY(cudaStreamWaitEvent(st, ws->ov.end, 0), "CUDA: stream wait");
        }
        if (timings) OZA_CUDA_TRY(cudaEventRecord(ws->ev[2], st), "CUDA: event record");
        // step 3
        oza::GemmPlan plan;
        plan.a_planes = ws->aplanes;
        plan.b_planes = ws->bplanes;
        plan.planes = ws->S;
        plan.Mp = ws->Mp;
        plan.Np = ws->Np;
        plan.Kp = ws->Kp;
        plan.M = ws->M;
        plan.N = ws->N;
        plan.pairs = ws->pairs;
        plan.err = ws->err;
        plan.sms = ex->sms;
        plan.ctc = ws->ctc;
        plan.coef = ws->fused ? ws->coef : nullptr;
        plan.band = ws->cfg.band;
        plan.wait_hint_ns = (uint32_t)ws->cfg.wait_hint_ns;
        OZA_CUDA_TRY(oza::launch_gemm_i8(plan, st), "step3 gemm");
        if (timings) OZA_CUDA_TRY(cudaEventRecord(ws->ev[3], st), "CUDA: event record");
        // step 4
        if (ws->fused) {
            OZA_CUDA_TRY(oza::launch_crt_coef(ws->coef, ws->Mp, ws->Np, M, N, ws->S, ws->shiftA, ws->shiftB, C,
                                              ex->sms, st),
                         "step4 crt");
        } else if (ws->scheme == OZA_SCHEME2) {
            OZA_CUDA_TRY(oza::launch_reconstruct2(ws->ctc, ws->Mp, ws->Np, M, N, ws->S, ws->shiftA, ws->shiftB, C, st),
                         "step4 crt");
        } else {
            OZA_CUDA_TRY(oza::launch_reconstruct1(ws->ctc, ws->Mp, ws->Np, M, N, ws->S, ws->beta, ws->shiftA,
                                                  ws->shiftB, C, ex->sms, st, &ws->pairs),
                         "step4 sum");
        }
        if (timings) OZA_CUDA_TRY(cudaEventRecord(ws->ev[4], st), "CUDA: event record");
        if (ws->a_ref) {
            // OZA_WS_REFERENCE_LAYOUT: the reference's buffers, outside the timed steps.
            // Scheme I: the last group (its planes summed where it was split)
            const bool s2 = ws->scheme == OZA_SCHEME2;
            const int c_first = s2 ? 0 : ws->pairs.first_unit[ws->S - 1];
            const int c_count = s2 ? ws->groups : ws->groups - c_first;
            OZA_CUDA_TRY(oza::launch_to_reference_layout(ws->aplanes, ws->bplanes, ws->ctc, ws->S, ws->groups, M, N,
                                                         K, ws->Mp, ws->Np, ws->Kp, ws->a_ref, ws->b_ref, ws->c_ref,
                                                         c_first, c_count, !s2, st),
                         "reference-layout copies");
        }
    }
    if (timings) {
        OZA_CUDA_TRY(cudaEventSynchronize(ws->ev[4]), "CUDA: event synchronize");
        if (ws->a_ref) OZA_CUDA_TRY(cudaStreamSynchronize(st), "CUDA: stream synchronize");
        cudaEventElapsedTime(&timings->step1_ms, ws->ev[0], ws->ev[1]);
        cudaEventElapsedTime(&timings->step2_ms, ws->ev[1], ws->ev[2]);
        cudaEventElapsedTime(&timings->step3_ms, ws->ev[2], ws->ev[3]);
        cudaEventElapsedTime(&timings->step4_ms, ws->ev[3], ws->ev[4]);
        cudaEventElapsedTime(&timings->total_ms, ws->ev[0], ws->ev[4]);
        int code = 0;
        OZA_CUDA_TRY(cudaMemcpy(&code, ws->err, sizeof(int), cudaMemcpyDeviceToHost), "CUDA: error word read");
        if (code) return fail(OZA_TIMEOUT, "OzaBLAS: a device-side wait expired (code %d)", code);
    }
    return OZA_OK;
}

oza_status_t oza_ws_set_gemm_config(oza_ws_t ws, const oza_gemm_config_t* cfg) {
    if (!ws) return fail(OZA_INVALID_ARG, "oza_ws_set_gemm_config: null workspace");
    if (!cfg) {
        ws->cfg = oza_gemm_config_t{0, 0, 0};
        return OZA_OK;
    }
    if (cfg->band < 0 || cfg->band > 4096) return fail(OZA_INVALID_ARG, "oza_ws_set_gemm_config: band out of range");
    if (cfg->overlap_chunks < 0 || cfg->overlap_chunks > oza_workspace::Overlap::kMaxChunks)
        return fail(OZA_INVALID_ARG, "oza_ws_set_gemm_config: overlap_chunks must be in [0, 16]");
    if (cfg->wait_hint_ns < 0 || cfg->wait_hint_ns > 1000000)
        return fail(OZA_INVALID_ARG, "oza_ws_set_gemm_config: wait_hint_ns must be in [0, 1e6]");
    ws->cfg = *cfg;
    return OZA_OK;
}

oza_status_t oza_set_residue_slicer(int mode) {
    if (mode != OZA_SLICER_AUTO && mode != OZA_SLICER_TENSOR && mode != OZA_SLICER_CUDA_CORES)
        return fail(OZA_INVALID_ARG,
                    "oza_set_residue_slicer: mode must be OZA_SLICER_AUTO, OZA_SLICER_TENSOR or OZA_SLICER_CUDA_CORES");
    oza::set_residue_slicer(mode);
    return OZA_OK;
}

int oza_get_residue_slicer(void) { return oza::residue_slicer(); }

oza_status_t oza_ws_get_gemm_config(oza_ws_t ws, oza_gemm_config_t* cfg) {
    if (!ws || !cfg) return fail(OZA_INVALID_ARG, "oza_ws_get_gemm_config: null argument");
    *cfg = ws->cfg;
    return OZA_OK;
}

oza_status_t oza_autotune_gemm(oza_ws_t ws, const double* A, const double* B, double* C, oza_gemm_config_t* best,
                               float* best_ms) {
    if (!ws || !best) return fail(OZA_INVALID_ARG, "oza_autotune_gemm: null argument");
    const oza_gemm_config_t saved = ws->cfg;
    std::vector<oza_gemm_config_t> cand;
    const int bands[] = {0, 8, 16, 32};   // 0: the library's default for the shape
    for (int b : bands) cand.push_back(oza_gemm_config_t{b, saved.wait_hint_ns, saved.overlap_chunks});
    float best_t = 1e30f;
    oza_gemm_config_t best_c = saved;
    for (const auto& c : cand) {
        ws->cfg = c;
        oza_timings_t t;
        float tmin = 1e30f;
        for (int rep = 0; rep < 3; ++rep) {
            oza_status_t r = oza_gemm(ws, A, B, C, &t);
            if (r != OZA_OK) {
                ws->cfg = saved;
                return r;
            }
            if (rep > 0) tmin = std::min(tmin, t.step3_ms);
        }
        if (tmin < best_t) {
            best_t = tmin;
            best_c = c;
        }
    }
    ws->cfg = best_c;
    *best = best_c;
    if (best_ms) *best_ms = best_t;
    return OZA_OK;
}

oza_status_t oza_gemm_host(oza_ws_t ws, const double* hA, const double* hB, double* hC, oza_timings_t* timings) {
    if (!ws) return fail(OZA_INVALID_ARG, "oza_gemm_host: null workspace");
    if (timings) std::memset(timings, 0, sizeof(*timings));
    if (ws->M == 0 || ws->N == 0) return OZA_OK;
    if (!hC || (ws->K && (!hA || !hB))) return fail(OZA_INVALID_ARG, "oza_gemm_host: null matrix pointer");
    oza_executor* ex = ws->ex;
    DeviceGuard g(ex->device);
    if (!g.ok) return fail(OZA_CUDA_ERROR, "CUDA: Failed to set device %d", ex->device);
    OZA_CUDA_TRY(host_pipe_init(ws), "oza_gemm_host: staging buffers");
    auto& h = ws->hp;
    cudaStream_t st = ex->stream;
    const size_t M = ws->M, N = ws->N, K = ws->K;
    OZA_CUDA_TRY(cudaEventRecord(h.t0, st), "CUDA: event record");

    // Scheme II fused and Scheme I (without the reference-layout copies) take
    // the row-chunk pipeline.
    const bool pipelined = K && (ws->fused || (ws->scheme == OZA_SCHEME1 && !ws->a_ref));
    if (!pipelined) {
        // The materialised Scheme II path, the reference layouts and K = 0:
        // copy in, compute, copy out.
        if (K) {
            OZA_CUDA_TRY(cudaMemcpyAsync(h.dA, hA, M * K * sizeof(double), cudaMemcpyHostToDevice, st), "H2D A");
            OZA_CUDA_TRY(cudaMemcpyAsync(h.dB, hB, K * N * sizeof(double), cudaMemcpyHostToDevice, st), "H2D B");
        }
        oza_status_t r = oza_gemm(ws, h.dA, h.dB, h.dC, nullptr);
        if (r != OZA_OK) return r;
        OZA_CUDA_TRY(cudaMemcpyAsync(hC, h.dC, M * N * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H C");
    } else {
        // Row-chunk pipeline: B is copied and sliced while A's chunks arrive;
        // each A chunk is sliced, multiplied against all of B (its m-tiles
        // only) and reconstructed, and its rows of C go back while the next
        // chunk is computed.  Copies in and out run on their own streams.
        const bool s2 = ws->scheme == OZA_SCHEME2;
        const int offset = s2 ? ws->k_param : 0;
        const size_t tile_m = oza::kTileM;
        const int mt_all = (int)((M + tile_m - 1) / tile_m);
        // Scheme II: 32 chunks.  The exposed tail after the last A chunk lands
        // (its GEMM, CRT and copy-out) is 1/32 of the compute and of C.  At
        // 8192^3 a chunk's compute (~0.28 ms) still keeps pace with its copy
        // (~0.31 ms), and the call ends ~1 ms above the PCIe floor (1 GiB in
        // with the copy-out of C running beside the second half).  Scheme I:
        // 8 chunks.  Its compute outlasts the copies, and each chunk's GEMM
        // streams every slice plane of B once per group, so fewer, larger
        // chunks.
        const int max_chunks = s2 ? (int)oza_workspace::HostPipe::kMaxChunks : 8;
        const int R0 = std::min(mt_all, max_chunks);
        const int q = (mt_all + R0 - 1) / R0;   // m-tiles per chunk
        const int R = (mt_all + q - 1) / q;
        OZA_CUDA_TRY(cudaStreamWaitEvent(h.cin, h.t0, 0), "CUDA: stream wait");
        OZA_CUDA_TRY(cudaStreamWaitEvent(h.cout, h.t0, 0), "CUDA: stream wait");
        OZA_CUDA_TRY(cudaMemcpyAsync(h.dB, hB, K * N * sizeof(double), cudaMemcpyHostToDevice, h.cin), "H2D B");
        OZA_CUDA_TRY(cudaEventRecord(h.b_in, h.cin), "CUDA: event record");
        OZA_CUDA_TRY(cudaStreamWaitEvent(st, h.b_in, 0), "CUDA: stream wait");
        OZA_CUDA_TRY(oza::launch_stats_cols(h.dB, K, N, ws->colmax, ex->sms, st), "step1 cols");
        OZA_CUDA_TRY(oza::launch_slice_cols(ws->scheme, h.dB, K, N, ws->colmax, offset, ws->S, ws->beta, ws->shiftB,
                                            ws->bplanes, ws->Np, ws->Kp, st, ws->err),
                     "step2 cols");
        for (int c = 0; c < R; ++c) {
            const size_t r0 = (size_t)c * q * tile_m;
            const size_t rows_p = std::min((size_t)q * tile_m, (size_t)mt_all * tile_m - r0);
            const size_t rows = std::min(M, r0 + rows_p) - r0;   // >= 1: every chunk starts below M
            OZA_CUDA_TRY(cudaMemcpyAsync(h.dA + r0 * K, hA + r0 * K, rows * K * sizeof(double),
                                         cudaMemcpyHostToDevice, h.cin),
                         "H2D A chunk");
            OZA_CUDA_TRY(cudaEventRecord(h.a_in[c], h.cin), "CUDA: event record");
            OZA_CUDA_TRY(cudaStreamWaitEvent(st, h.a_in[c], 0), "CUDA: stream wait");
            OZA_CUDA_TRY(oza::launch_stats_rows(h.dA + r0 * K, rows, K, offset, ws->shiftA + r0, ex->sms, st),
                         "step1 rows");
            OZA_CUDA_TRY(oza::launch_slice_rows(ws->scheme, h.dA + r0 * K, rows, K, ws->shiftA + r0, ws->S, ws->beta,
                                                offset, ws->aplanes + r0 * ws->Kp, rows_p, ws->Kp, ex->sms, st,
                                                ws->Mp, ws->err),
                         "step2 rows");
            oza::GemmPlan plan;
            plan.a_planes = ws->aplanes;
            plan.b_planes = ws->bplanes;
            plan.planes = ws->S;
            plan.Mp = ws->Mp;
            plan.Np = ws->Np;
            plan.Kp = ws->Kp;
            plan.M = ws->M;
            plan.N = ws->N;
            plan.pairs = ws->pairs;
            plan.err = ws->err;
            plan.sms = ex->sms;
            plan.ctc = s2 ? nullptr : ws->ctc;
            plan.coef = s2 ? ws->coef : nullptr;
            plan.m_tile_begin = c * q;
            plan.m_tile_count = std::min(q, mt_all - c * q);
            plan.band = ws->cfg.band;
            plan.wait_hint_ns = (uint32_t)ws->cfg.wait_hint_ns;
            OZA_CUDA_TRY(oza::launch_gemm_i8(plan, st), "step3 gemm");
            if (s2) {
                OZA_CUDA_TRY(oza::launch_crt_coef(ws->coef + r0 * ws->Np, ws->Mp, ws->Np, rows, N, ws->S,
                                                  ws->shiftA + r0, ws->shiftB, h.dC + r0 * N, ex->sms, st),
                             "step4 crt");
            } else {
                OZA_CUDA_TRY(oza::launch_reconstruct1(ws->ctc + r0 * ws->Np, ws->Mp, ws->Np, rows, N, ws->S, ws->beta,
                                                      ws->shiftA + r0, ws->shiftB, h.dC + r0 * N, ex->sms, st,
                                                      &ws->pairs),
                             "step4 sum");
            }
            OZA_CUDA_TRY(cudaEventRecord(h.done[c], st), "CUDA: event record");
            OZA_CUDA_TRY(cudaStreamWaitEvent(h.cout, h.done[c], 0), "CUDA: stream wait");
            OZA_CUDA_TRY(cudaMemcpyAsync(hC + r0 * N, h.dC + r0 * N, rows * N * sizeof(double),
                                         cudaMemcpyDeviceToHost, h.cout),
                         "D2H C chunk");
        }
        OZA_CUDA_TRY(cudaEventRecord(h.out_done, h.cout), "CUDA: event record");
        OZA_CUDA_TRY(cudaStreamWaitEvent(st, h.out_done, 0), "CUDA: stream wait");
    }
    OZA_CUDA_TRY(cudaEventRecord(h.t1, st), "CUDA: event record");
    OZA_CUDA_TRY(cudaEventSynchronize(h.t1), "CUDA: event synchronize");
    if (timings) cudaEventElapsedTime(&timings->total_ms, h.t0, h.t1);
    int code = 0;
    OZA_CUDA_TRY(cudaMemcpy(&code, ws->err, sizeof(int), cudaMemcpyDeviceToHost), "CUDA: error word read");
    if (code) return fail(OZA_TIMEOUT, "OzaBLAS: a device-side wait expired (code %d)", code);
    return OZA_OK;
}

oza_status_t oza_selftest_wait_timeout(oza_exec_t ex, double limit_s, int* code, double* elapsed_s) {
    if (!ex || !code) return fail(OZA_INVALID_ARG, "oza_selftest_wait_timeout: null argument");
    if (!(limit_s > 0.0) || limit_s > 5.0) return fail(OZA_INVALID_ARG, "oza_selftest_wait_timeout: limit in (0, 5] s");
    DeviceGuard g(ex->device);
    if (!g.ok) return fail(OZA_CUDA_ERROR, "CUDA: Failed to set device %d", ex->device);
    int* buf = nullptr;
    OZA_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(&buf), 2 * sizeof(int)), "oza_selftest_wait_timeout: alloc");
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaMemset(buf, 0, 2 * sizeof(int));
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) e = cudaEventRecord(e0, ex->stream);
    if (e == cudaSuccess) e = oza::launch_wait_probe(buf, (unsigned long long)(limit_s * 1e9), buf + 1, ex->stream);
    if (e == cudaSuccess) e = cudaEventRecord(e1, ex->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    int host[2] = {0, 0};
    if (e == cudaSuccess) e = cudaMemcpy(host, buf, sizeof(host), cudaMemcpyDeviceToHost);
    float ms = 0.f;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(buf);
    if (e != cudaSuccess) return cuda_fail(e, "oza_selftest_wait_timeout");
    if (host[1]) return fail(OZA_CUDA_ERROR, "oza_selftest_wait_timeout: the wait returned without an arrival");
    *code = host[0];
    if (elapsed_s) *elapsed_s = ms * 1e-3;
    return OZA_OK;
}

// ---------------------------------------------------------------- host utilities
oza_status_t oza_generate_matrix(int rows, int cols, double phi, int seed, double* out) {
    if (rows < 0 || cols < 0 || (!out && rows && cols)) return fail(OZA_INVALID_ARG, "oza_generate_matrix: bad argument");
    std::mt19937 rng(seed);
    std::uniform_real_distribution<double> unif(0.0, 1.0);
    std::normal_distribution<double> norm(0.0, 1.0);
    const size_t n = (size_t)rows * (size_t)cols;
    for (size_t i = 0; i < n; ++i) {
        const double u = 1.0 - unif(rng);   // (0, 1]
        const double g = norm(rng);
        out[i] = (u - 0.5) * std::exp(phi * g);
    }
    return OZA_OK;
}

int oza_scheme1_beta(size_t K) {
    int beta = (int)std::floor((31.0 - std::log2((double)K)) / 2.0);
    return beta < 1 ? 1 : (beta > 7 ? 7 : beta);
}

int oza_scheme2_k_param(int slices, size_t K) {
    if (slices < 1 || slices > 20 || K == 0) return 0;
    // M = prod of the first S moduli, converted to double through 64-bit limbs
    // and a left-to-right sum as the reference does (crt_math.hpp:73-80).
    static const unsigned mod[20] = {251, 241, 239, 233, 229, 227, 223, 211, 199, 197,
                                     193, 191, 181, 179, 173, 167, 163, 157, 151, 149};
    uint64_t w[4] = {1, 0, 0, 0};
    for (int i = 0; i < slices; ++i) {
        unsigned __int128 carry = 0;
        for (int l = 0; l < 4; ++l) {
            unsigned __int128 p = (unsigned __int128)w[l] * mod[i] + carry;
            w[l] = (uint64_t)p;
            carry = p >> 64;
        }
    }
    double Md = 0.0;
    Md += (double)w[0];
    Md += std::ldexp((double)w[1], 64);
    Md += std::ldexp((double)w[2], 128);
    Md += std::ldexp((double)w[3], 192);
    double frac = (Md / 2.0 - 1.0) / (double)K;
    return (int)std::floor(0.5 * std::log2(frac));
}

}  // extern "C"
