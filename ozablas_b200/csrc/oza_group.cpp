// oza_group.cpp -- C ABI of the grouped Scheme II GEMM: many independent FP64
// GEMMs of different shapes run as one launch per stage (stats, slicers,
// one persistent tcgen05 GEMM over all problems' work units, CRT), captured
// once into a CUDA graph and replayed by every call.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "oza_capi.h"
#include "oza_internal.h"
#include "oza_kernels.h"

using oza::DeviceGuard;

namespace {

oza_status_t gfail(oza_status_t st, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    oza::set_last_error(buf);
    return st;
}

oza_status_t gcuda(cudaError_t e, const char* what) {
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return gfail(OZA_OOM, "%s: %s", what, cudaGetErrorString(e));
    }
    return gfail(OZA_CUDA_ERROR, "%s: %s", what, cudaGetErrorString(e));
}

#define G_TRY(call, what)                                  \
    do {                                                   \
        cudaError_t e__ = (call);                          \
        if (e__ != cudaSuccess) return gcuda(e__, what);   \
    } while (0)

constexpr size_t kAlign = 1024;
size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

}  // namespace

struct oza_group {
    oza_executor* ex = nullptr;
    unsigned flags = 0;
    size_t count = 0;
    std::vector<oza::GroupProblem> probs;
    void* pool = nullptr;                 // all per-problem buffers
    unsigned long long* colmax = nullptr; // all problems' column maxima, contiguous
    size_t colmax_count = 0;
    size_t bytes = 0;
    int* err = nullptr;
    oza::GroupPlan* plan = nullptr;
    cudaStream_t capture = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    std::vector<const double*> A, B;
    std::vector<double*> C;
};

namespace {

void group_release(oza_group* g) {
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    if (g->capture) cudaStreamDestroy(g->capture);
    oza::group_plan_destroy(g->plan);
    for (auto& e : g->ev)
        if (e) cudaEventDestroy(e);
    if (g->pool) cudaFree(g->pool);
    if (g->colmax) cudaFree(g->colmax);
    if (g->err) cudaFree(g->err);
}

}  // namespace

extern "C" {

oza_status_t oza_group_create(oza_exec_t ex, int scheme, size_t count, const size_t* M, const size_t* N,
                              const size_t* K, const int* slices, unsigned flags, oza_group_t* out) {
    if (!out) return gfail(OZA_INVALID_ARG, "oza_group_create: null output handle");
    *out = nullptr;
    if (scheme != OZA_SCHEME2) return gfail(OZA_UNSUPPORTED, "oza_group_create: only Scheme II is grouped");
    if (count == 0 || !M || !N || !K || !slices) return gfail(OZA_INVALID_ARG, "oza_group_create: empty problem list");
    if (count > (1u << 20)) return gfail(OZA_INVALID_ARG, "oza_group_create: too many problems (%zu)", count);
    if (flags & ~OZA_GROUP_NO_GRAPH) return gfail(OZA_INVALID_ARG, "oza_group_create: unknown flags 0x%x", flags);
    for (size_t i = 0; i < count; ++i) {
        if (M[i] == 0 || N[i] == 0 || K[i] == 0)
            return gfail(OZA_INVALID_ARG, "oza_group_create: problem %zu has a zero dimension", i);
        if (M[i] > (1u << 30) || N[i] > (1u << 30) || K[i] > (1u << 30))
            return gfail(OZA_INVALID_ARG, "oza_group_create: problem %zu is too large", i);
        if (slices[i] < 1 || slices[i] > 20)
            return gfail(OZA_INVALID_ARG, "oza_group_create: problem %zu: Scheme II supports 1 to 20 slices", i);
        const oza_status_t chk = oza::check_problem("oza_group_create", OZA_SCHEME2, M[i], N[i], K[i], slices[i]);
        if (chk != OZA_OK) return chk;
    }
    if (!ex) return gfail(OZA_INVALID_ARG, "oza_group_create: null executor");
    DeviceGuard dg(ex->device);
    if (!dg.ok) return gfail(OZA_CUDA_ERROR, "CUDA: Failed to set device %d", ex->device);
    G_TRY(oza::upload_tables(), "CUDA: constant tables");

    auto* g = new (std::nothrow) oza_group();
    if (!g) return gfail(OZA_OOM, "oza_group_create: host allocation failed");
    g->ex = ex;
    g->flags = flags;
    g->count = count;
    g->probs.resize(count);
    // Layout: per problem shiftA, shiftB, A planes, B^T planes, coefficient planes.
    size_t off = 0, ncol = 0;
    std::vector<size_t> offs(count * 5), coloff(count);
    for (size_t i = 0; i < count; ++i) {
        oza::GroupProblem& p = g->probs[i];
        p.M = M[i];
        p.N = N[i];
        p.K = K[i];
        p.Mp = oza::round_up(M[i], oza::kTileM);
        p.Np = oza::round_up(N[i], oza::kTileN);
        p.Kp = oza::round_up(K[i], oza::kTileK);
        p.S = slices[i];
        p.k_param = oza_scheme2_k_param(p.S, K[i]);
        const size_t S = (size_t)p.S;
        const size_t sz[5] = {p.M * 4, p.N * 4, S * p.Mp * p.Kp, S * p.Np * p.Kp, S * p.Mp * p.Np};
        for (int k = 0; k < 5; ++k) {
            offs[5 * i + k] = off;
            off = align_up(off + sz[k]);
        }
        coloff[i] = ncol;
        ncol += p.N;
    }
    g->bytes = off + ncol * 8 + sizeof(int);
    cudaError_t e = cudaMalloc(&g->pool, off);
    if (e == cudaSuccess) e = cudaMalloc((void**)&g->colmax, ncol * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc((void**)&g->err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(g->err, 0, sizeof(int));
    for (int i = 0; i < 5 && e == cudaSuccess; ++i) e = cudaEventCreate(&g->ev[i]);
    if (e != cudaSuccess) {
        group_release(g);
        delete g;
        return gcuda(e, "oza_group_create: device allocation");
    }
    g->colmax_count = ncol;
    uint8_t* base = static_cast<uint8_t*>(g->pool);
    for (size_t i = 0; i < count; ++i) {
        oza::GroupProblem& p = g->probs[i];
        p.shiftA = reinterpret_cast<int32_t*>(base + offs[5 * i]);
        p.shiftB = reinterpret_cast<int32_t*>(base + offs[5 * i + 1]);
        p.a_planes = reinterpret_cast<int8_t*>(base + offs[5 * i + 2]);
        p.b_planes = reinterpret_cast<int8_t*>(base + offs[5 * i + 3]);
        p.coef = base + offs[5 * i + 4];
        p.colmax = g->colmax + coloff[i];
        p.A = nullptr;
        p.B = nullptr;
        p.C = nullptr;
    }
    e = oza::group_plan_create(g->probs.data(), (int)count, g->err, &g->plan);
    if (e != cudaSuccess) {
        group_release(g);
        delete g;
        return gcuda(e, "oza_group_create: work tables");
    }
    g->A.assign(count, nullptr);
    g->B.assign(count, nullptr);
    g->C.assign(count, nullptr);
    *out = g;
    return OZA_OK;
}

oza_status_t oza_group_destroy(oza_group_t g) {
    if (!g) return OZA_OK;
    DeviceGuard dg(g->ex->device);
    cudaStreamSynchronize(g->ex->stream);
    group_release(g);
    delete g;
    return OZA_OK;
}

oza_status_t oza_group_gemm(oza_group_t g, const double* const* A, const double* const* B, double* const* C,
                            oza_timings_t* timings) {
    if (!g) return gfail(OZA_INVALID_ARG, "oza_group_gemm: null group");
    if (!A || !B || !C) return gfail(OZA_INVALID_ARG, "oza_group_gemm: null pointer array");
    for (size_t i = 0; i < g->count; ++i)
        if (!A[i] || !B[i] || !C[i]) return gfail(OZA_INVALID_ARG, "oza_group_gemm: null matrix of problem %zu", i);
    oza_executor* ex = g->ex;
    DeviceGuard dg(ex->device);
    if (!dg.ok) return gfail(OZA_CUDA_ERROR, "CUDA: Failed to set device %d", ex->device);
    cudaStream_t st = ex->stream;
    G_TRY(oza::group_plan_set_matrices(g->plan, A, B, C, st), "oza_group_gemm: pointer upload");

    if (timings) {
        // Eager launches with events between the steps.
        G_TRY(oza::group_plan_launch(g->plan, g->colmax, g->colmax_count, ex->sms, st, g->ev), "oza_group_gemm");
        G_TRY(cudaEventSynchronize(g->ev[4]), "CUDA: event synchronize");
        cudaEventElapsedTime(&timings->step1_ms, g->ev[0], g->ev[1]);
        cudaEventElapsedTime(&timings->step2_ms, g->ev[1], g->ev[2]);
        cudaEventElapsedTime(&timings->step3_ms, g->ev[2], g->ev[3]);
        cudaEventElapsedTime(&timings->step4_ms, g->ev[3], g->ev[4]);
        cudaEventElapsedTime(&timings->total_ms, g->ev[0], g->ev[4]);
        int code = 0;
        G_TRY(cudaMemcpy(&code, g->err, sizeof(int), cudaMemcpyDeviceToHost), "CUDA: error word read");
        if (code) return gfail(OZA_TIMEOUT, "OzaBLAS: a device-side wait expired (code %d)", code);
        return OZA_OK;
    }
    if (g->flags & OZA_GROUP_NO_GRAPH) {
        G_TRY(oza::group_plan_launch(g->plan, g->colmax, g->colmax_count, ex->sms, st, nullptr), "oza_group_gemm");
        return OZA_OK;
    }
    if (!g->exec) {
        // Capture the launch sequence once on a private stream; replays run on
        // the executor's stream.
        if (!g->capture) G_TRY(cudaStreamCreateWithFlags(&g->capture, cudaStreamNonBlocking), "CUDA: stream");
        G_TRY(cudaStreamBeginCapture(g->capture, cudaStreamCaptureModeThreadLocal), "CUDA: begin capture");
        cudaError_t le = oza::group_plan_launch(g->plan, g->colmax, g->colmax_count, ex->sms, g->capture, nullptr);
        cudaGraph_t graph = nullptr;
        cudaError_t ce = cudaStreamEndCapture(g->capture, &graph);
        if (le != cudaSuccess || ce != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            return gcuda(le != cudaSuccess ? le : ce, "oza_group_gemm: graph capture");
        }
        cudaGraphExec_t exec = nullptr;
        cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
        if (ie != cudaSuccess) {
            cudaGraphDestroy(graph);
            return gcuda(ie, "oza_group_gemm: graph instantiate");
        }
        g->graph = graph;
        g->exec = exec;
    }
    G_TRY(cudaGraphLaunch(g->exec, st), "oza_group_gemm: graph launch");
    return OZA_OK;
}

oza_status_t oza_group_get_info(oza_group_t g, oza_group_info_t* info) {
    if (!g || !info) return gfail(OZA_INVALID_ARG, "oza_group_get_info: null argument");
    info->count = g->count;
    info->units = oza::group_plan_units(g->plan);
    info->bytes = g->bytes + oza::group_plan_table_bytes(g->plan);
    info->launches = oza::group_plan_launches(g->plan);
    info->graph = (g->flags & OZA_GROUP_NO_GRAPH) ? 0 : 1;
    return OZA_OK;
}

oza_status_t oza_group_device_error(oza_group_t g, int* code) {
    if (!g || !code) return gfail(OZA_INVALID_ARG, "oza_group_device_error: null argument");
    DeviceGuard dg(g->ex->device);
    G_TRY(cudaMemcpy(code, g->err, sizeof(int), cudaMemcpyDeviceToHost), "CUDA: error word read");
    return OZA_OK;
}

}  // extern "C"
