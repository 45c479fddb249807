// oza_noalloc.cu -- oza_gemm_noalloc: the Ozaki GEMM for callers that cannot
// allocate device memory.
//
// Some callers must not call cudaMalloc: code running while a CUDA stream is
// being captured into a graph (an allocation would break or serialise the
// capture), code inside an application's own memory pool or allocator
// callback, and latency-critical paths that cannot afford the device-wide
// synchronisation cudaMalloc/cudaFree may imply.  For problems whose scratch
// fits in a fixed, statically sized device array, this entry point runs the
// same kernels as oza_gemm with all intermediates placed in that array; the
// caller passes only A, B and C.
//
// The scratch is a file-scope __device__ array of OZA_NOALLOC_SCRATCH_BYTES
// (64 MiB) that every GPU which loads the library holds until the process
// exits.  Host code cannot use the array's name as a device address, so the
// first call on each device looks the address up with cudaGetSymbolAddress
// (and uploads the CRT constant tables); that first call should therefore
// happen before any stream capture.  The looked-up address is cached per
// device for the life of the process: a cudaDeviceReset between calls is not
// supported.  All calls share the one array and it keeps the previous call's
// contents: everything that must start at zero is cleared on the stream.
// Calls whose work overlaps on the GPU (different streams, or host threads
// issuing concurrently) race on the array; issue them on one stream or
// serialise them.
//
// The first 256 bytes of the array hold the device error word (int at offset
// 0): a kernel whose bounded wait expires sets it to 1.  No call clears it;
// oza_noalloc_device_error() reads and clears it, so it reports every call
// since the previous query.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "oza_capi.h"
#include "oza_internal.h"
#include "oza_kernels.h"

namespace {

__device__ __align__(256) unsigned char g_noalloc_scratch[OZA_NOALLOC_SCRATCH_BYTES];

struct DeviceScratch {
    unsigned char* ptr = nullptr;   // device address of g_noalloc_scratch on this device
    int sms = 0;
    bool ready = false;
};

constexpr int kMaxDevices = 64;
std::mutex g_mu;
DeviceScratch g_dev[kMaxDevices];

oza_status_t na_fail(oza_status_t st, const std::string& msg) {
    oza::set_last_error(msg.c_str());   // read back with oza_last_error_string()
    return st;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Per-device set-up, with that device current: scratch address, SM count,
// architecture check and the CRT constant tables.
oza_status_t setup_device(int dev, DeviceScratch** out) {
    if (dev < 0 || dev >= kMaxDevices) return na_fail(OZA_UNSUPPORTED, "oza_gemm_noalloc: device ordinal too large");
    std::lock_guard<std::mutex> lk(g_mu);
    DeviceScratch& d = g_dev[dev];
    if (!d.ready) {
        int major = 0, minor = 0, sms = 0;
        if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return na_fail(OZA_CUDA_ERROR, "oza_gemm_noalloc: cannot query the current device");
        if (major != 10 || minor != 0)
            return na_fail(OZA_UNSUPPORTED, "oza_gemm_noalloc: the current device is not sm_100 (B200)");
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr)
            return na_fail(OZA_CUDA_ERROR, std::string("oza_gemm_noalloc: cudaGetSymbolAddress failed: ") +
                                               cudaGetErrorString(e));
        e = oza::upload_tables();
        if (e != cudaSuccess)
            return na_fail(OZA_CUDA_ERROR, std::string("oza_gemm_noalloc: constant tables: ") + cudaGetErrorString(e));
        d.ptr = static_cast<unsigned char*>(p);
        d.sms = sms;
        d.ready = true;
    }
    *out = &d;
    return OZA_OK;
}

}  // namespace

extern "C" oza_status_t oza_gemm_noalloc(int scheme, int slices, size_t M, size_t N, size_t K, const double* A,
                                         const double* B, double* C, void* stream) {
    if (scheme != OZA_SCHEME1 && scheme != OZA_SCHEME2) return na_fail(OZA_INVALID_ARG, "oza_gemm_noalloc: unknown scheme");
    if (slices < 1 || slices > 20)
        return na_fail(OZA_INVALID_ARG, "oza_gemm_noalloc: slices must be between 1 and 20");
    {
        const oza_status_t chk = oza::check_problem("oza_gemm_noalloc", scheme, M, N, K, slices);
        if (chk != OZA_OK) return chk;
    }
    if (M == 0 || N == 0) return OZA_OK;
    if (!C || (K && (!A || !B))) return na_fail(OZA_INVALID_ARG, "oza_gemm_noalloc: null matrix pointer");
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return na_fail(OZA_CUDA_ERROR, "oza_gemm_noalloc: no current device");
    DeviceScratch* d = nullptr;
    oza_status_t sst = setup_device(dev, &d);
    if (sst != OZA_OK) return sst;

    if (K == 0) {
        if (cudaMemsetAsync(C, 0, M * N * sizeof(double), st) != cudaSuccess)
            return na_fail(OZA_CUDA_ERROR, "oza_gemm_noalloc: memset of C failed");
        return OZA_OK;
    }

    // Same padded layouts as a workspace of oza_ws_create.
    const size_t Mp = oza::round_up(M, oza::kTileM);
    const size_t Np = oza::round_up(N, oza::kTileN);
    const size_t Kp = oza::round_up(K, oza::kTileK);
    const size_t S = (size_t)slices;
    const size_t need_err = 256, need_sa = align256(M * 4), need_sb = align256(N * 4), need_cm = align256(N * 8);
    const size_t need_ap = align256(S * Mp * Kp + 16), need_bp = align256(S * Np * Kp + 16);
    // Scheme I: one INT32 plane per accumulation unit (groups split at large K)
    const size_t planes_out = scheme == OZA_SCHEME2 ? S : (size_t)oza::make_pairs(scheme, slices, K).num_groups;
    const size_t need_out = align256(scheme == OZA_SCHEME2 ? S * Mp * Np + 16 : planes_out * Mp * Np * 4 + 16);
    const size_t need = need_err + need_sa + need_sb + need_cm + need_ap + need_bp + need_out;
    if (need > (size_t)OZA_NOALLOC_SCRATCH_BYTES) {
        char msg[256];
        snprintf(msg, sizeof(msg),
                 "oza_gemm_noalloc: M=%zu N=%zu K=%zu S=%d needs %zu bytes of scratch, more than the built-in "
                 "%zu bytes; use oza_gemm with a workspace",
                 M, N, K, slices, need, (size_t)OZA_NOALLOC_SCRATCH_BYTES);
        return na_fail(OZA_UNSUPPORTED, msg);
    }

    unsigned char* p = d->ptr;
    int* err = reinterpret_cast<int*>(p);
    p += need_err;
    int32_t* shiftA = reinterpret_cast<int32_t*>(p);
    p += need_sa;
    int32_t* shiftB = reinterpret_cast<int32_t*>(p);
    p += need_sb;
    unsigned long long* colmax = reinterpret_cast<unsigned long long*>(p);
    p += need_cm;
    int8_t* aplanes = reinterpret_cast<int8_t*>(p);
    p += need_ap;
    int8_t* bplanes = reinterpret_cast<int8_t*>(p);
    p += need_bp;
    unsigned char* out = p;

    const int k_param = scheme == OZA_SCHEME2 ? oza_scheme2_k_param(slices, K) : 0;
    const int beta = scheme == OZA_SCHEME1 ? oza_scheme1_beta(K) : 0;
    const int sms = d->sms;
#define NA_TRY(call, what)                                                                      \
    do {                                                                                        \
        cudaError_t e__ = (call);                                                               \
        if (e__ != cudaSuccess)                                                                 \
            return na_fail(OZA_CUDA_ERROR, std::string("oza_gemm_noalloc: ") + what + ": " + cudaGetErrorString(e__)); \
    } while (0)
    // The array keeps the last call's contents.  The column maxima are zeroed
    // by the statistics launch; every other intermediate is fully rewritten
    // before it is read; the error word is left as it is (sticky until
    // oza_noalloc_device_error reads it).
    NA_TRY(oza::launch_stats_rows(A, M, K, k_param, shiftA, sms, st), "step 1 (rows)");
    NA_TRY(oza::launch_stats_cols(B, K, N, colmax, sms, st), "step 1 (columns)");
    NA_TRY(oza::launch_slice_rows(scheme, A, M, K, shiftA, slices, beta, k_param, aplanes, Mp, Kp, sms, st, 0, err),
           "step 2 (A)");
    NA_TRY(oza::launch_slice_cols(scheme, B, K, N, colmax, k_param, slices, beta, shiftB, bplanes, Np, Kp, st, err),
           "step 2 (B)");
    oza::GemmPlan plan{};
    plan.a_planes = aplanes;
    plan.b_planes = bplanes;
    plan.planes = slices;
    plan.Mp = Mp;
    plan.Np = Np;
    plan.Kp = Kp;
    plan.M = M;
    plan.N = N;
    plan.pairs = oza::make_pairs(scheme, slices, K);
    plan.err = err;
    plan.sms = sms;
    plan.ctc = scheme == OZA_SCHEME1 ? reinterpret_cast<int32_t*>(out) : nullptr;
    plan.coef = scheme == OZA_SCHEME2 ? out : nullptr;
    NA_TRY(oza::launch_gemm_i8(plan, st), "step 3");
    if (scheme == OZA_SCHEME2)
        NA_TRY(oza::launch_crt_coef(out, Mp, Np, M, N, slices, shiftA, shiftB, C, sms, st), "step 4");
    else
        NA_TRY(oza::launch_reconstruct1(reinterpret_cast<int32_t*>(out), Mp, Np, M, N, slices, beta, shiftA, shiftB,
                                        C, sms, st, &plan.pairs),
               "step 4");
#undef NA_TRY
    return OZA_OK;
}

extern "C" oza_status_t oza_noalloc_device_error(void* stream, int* code) {
    if (!code) return na_fail(OZA_INVALID_ARG, "oza_noalloc_device_error: null argument");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return na_fail(OZA_CUDA_ERROR, "oza_noalloc_device_error: no current device");
    DeviceScratch* d = nullptr;
    oza_status_t sst = setup_device(dev, &d);
    if (sst != OZA_OK) return sst;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int host = 0;
    cudaError_t e = cudaMemcpyAsync(&host, d->ptr, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d->ptr, 0, sizeof(int), st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return na_fail(OZA_CUDA_ERROR, std::string("oza_noalloc_device_error: ") + cudaGetErrorString(e));
    *code = host;
    return OZA_OK;
}

extern "C" oza_status_t oza_noalloc_selftest_wait_timeout(double limit_s, void* stream) {
    if (!(limit_s > 0.0) || limit_s > 5.0)
        return na_fail(OZA_INVALID_ARG, "oza_noalloc_selftest_wait_timeout: limit in (0, 5] s");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
        return na_fail(OZA_CUDA_ERROR, "oza_noalloc_selftest_wait_timeout: no current device");
    DeviceScratch* d = nullptr;
    oza_status_t sst = setup_device(dev, &d);
    if (sst != OZA_OK) return sst;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int* err = reinterpret_cast<int*>(d->ptr);
    int* status = err + 1;   // inside the 256-byte error block
    int host = 0;
    cudaError_t e = cudaMemsetAsync(status, 0, sizeof(int), st);
    if (e == cudaSuccess) e = oza::launch_wait_probe(err, (unsigned long long)(limit_s * 1e9), status, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&host, status, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return na_fail(OZA_CUDA_ERROR, std::string("oza_noalloc_selftest_wait_timeout: ") + cudaGetErrorString(e));
    if (host) return na_fail(OZA_CUDA_ERROR, "oza_noalloc_selftest_wait_timeout: the wait returned without an arrival");
    return OZA_OK;
}
