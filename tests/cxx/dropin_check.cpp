// dropin_check.cpp -- a C++ program written against the drop-in headers only
// (<ozablas/ozablas.hpp>, <ozablas/core/executor.hpp>,
// <ozablas/core/workspace.hpp>) and linked with liboza_b200.so, the way code
// written for the reference's API (include/ozablas/ozablas.hpp:20,31,
// core/executor.hpp:65-87, core/workspace.hpp:14-103) uses it.
//
//   dropin_check <dir> <M> <N> <K> <S2> <S1>
//
// Reads <dir>/A.bin (M x K) and <dir>/B.bin (K x N), row-major FP64; runs
// ozaki_scheme2_gemm with S2 moduli and ozaki_scheme1_gemm with S1 slices,
// each once without and once with OzaTimings; writes C2_async.bin,
// C2_timed.bin, C1_async.bin, C1_timed.bin and shiftA2.bin (int32[M]); checks
// the reference's exceptions; prints one "ok" line per check and "DONE".
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "ozablas/core/executor.hpp"
#include "ozablas/core/workspace.hpp"
#include "ozablas/ozablas.hpp"

namespace {

std::vector<char> read_file(const std::string& path, size_t bytes) {
    std::ifstream f(path, std::ios::binary);
    std::vector<char> buf(bytes);
    if (!f.read(buf.data(), (std::streamsize)bytes)) throw std::runtime_error("cannot read " + path);
    return buf;
}

void write_file(const std::string& path, const void* p, size_t bytes) {
    std::ofstream f(path, std::ios::binary);
    if (!f.write(static_cast<const char*>(p), (std::streamsize)bytes)) throw std::runtime_error("cannot write " + path);
}

template <class Ex, class F>
bool throws(F&& f) {
    try {
        f();
    } catch (const Ex&) {
        return true;
    } catch (...) {
        return false;
    }
    return false;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 7) {
        std::fprintf(stderr, "usage: %s dir M N K S2 S1\n", argv[0]);
        return 2;
    }
    const std::string dir = argv[1];
    const size_t M = std::strtoull(argv[2], nullptr, 10), N = std::strtoull(argv[3], nullptr, 10),
                 K = std::strtoull(argv[4], nullptr, 10);
    const int S2 = std::atoi(argv[5]), S1 = std::atoi(argv[6]);
    const size_t bA = M * K * sizeof(double), bB = K * N * sizeof(double), bC = M * N * sizeof(double);

    // Reference usage: a shared_ptr<Executor> holding a CudaExecutor.
    std::shared_ptr<ozablas::Executor> exec = std::make_shared<ozablas::CudaExecutor>(0);
    std::vector<char> hA = read_file(dir + "/A.bin", bA), hB = read_file(dir + "/B.bin", bB);
    double *dA = nullptr, *dB = nullptr, *dC = nullptr;
    exec->allocate((void**)&dA, bA);
    exec->allocate((void**)&dB, bB);
    exec->allocate((void**)&dC, bC);
    exec->copy_from_host(dA, hA.data(), bA);
    exec->copy_from_host(dB, hB.data(), bB);
    std::vector<double> hC(M * N);

    {
        ozablas::WorkspaceScheme2 ws(exec, M, N, K, S2);
        if (ws.get_M() != M || ws.get_N() != N || ws.get_K() != K || ws.get_slices() != S2 ||
            ws.get_executor() != exec)
            throw std::runtime_error("WorkspaceScheme2 getters");
        ozablas::ozaki_scheme2_gemm(ws, dA, dB, dC);   // asynchronous, no timings
        exec->synchronize();
        exec->copy_to_host(hC.data(), dC, bC);
        write_file(dir + "/C2_async.bin", hC.data(), bC);
        ozablas::OzaTimings t;
        ozablas::ozaki_scheme2_gemm(ws, dA, dB, dC, &t);   // synchronous, per-step times
        exec->copy_to_host(hC.data(), dC, bC);
        write_file(dir + "/C2_timed.bin", hC.data(), bC);
        if (!(t.total_ms > 0.0f) || t.step1_ms < 0.0f || t.step2_ms < 0.0f || t.step3_ms <= 0.0f || t.step4_ms < 0.0f)
            throw std::runtime_error("OzaTimings not filled");
        std::vector<int32_t> sh(M);
        exec->copy_to_host(sh.data(), ws.get_shift_A(), M * sizeof(int32_t));
        write_file(dir + "/shiftA2.bin", sh.data(), M * sizeof(int32_t));
        std::printf("ok scheme2 S=%d total_ms=%.3f\n", S2, t.total_ms);
    }
    {
        // Extension: the reference's buffer layouts from the getters.
        ozablas::WorkspaceScheme2 ws(exec, M, N, K, S2, ozablas::WorkspaceLayout::Reference);
        ozablas::ozaki_scheme2_gemm(ws, dA, dB, dC);
        exec->synchronize();
        std::vector<int8_t> sl((size_t)S2 * M * K);
        exec->copy_to_host(sl.data(), ws.get_A_slices(), sl.size());
        write_file(dir + "/A2_slices.bin", sl.data(), sl.size());
        std::vector<int8_t> slb((size_t)S2 * K * N);
        exec->copy_to_host(slb.data(), ws.get_B_slices(), slb.size());
        write_file(dir + "/B2_slices.bin", slb.data(), slb.size());
        std::printf("ok reference layout\n");
    }
    {
        ozablas::WorkspaceScheme1 ws(exec, M, N, K, S1);
        ozablas::ozaki_scheme1_gemm(ws, dA, dB, dC);
        exec->synchronize();
        exec->copy_to_host(hC.data(), dC, bC);
        write_file(dir + "/C1_async.bin", hC.data(), bC);
        ozablas::OzaTimings t;
        ozablas::ozaki_scheme1_gemm(ws, dA, dB, dC, &t);
        exec->copy_to_host(hC.data(), dC, bC);
        write_file(dir + "/C1_timed.bin", hC.data(), bC);
        std::printf("ok scheme1 S=%d total_ms=%.3f\n", S1, t.total_ms);
    }

    // The reference's error contract (src/core/workspace.cpp:24-25, 68-71;
    // src/ozablas.cpp:42-45, 71-73).
    if (!throws<std::invalid_argument>([&] { ozablas::WorkspaceScheme2 w(exec, M, N, K, 21); }))
        throw std::runtime_error("slices = 21 must throw std::invalid_argument");
    if (!throws<std::invalid_argument>([&] { ozablas::WorkspaceScheme2 w(exec, M, N, K, 0); }))
        throw std::runtime_error("slices = 0 must throw std::invalid_argument");
    if (!throws<std::invalid_argument>([&] { ozablas::WorkspaceScheme1 w(exec, M, N, K, 0); }))
        throw std::runtime_error("Scheme I slices = 0 must throw std::invalid_argument");
    if (!throws<std::invalid_argument>([&] { ozablas::WorkspaceScheme2 w(nullptr, M, N, K, 8); }))
        throw std::runtime_error("a null executor must throw std::invalid_argument");
    std::shared_ptr<ozablas::Executor> cpu = std::make_shared<ozablas::CpuExecutor>();
    if (!throws<std::runtime_error>([&] { ozablas::WorkspaceScheme2 w(cpu, M, N, K, 8); }))
        throw std::runtime_error("a CpuExecutor must throw std::runtime_error");
    if (!throws<std::runtime_error>([&] { ozablas::HipExecutor h(0); }))
        throw std::runtime_error("HipExecutor must throw std::runtime_error");
    std::printf("ok exceptions\n");

    exec->free(dA);
    exec->free(dB);
    exec->free(dC);
    std::printf("DONE\n");
    return 0;
}
