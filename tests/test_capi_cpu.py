"""The C-ABI library on a host without a GPU: it loads, exports every symbol
include/oza_capi.h declares and the drop-in C++ API, its host utilities match
the reference, and its argument checks fail cleanly.  No GPU compute."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import ozablas_b200 as oz

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_library_exports_every_declared_symbol():
    L = oz.lib()
    declared = oz.exported_symbols()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", oz.LIB_PATH], capture_output=True, text=True).stdout
    for name in declared:
        assert f" T {name}\n" in out, name


def test_library_exports_drop_in_cxx_api():
    out = subprocess.run(["nm", "-DC", "--defined-only", oz.LIB_PATH], capture_output=True, text=True).stdout
    for sym in ("ozablas::ozaki_scheme1_gemm(ozablas::WorkspaceScheme1&, double const*, double const*, double*, "
                "ozablas::OzaTimings*)",
                "ozablas::ozaki_scheme2_gemm(ozablas::WorkspaceScheme2&, double const*, double const*, double*, "
                "ozablas::OzaTimings*)",
                "ozablas::CudaExecutor::CudaExecutor(int)",
                "ozablas::WorkspaceScheme2::WorkspaceScheme2(std::shared_ptr<ozablas::Executor const>, unsigned long, "
                "unsigned long, unsigned long, int)",
                "ozablas::WorkspaceScheme1::get_C_tc() const"):
        assert sym in out, sym


def test_library_has_no_cpu_fallback_symbols():
    """The product library links nothing from the oracle."""
    out = subprocess.run(["nm", "-D", oz.LIB_PATH], capture_output=True, text=True).stdout
    assert " oo_" not in out and " ref_" not in out


def test_version_and_errors():
    L = oz.lib()
    assert b"sm_100a" in L.oza_version()
    h = ctypes.c_void_p()
    assert L.oza_ws_create(None, 2, 8, 8, 8, 8, 0, ctypes.byref(h)) == oz.OZA_INVALID_ARG
    assert b"Executor cannot be null" in L.oza_last_error_string()
    assert L.oza_gemm(None, None, None, None, None) == oz.OZA_INVALID_ARG
    assert L.oza_ws_get_ptr(None, 0, ctypes.byref(h)) == oz.OZA_INVALID_ARG


def test_executor_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(oz.OzaError):
        oz.CudaExecutor(0)


def test_python_api_argument_checks():
    with pytest.raises(ValueError):
        oz.WorkspaceScheme2(None, 4, 4, 4, 8)
    with pytest.raises(oz.OzaError):
        oz.WorkspaceScheme2(oz.CpuExecutor(), 4, 4, 4, 8)


def test_generator_matches_reference_fixture():
    g = np.load(os.path.join(GOLDEN, "generator.npz"))
    for i in range(4):
        r, c, phi, seed = g[f"params{i}"]
        got = oz.generate_matrix(int(r), int(c), float(phi), int(seed))
        assert np.array_equal(got.view(np.int64), g[f"case{i}"].view(np.int64))


def test_reference_generator_build_matches_fixture_and_library():
    """The reference's own generator compiled into oracle/_ref (the bench's
    reference arm draws its inputs with it) gives the fixture's values and
    this library's, bit for bit."""
    from oracle import Ref, ref_available
    if not ref_available():
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    g = np.load(os.path.join(GOLDEN, "generator.npz"))
    for i in range(4):
        r, c, phi, seed = g[f"params{i}"]
        got = Ref.generate_matrix(int(r), int(c), float(phi), int(seed))
        assert np.array_equal(got.view(np.int64), g[f"case{i}"].view(np.int64))
    for r, c, phi, seed in [(64, 8192, 0.5, 42), (8192, 64, 0.5, 43), (33, 77, 4.0, 9)]:
        a, b = Ref.generate_matrix(r, c, phi, seed), oz.generate_matrix(r, c, phi, seed)
        assert np.array_equal(a.view(np.int64), b.view(np.int64))


@pytest.mark.parametrize("K", [1, 5, 64, 1000, 1024, 8192, 65536, 100000])
def test_host_scheme_parameters_match_oracle(K):
    from oracle import Oracle
    assert oz.scheme1_beta(K) == Oracle.beta(K)
    for S in range(1, 21):
        assert oz.scheme2_k_param(S, K) == Oracle.k_param(S, K)


def test_headers_compile_standalone(tmp_path):
    """The drop-in headers compile and link against the library (no GPU needed)."""
    src = tmp_path / "use.cpp"
    src.write_text(r'''
#include <ozablas/ozablas.hpp>
#include <ozablas/core/executor.hpp>
#include <ozablas/core/workspace.hpp>
#include <oza_capi.h>
#include <cstdio>
int main() {
    ozablas::OzaTimings t;
    std::printf("%s %f\n", oza_version(), t.total_ms);
    try { ozablas::HipExecutor h(0); } catch (const std::runtime_error&) { std::printf("hip rejected\n"); }
    return 0;
}
''')
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = tmp_path / "use"
    subprocess.run(["/usr/bin/g++", "-std=c++17", f"-I{root}/include", str(src), "-o", str(exe),
                    f"-L{root}/ozablas_b200", "-loza_b200", f"-Wl,-rpath,{root}/ozablas_b200"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    assert "sm_100a" in out and "hip rejected" in out


def test_accuracy_tools_reject_null_arguments():
    """oza_block_error / oza_autotune_slices validate their arguments before
    touching a device."""
    L = oz.lib()
    s, e = ctypes.c_int(), ctypes.c_double()
    assert L.oza_autotune_slices(None, 2, 4, 4, 4, None, None, 1e-10, 8, 0, ctypes.byref(s),
                                 ctypes.byref(e)) == oz.OZA_INVALID_ARG
    assert L.oza_block_error(None, None, None, None, 4, 4, 4, 8, 0, ctypes.byref(e)) == oz.OZA_INVALID_ARG
    assert "null" in L.oza_last_error_string().decode()
    sc = ctypes.c_int()
    assert L.oza_autotune_scheme_like(None, 4, 4, 4, None, None, None, 1.0, 8, 0, ctypes.byref(sc), ctypes.byref(s),
                                      ctypes.byref(e)) == oz.OZA_INVALID_ARG
    assert "oza_autotune_scheme_like: null" in L.oza_last_error_string().decode()
    assert L.oza_estimate_phi(None, 4, 4, 4, None, None, 8, 0, ctypes.byref(e)) == oz.OZA_INVALID_ARG


def test_group_api_rejects_bad_arguments_without_a_device():
    L = oz.lib()
    h = ctypes.c_void_p()
    one = (ctypes.c_size_t * 1)(4)
    s = (ctypes.c_int * 1)(8)
    assert L.oza_group_create(None, 2, 1, one, one, one, s, 0, ctypes.byref(h)) == oz.OZA_INVALID_ARG
    assert L.oza_group_gemm(None, None, None, None, None) == oz.OZA_INVALID_ARG
    assert L.oza_group_destroy(None) == oz.OZA_OK


@pytest.mark.parametrize("K,want", [(137438, "ok"), (137439, "unsupported")])
def test_scheme2_int32_bound_enforced_by_every_entry_point(K, want):
    """Scheme II's INT32-exact bound (K * 125^2 < 2^31, K <= 137438) and the
    slice range are enforced by one shared check in every GEMM entry point:
    a request beyond the bound is refused with OZA_UNSUPPORTED before any
    device work, in the workspace path, the allocation-free path, the grouped
    GEMM and the request loop.  (At the bound itself the calls reach their
    next check: a missing executor, server or matrix pointer.)"""
    L = oz.lib()
    h = ctypes.c_void_p()
    one = lambda v: (ctypes.c_size_t * 1)(v)   # noqa: E731
    s = (ctypes.c_int * 1)(4)
    rid = ctypes.c_uint64()
    results = {
        "group": L.oza_group_create(None, 2, 1, one(8), one(8), one(K), s, 0, ctypes.byref(h)),
        "server": L.oza_server_submit(None, 2, 8, 8, K, None, None, None, 4, ctypes.byref(rid)),
        "noalloc": L.oza_gemm_noalloc(2, 4, 8, 8, K, None, None, None, None),
    }
    for name, st in results.items():
        if want == "unsupported":
            assert st == oz.OZA_UNSUPPORTED, name
        else:
            assert st == oz.OZA_INVALID_ARG, name   # past the size check, stopped at a null handle/pointer
    assert (oz.Server.request_bytes(8, 8, K, 4) == 0) == (want == "unsupported")
    if want == "unsupported":
        assert "INT32-exact" in L.oza_last_error_string().decode()


def test_shared_check_rejects_slice_counts_and_tma_extents():
    L = oz.lib()
    # slices outside 1..20 (Scheme II: the reference's message)
    assert L.oza_gemm_noalloc(2, 21, 8, 8, 8, None, None, None, None) == oz.OZA_INVALID_ARG
    h = ctypes.c_void_p()
    one = lambda v: (ctypes.c_size_t * 1)(v)   # noqa: E731
    assert L.oza_group_create(None, 2, 1, one(8), one(8), one(8), (ctypes.c_int * 1)(0), 0,
                              ctypes.byref(h)) == oz.OZA_INVALID_ARG
    # 20 planes of 2^27 rows: S * Mp reaches 2^31, beyond 32-bit TMA coordinates
    assert L.oza_gemm_noalloc(1, 20, 1 << 27, 8, 8, None, None, None, None) == oz.OZA_UNSUPPORTED
    assert "too large" in L.oza_last_error_string().decode()


def test_scheme_for_target_picks_the_cheaper_scheme_that_reaches():
    """oza_scheme_for_target: Scheme II whenever its table reaches the target
    with no more INT8 GEMMs than Scheme I's; otherwise Scheme I (its count from
    its own calibrated table); 21 when neither reaches it."""
    for t in (1e-9, 1e-12, 1e-14, 1e-15, 1e-16):
        for K in (128, 1024, 8192, 65536, 200000):
            for phi in (0.5, 1.0, 2.0, 4.0):
                sc, S = oz.scheme_for_target(t, K, phi)
                assert sc in (1, 2) and 1 <= S <= 21
                s2 = oz.slices_for_target(t, K, phi) if K <= 137438 else 21
                if sc == 2:
                    assert S == s2 <= 20
                else:
                    assert s2 > 20 or S * (S + 1) // 2 < s2
    # wide exponent range and tight target: Scheme II's 20 moduli run out
    assert oz.scheme_for_target(1e-15, 16384, 4.0)[0] == 1
    # easy target: Scheme II
    assert oz.scheme_for_target(1e-9, 1024, 0.5)[0] == 2
    with pytest.raises(ValueError):
        oz.scheme_for_target(0.0, 1024, 1.0)


def test_server_api_without_a_device():
    L = oz.lib()
    h = ctypes.c_void_p()
    assert L.oza_server_create(None, None, ctypes.byref(h)) == oz.OZA_INVALID_ARG
    rid = ctypes.c_uint64()
    assert L.oza_server_submit(None, 2, 4, 4, 4, None, None, None, 8, ctypes.byref(rid)) == oz.OZA_INVALID_ARG
    assert L.oza_server_submit(None, 3, 4, 4, 4, None, None, None, 8, ctypes.byref(rid)) == oz.OZA_INVALID_ARG
    assert L.oza_server_destroy(None) == oz.OZA_OK


def test_server_request_bytes_layout():
    """Workspace of one request: shifts, S x (Mp Kp + Np Kp + Mp Np), each part
    rounded to 1 KiB; tiles 128 (M), 256 (N), 128 (K)."""
    ru = lambda x, m: (x + m - 1) // m * m   # noqa: E731
    for M, N, K, S in [(1, 1, 1, 1), (100, 300, 77, 16), (8192, 8192, 1000, 20)]:
        Mp, Np, Kp = ru(M, 128), ru(N, 256), ru(K, 128)
        want = sum(ru(x, 1024) for x in (4 * M, 4 * N, S * Mp * Kp, S * Np * Kp, S * Mp * Np))
        assert oz.Server.request_bytes(M, N, K, S) == want
        want1 = sum(ru(x, 1024) for x in (4 * M, 4 * N, S * Mp * Kp, S * Np * Kp, 4 * S * Mp * Np))
        assert oz.Server.request_bytes(M, N, K, S, scheme=1) == want1
    assert oz.Server.request_bytes(0, 4, 4, 8) == 0
    assert oz.Server.request_bytes(4, 4, 4, 21) == 0
    # Scheme I at K = 65536, S = 9: the groups of 8 and 9 slice pairs take two
    # INT32 planes each (at most 7 pairs per exact INT32 sum): 11 planes
    M, N, K, S = 64, 64, 65536, 9
    Mp, Np, Kp = ru(M, 128), ru(N, 256), ru(K, 128)
    want1 = sum(ru(x, 1024) for x in (4 * M, 4 * N, S * Mp * Kp, S * Np * Kp, 4 * 11 * Mp * Np))
    assert oz.Server.request_bytes(M, N, K, S, scheme=1) == want1


def test_slices_for_target_is_a_monotone_lookup():
    f = oz.slices_for_target
    for phi in (0.5, 1.0, 2.0, 4.0):
        for t in (1e-9, 1e-12, 1e-15):
            s = [f(t, K, phi) for K in (100, 128, 1000, 4096, 65536, 10 ** 6)]
            assert s == sorted(s) and all(1 <= x <= 21 for x in s)
    for K in (256, 8192):
        assert [f(1e-12, K, p) for p in (0.1, 0.5, 1.0, 2.0, 4.0, 9.0)] == sorted(
            f(1e-12, K, p) for p in (0.1, 0.5, 1.0, 2.0, 4.0, 9.0))
        assert [f(t, K, 1.0) for t in (1e-6, 1e-9, 1e-12, 1e-14)] == sorted(
            f(t, K, 1.0) for t in (1e-6, 1e-9, 1e-12, 1e-14))
    assert f(1e-17, 1024, 0.5) == 21
    with pytest.raises(ValueError):
        f(0.0, 1024, 0.5)


def test_selftest_rejects_null_executor():
    code = ctypes.c_int()
    assert oz.lib().oza_selftest_wait_timeout(None, 0.1, ctypes.byref(code), None) == oz.OZA_INVALID_ARG


HARNESSES = ["precision_benchmarks/01_ozaki_scheme2_example.cpp", "precision_benchmarks/02_ozaki_scheme2_fp128_benchmark.cpp",
             "precision_benchmarks/03_ozaki_scheme1_example.cpp", "precision_benchmarks/04_ozaki_scheme1_fp128_benchmark.cpp",
             "performance_benchmarks/01_ozaki_scheme1_2_raw_performance.cpp",
             "performance_benchmarks/02_ozaki_scheme2_pipeline_steps.cpp",
             "performance_benchmarks/03_ozaki_scheme1_pipeline_steps.cpp"]


@pytest.mark.parametrize("src", HARNESSES)
def test_reference_harnesses_build_against_drop_in_headers(src, tmp_path):
    """Every benchmark and example program of the reference compiles, unmodified,
    against this repository's headers (include/ozablas/...) with
    -DOZA_BUILD_CUDA and links against liboza_b200.so: the reference's whole
    public API surface that its own programs use is present here."""
    import __graft_entry__
    ref = __graft_entry__.reference_tree()
    if ref is None:
        pytest.skip("reference tree not available")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = tmp_path / "harness"
    subprocess.run(["/usr/bin/g++", "-std=c++20", "-O0", "-fopenmp", "-DOZA_BUILD_CUDA", f"-I{root}/include",
                    f"-I{ref}/utils", "-I/usr/local/cuda/include", os.path.join(ref, src), "-o", str(exe),
                    f"-L{root}/ozablas_b200", "-loza_b200", "-L/usr/local/cuda/lib64", "-lcublas"], check=True)
    syms = subprocess.run(["nm", "-u", "-C", str(exe)], capture_output=True, text=True, check=True).stdout
    assert "ozablas::CudaExecutor::CudaExecutor(int)" in syms


def test_residue_slicer_knob():
    """The process-wide slicer choice round-trips and rejects unknown modes
    (no GPU call)."""
    import ozablas_b200 as oz
    saved = oz.residue_slicer()
    try:
        assert saved == oz.OZA_SLICER_AUTO
        oz.set_residue_slicer(oz.OZA_SLICER_TENSOR)
        assert oz.residue_slicer() == oz.OZA_SLICER_TENSOR
        oz.set_residue_slicer(oz.OZA_SLICER_CUDA_CORES)
        assert oz.residue_slicer() == oz.OZA_SLICER_CUDA_CORES
        with pytest.raises(ValueError):
            oz.set_residue_slicer(7)
        assert oz.residue_slicer() == oz.OZA_SLICER_CUDA_CORES
    finally:
        oz.set_residue_slicer(saved)
