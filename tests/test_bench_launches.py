"""The bench's `gpu_launches` claim: kernels per GEMM call under the library's
chunk rule for overlapped Scheme II stages (oza_gemm in oza_capi.cpp)."""
import importlib.util
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.parametrize("M,N,K,want", [
    (8192, 8192, 8192, 6),      # 64 row tiles: the steps in order
    (6144, 6144, 6144, 6),      # 48 tiles: in order
    (6016, 6016, 6016, 10),     # 47 tiles: 2 chunks
    (4096, 4096, 4096, 10),     # 32 tiles: 2 chunks
    (1024, 1024, 65536, 10),    # 8 tiles: 2 chunks
    (1000, 1000, 65536, 10),    # ceil(1000 / 128) = 8 tiles: 2 chunks
    (2048, 2048, 1024, 10),     # 2 M N K = 2^33: 2 chunks
    (2048, 2048, 1023, 6),      # just below 2^33: in order
    (1024, 1024, 1024, 6),      # 8 tiles but 2^31 flops: in order
    (896, 896, 65536, 6),       # 7 tiles: in order
    (100, 100, 100, 6),
])
def test_default_chunk_rule(M, N, K, want):
    assert _bench().launches_per_call(M, N, K, 2, False) == want


@pytest.mark.parametrize("M,chunks,want", [
    (8192, 1, 6), (8192, 2, 10), (8192, 3, 14), (8192, 4, 18), (8192, 16, 66),
    (8192, 20, 66),     # at most 16 chunks
    (896, 5, 18),       # 7 tiles in chunks of 2: 4 chunks
    (896, 16, 30),      # 7 tiles: 7 chunks
    (8320, 16, 2 + 4 * 13),   # 65 tiles in chunks of 5: 13 chunks
])
def test_requested_chunks(M, chunks, want):
    assert _bench().launches_per_call(M, M, M, 2, False, chunks) == want


@pytest.mark.parametrize("scheme,materialize", [(1, False), (2, True)])
def test_unfused_paths_run_in_order(scheme, materialize):
    b = _bench()
    for M in (512, 4096, 8192):
        assert b.launches_per_call(M, M, M, scheme, materialize) == 6
        assert b.launches_per_call(M, M, M, scheme, materialize, 4) == 6
