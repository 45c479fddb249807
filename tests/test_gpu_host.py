"""oza_gemm_host: host-buffer GEMM with the row-chunk copy/compute pipeline;
results bit-identical to the device-buffer call (pinned and pageable host
memory, ragged shapes, every fallback path)."""
import numpy as np
import pytest

import ozablas_b200 as oz

pytestmark = pytest.mark.gpu


def _device_result(executor, scheme, A, B, S, materialize=False):
    import torch
    M, K = A.shape
    N = B.shape[1]
    W = (oz.WorkspaceScheme2 if scheme == 2 else oz.WorkspaceScheme1)(executor, M, N, K, S, materialize=materialize)
    C = torch.empty(M, N, dtype=torch.float64, device="cuda")
    (oz.ozaki_scheme2_gemm if scheme == 2 else oz.ozaki_scheme1_gemm)(W, torch.from_numpy(A).cuda(),
                                                                      torch.from_numpy(B).cuda(), C)
    return C.cpu().numpy()


@pytest.mark.parametrize("M,N,K,S", [(1000, 700, 900, 16), (2304, 512, 300, 12), (130, 2000, 64, 20),
                                     (1, 1, 1, 8), (257, 255, 129, 19)])
@pytest.mark.parametrize("pinned", [True, False])
def test_host_gemm_matches_device_gemm(executor, M, N, K, S, pinned):
    import torch
    A = oz.generate_matrix(M, K, 1.0, 3)
    B = oz.generate_matrix(K, N, 1.0, 4)
    want = _device_result(executor, 2, A, B, S)
    ws = oz.WorkspaceScheme2(executor, M, N, K, S)
    if pinned:
        hA = torch.from_numpy(A).pin_memory()
        hB = torch.from_numpy(B).pin_memory()
        hC = torch.full((M, N), float("nan"), dtype=torch.float64).pin_memory()
    else:
        hA, hB, hC = A, B, np.full((M, N), np.nan)
    t = oz.OzaTimings()
    for _ in range(2):   # the second call reuses the staging buffers
        oz.ozaki_gemm_host(ws, hA, hB, hC, t)
    got = hC.numpy() if pinned else hC
    assert np.array_equal(got.view(np.int64), want.view(np.int64))
    assert t.total_ms > 0


@pytest.mark.parametrize("M,N,K,S", [(300, 200, 500, 6), (1000, 700, 900, 8), (2304, 512, 300, 4), (1, 1, 1, 3),
                                     (1500, 130, 257, 9)])
def test_host_gemm_scheme1_pipeline(executor, M, N, K, S):
    """Scheme I on the row-chunk pipeline (up to 8 chunks), pinned and not."""
    import torch
    A = oz.generate_matrix(M, K, 0.5, 8)
    B = oz.generate_matrix(K, N, 0.5, 9)
    want = _device_result(executor, 1, A, B, S)
    W = oz.WorkspaceScheme1(executor, M, N, K, S)
    C = np.full((M, N), np.nan)
    oz.ozaki_gemm_host(W, A, B, C)
    assert np.array_equal(C.view(np.int64), want.view(np.int64))
    hC = torch.full((M, N), float("nan"), dtype=torch.float64).pin_memory()
    oz.ozaki_gemm_host(W, torch.from_numpy(A).pin_memory(), torch.from_numpy(B).pin_memory(), hC)
    assert np.array_equal(hC.numpy().view(np.int64), want.view(np.int64))


def test_host_gemm_unpipelined_path(executor):
    """Materialised Scheme II: copy in, compute, copy out."""
    M, N, K, S = 300, 200, 500, 6
    A = oz.generate_matrix(M, K, 0.5, 8)
    B = oz.generate_matrix(K, N, 0.5, 9)
    want = _device_result(executor, 2, A, B, S, True)
    W = oz.WorkspaceScheme2(executor, M, N, K, S, materialize=True)
    C = np.empty((M, N))
    oz.ozaki_gemm_host(W, A, B, C)
    assert np.array_equal(C.view(np.int64), want.view(np.int64))


def test_host_gemm_rejects_device_and_misshaped_buffers(executor):
    import torch
    ws = oz.WorkspaceScheme2(executor, 8, 8, 8, 8)
    with pytest.raises(ValueError):
        oz.ozaki_gemm_host(ws, torch.zeros(8, 8, dtype=torch.float64, device="cuda"), np.zeros((8, 8)),
                           np.zeros((8, 8)))
    with pytest.raises(ValueError):
        oz.ozaki_gemm_host(ws, np.zeros((8, 7)), np.zeros((7, 8)), np.zeros((8, 8)))


@pytest.mark.parametrize("M,N,K,S", [(257, 255, 129, 19), (2304, 512, 300, 12), (700, 130, 96, 8),
                                     (4500, 136, 96, 8), (8300, 72, 40, 5)])
def test_host_gemm_row_chunks_cover_m(executor, M, N, K, S):
    """Row chunks of 128-row tiles cover M exactly, also when M is not a
    multiple of the tile and when a chunk holds several tiles (more tiles
    than the 32 chunks)."""
    import torch
    A = oz.generate_matrix(M, K, 0.5, 13)
    B = oz.generate_matrix(K, N, 0.5, 14)
    want = _device_result(executor, 2, A, B, S)
    ws = oz.WorkspaceScheme2(executor, M, N, K, S)
    hC = torch.full((M, N), float("nan"), dtype=torch.float64).pin_memory()
    oz.ozaki_gemm_host(ws, torch.from_numpy(A).pin_memory(), torch.from_numpy(B).pin_memory(), hC)
    assert np.array_equal(hC.numpy().view(np.int64), want.view(np.int64))
