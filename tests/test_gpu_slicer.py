"""Scheme II step 2 on the tensor cores (default for S <= 16) against the
CUDA-core slicer: the residue planes, including their zero K padding, and the
shifts and C must be identical byte for byte, on ragged shapes, every slice
count, the overlapped-stage and host-buffer paths, and inputs with special
values.  Both are also pinned to the oracle elsewhere (test_gpu_parity.py runs
the default)."""
import numpy as np
import pytest

from tests.gpu_helpers import bits, run_pipeline

pytestmark = pytest.mark.gpu


@pytest.fixture
def slicer_mode():
    import ozablas_b200 as oz
    saved = oz.residue_slicer()
    yield oz
    oz.set_residue_slicer(saved)


def _both(oz, executor, A, B, S):
    out = []
    for mode in (oz.OZA_SLICER_TENSOR, oz.OZA_SLICER_CUDA_CORES):
        oz.set_residue_slicer(mode)
        out.append(run_pipeline(oz, executor, 2, A, B, S, materialize=False))
    return out


def _same(a, b):
    for k in ("shift_A", "shift_B"):
        assert np.array_equal(a[k], b[k]), k
    i = a["ws"].info
    M, N = i["M"], i["N"]
    # rows past M / N are never written (nor read); everything else must match
    assert np.array_equal(a["A_planes"][:, :M], b["A_planes"][:, :M]), "A planes"
    assert np.array_equal(a["B_planes"][:, :N], b["B_planes"][:, :N]), "B planes"
    assert np.array_equal(bits(a["C"]), bits(b["C"])), "C"


@pytest.mark.parametrize("S", list(range(1, 17)))
def test_tensor_slicer_matches_cuda_cores_every_S(executor, slicer_mode, S):
    oz = slicer_mode
    A = oz.generate_matrix(200, 300, 1.0, 40 + S)
    B = oz.generate_matrix(300, 136, 1.0, 60 + S)
    t, c = _both(oz, executor, A, B, S)
    _same(t, c)


@pytest.mark.parametrize("shape", [(1, 1, 1), (7, 5, 3), (129, 257, 129), (64, 33, 1000), (300, 17, 64),
                                   (130, 70, 4099), (1000, 1000, 256)])
def test_tensor_slicer_ragged_shapes(executor, slicer_mode, shape):
    oz = slicer_mode
    from oracle import Oracle
    M, N, K = shape
    A = oz.generate_matrix(M, K, 2.0, 3)
    B = oz.generate_matrix(K, N, 2.0, 4)
    t, c = _both(oz, executor, A, B, 16)
    _same(t, c)
    if M * N * K <= 2_000_000:
        ref = Oracle.scheme2(A, B, 16)
        assert np.array_equal(t["A_slices"], ref["A_slices"])
        assert np.array_equal(t["B_slices"], ref["B_slices"])
        assert np.array_equal(bits(t["C"]), bits(ref["C"]))


def test_tensor_slicer_special_values(executor, slicer_mode):
    """Zeros, -0.0, subnormals, powers of two, +-inf and NaN, rows and columns
    scaled far apart: the digits (and so the residues) are those of the
    CUDA-core slicer, whatever the conversion makes of them."""
    oz = slicer_mode
    M, N, K = 96, 80, 136
    A = oz.generate_matrix(M, K, 4.0, 5)
    B = oz.generate_matrix(K, N, 4.0, 6)
    A[3, :] = 0.0
    A[4, :] = -0.0
    A[5, ::3] = 0.0
    A[6, :] = 2.0 ** np.arange(K) % 7
    A[7, :] *= 2.0 ** 300
    A[8, :] = 5e-324 * (np.arange(K) + 1)
    A[9, 5] = np.inf
    A[10, 7] = -np.inf
    A[11, 9] = np.nan
    B[:, 2] = 0.0
    B[:, 3] *= 2.0 ** -300
    B[17, 4] = np.inf
    B[19, 5] = np.nan
    for S in (3, 8, 16):
        t, c = _both(oz, executor, A, B, S)
        _same(t, c)


@pytest.mark.parametrize("chunks", [2, 3, 16])
def test_tensor_slicer_overlapped_and_host_paths(executor, slicer_mode, chunks):
    """Row chunks sliced into their place in full-size planes (overlapped
    stages, and the host-buffer pipeline) give the bits of one full call."""
    import torch
    oz = slicer_mode
    M, N, K = 1100, 700, 520
    hA = oz.generate_matrix(M, K, 1.0, 8)
    hB = oz.generate_matrix(K, N, 1.0, 9)
    A, B = torch.from_numpy(hA).cuda(), torch.from_numpy(hB).cuda()
    W = oz.WorkspaceScheme2(executor, M, N, K, 16)
    oz.set_residue_slicer(oz.OZA_SLICER_CUDA_CORES)
    ref = torch.empty(M, N, dtype=torch.float64, device="cuda")
    oz.ozaki_scheme2_gemm(W, A, B, ref)
    oz.set_residue_slicer(oz.OZA_SLICER_TENSOR)
    W.set_gemm_config(overlap_chunks=chunks)
    for _ in range(2):
        C = torch.full_like(ref, float("nan"))
        oz.ozaki_scheme2_gemm(W, A, B, C)
        assert torch.equal(C.view(torch.int64), ref.view(torch.int64)), chunks
    hC = np.full((M, N), np.nan)
    oz.ozaki_gemm_host(W, hA, hB, hC)
    assert np.array_equal(bits(hC), bits(ref.cpu().numpy()))


def test_tensor_slicer_does_not_report_device_errors(executor, slicer_mode):
    import torch
    oz = slicer_mode
    oz.set_residue_slicer(oz.OZA_SLICER_TENSOR)
    M = N = K = 512
    A = torch.from_numpy(oz.generate_matrix(M, K, 0.5, 1)).cuda()
    B = torch.from_numpy(oz.generate_matrix(K, N, 0.5, 2)).cuda()
    W = oz.WorkspaceScheme2(executor, M, N, K, 16)
    C = torch.empty(M, N, dtype=torch.float64, device="cuda")
    for _ in range(5):
        oz.ozaki_scheme2_gemm(W, A, B, C)
    assert W.device_error() == 0


def test_concurrent_calls_on_two_streams_are_bit_identical(slicer_mode):
    """Calls issued on two streams at once put one call's tensor-core slicers
    beside the other's GEMM or CRT on the same GPU, and the two calls' slicers
    beside each other (TMEM shared by co-resident CTAs).  Every result must
    equal the same call made alone, and no bounded wait may expire."""
    import torch
    oz = slicer_mode
    oz.set_residue_slicer(oz.OZA_SLICER_TENSOR)
    shapes = [(1024, 768, 2048, 16), (2048, 1024, 1024, 12)]
    runs = []
    for (M, N, K, S), seed in zip(shapes, (21, 31)):
        ex = oz.CudaExecutor(0)
        st = torch.cuda.Stream()
        ex.set_stream(st)
        A = torch.from_numpy(oz.generate_matrix(M, K, 1.0, seed)).cuda()
        B = torch.from_numpy(oz.generate_matrix(K, N, 1.0, seed + 1)).cuda()
        W = oz.WorkspaceScheme2(ex, M, N, K, S)
        ref = torch.empty(M, N, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        oz.ozaki_scheme2_gemm(W, A, B, ref)
        st.synchronize()
        outs = [torch.full_like(ref, float("nan")) for _ in range(6)]
        runs.append((ex, st, W, A, B, ref, outs))
    torch.cuda.synchronize()
    for k in range(6):           # interleaved issue: both streams busy at once
        for ex, st, W, A, B, ref, outs in runs:
            oz.ozaki_scheme2_gemm(W, A, B, outs[k])
    torch.cuda.synchronize()
    for ex, st, W, A, B, ref, outs in runs:
        assert W.device_error() == 0
        for C in outs:
            assert torch.equal(C.view(torch.int64), ref.view(torch.int64))
