"""Parity against the reference itself on the GPU: the unmodified OzaBLAS
cuBLAS pipeline (baseline/_ref) and the sm_100a pipeline on the same inputs
must agree bit for bit on shifts, slices/residues, INT32 products and C."""
import numpy as np
import pytest

from tests import ref_gpu
from tests.gpu_helpers import bits, run_pipeline

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_gpu.available(), reason="reference GPU build (baseline/_ref) missing")]


def _oz():
    import ozablas_b200 as oz
    return oz


@pytest.mark.parametrize("S", [3, 7, 8, 13, 16, 20])
def test_scheme2_matches_reference_gpu(executor, S):
    oz = _oz()
    A = oz.generate_matrix(512, 384, 1.0, 42)
    B = oz.generate_matrix(384, 640, 1.0, 43)
    ref = ref_gpu.run(executor, 2, A, B, S)
    got = run_pipeline(oz, executor, 2, A, B, S)
    assert np.array_equal(got["shift_A"], ref["shift_A"])
    assert np.array_equal(got["shift_B"], ref["shift_B"])
    assert np.array_equal(got["A_slices"], ref["A_slices"])
    assert np.array_equal(got["B_slices"], ref["B_slices"])
    assert np.array_equal(got["C_tc"], ref["C_tc"])
    assert np.array_equal(bits(got["C"]), bits(ref["C"]))


@pytest.mark.parametrize("S", [2, 5, 9])
def test_scheme1_matches_reference_gpu(executor, S):
    oz = _oz()
    A = oz.generate_matrix(256, 512, 2.0, 42)
    B = oz.generate_matrix(512, 384, 2.0, 43)
    A[7, :] = 0.0          # all-zero row: the reference casts NaN to int8 here
    B[:, 11] = 0.0
    # maxima within 2^7 of the subnormal range: the reference casts +-inf to int8
    A[9, :] = np.ldexp(1.0, -1024) * (1 + np.arange(A.shape[1]) % 3)
    B[:, 13] = -np.ldexp(1.0, -1020) * (1 + np.arange(B.shape[0]) % 5)
    ref = ref_gpu.run(executor, 1, A, B, S)
    got = run_pipeline(oz, executor, 1, A, B, S)
    assert np.array_equal(got["shift_A"], ref["shift_A"])
    assert np.array_equal(got["shift_B"], ref["shift_B"])
    for name, ax in (("A_slices", 1), ("B_slices", 2)):
        bad = np.unique(np.argwhere(got[name] != ref[name])[:, ax])
        detail = {int(r): (np.unique(np.take(ref[name], r, axis=ax)).tolist()[:8],
                           np.unique(np.take(got[name], r, axis=ax)).tolist()[:8]) for r in bad[:4]}
        assert bad.size == 0, f"{name}: rows/cols {bad.tolist()} differ (reference, ours): {detail}"
    assert np.array_equal(got["C_tc"][S - 1], ref["C_tc"][0])   # last group, g = S + 1
    assert np.array_equal(bits(got["C"]), bits(ref["C"]))


def test_scheme2_4096_matches_reference_gpu(executor):
    """4096^3, phi = 2, 16 moduli, end to end."""
    oz = _oz()
    n = 4096
    A = oz.generate_matrix(n, n, 2.0, 42)
    B = oz.generate_matrix(n, n, 2.0, 43)
    ref = ref_gpu.run(executor, 2, A, B, 16)
    got = run_pipeline(oz, executor, 2, A, B, 16, materialize=False)
    assert np.array_equal(bits(got["C"]), bits(ref["C"]))


@pytest.mark.parametrize("scheme,S", [(2, 12), (1, 6)])
def test_reference_layout_getters_match_reference_buffers(executor, scheme, S):
    """With OZA_WS_REFERENCE_LAYOUT the workspace getters return the
    reference's own layouts, byte for byte what the reference's getters
    (workspace.hpp:14-94) return after the same call: A slices [S][M][K],
    B slices [S][K][N], C_tc [S][M][N] (Scheme II) or the last group (Scheme I)."""
    import ctypes
    import torch
    oz = _oz()
    # sizes the reference's cuBLAS INT8 GEMMs accept (it does not check their
    # status; with K = 333 they refuse and its C_tc stays zero)
    M, N, K = 320, 192, 352
    A = oz.generate_matrix(M, K, 1.0, 42)
    B = oz.generate_matrix(K, N, 1.0, 43)
    ref = ref_gpu.run(executor, scheme, A, B, S)
    ws = (oz.WorkspaceScheme2 if scheme == 2 else oz.WorkspaceScheme1)(executor, M, N, K, S, reference_layout=True)
    dC = torch.empty(M, N, dtype=torch.float64, device="cuda")
    (oz.ozaki_scheme2_gemm if scheme == 2 else oz.ozaki_scheme1_gemm)(
        ws, torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda(), dC)
    torch.cuda.synchronize()

    def grab(ptr, shape, dtype):
        a = np.empty(shape, dtype)
        executor.copy_to_host(a.ctypes.data_as(ctypes.c_void_p).value, ptr, a.nbytes)
        return a

    G = S if scheme == 2 else 1
    assert np.array_equal(grab(ws.get_A_slices(), (S, M, K), np.int8), ref["A_slices"])
    assert np.array_equal(grab(ws.get_B_slices(), (S, K, N), np.int8), ref["B_slices"])
    assert np.array_equal(grab(ws.get_C_tc(), (G, M, N), np.int32), ref["C_tc"])
    assert np.array_equal(grab(ws.get_shift_A(), (M,), np.int32), ref["shift_A"])
    assert np.array_equal(bits(dC.cpu().numpy()), bits(ref["C"]))


def test_scheme1_split_groups_match_reference_gpu(executor):
    """At K = 65536 (beta = 7) a Scheme I group of more than 7 slice pairs
    could overflow an INT32 sum in the worst case, so the library splits such
    groups over several INT32 planes and adds them exactly.  Where the
    reference's INT32 sums do not overflow (random data), everything matches
    it bit for bit: C, shifts, slices, and the last group's buffer, whose
    planes are summed for the reference layout."""
    import ctypes
    import torch
    oz = _oz()
    M, N, K, S = 64, 64, 65536, 9     # groups of 8 and 9 pairs: 11 INT32 planes
    A = oz.generate_matrix(M, K, 1.0, 42)
    B = oz.generate_matrix(K, N, 1.0, 43)
    ref = ref_gpu.run(executor, 1, A, B, S)
    ws = oz.WorkspaceScheme1(executor, M, N, K, S, reference_layout=True)
    assert ws.info["groups"] == 11
    dC = torch.empty(M, N, dtype=torch.float64, device="cuda")
    oz.ozaki_scheme1_gemm(ws, torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda(), dC)
    torch.cuda.synchronize()

    def grab(ptr, shape, dtype):
        a = np.empty(shape, dtype)
        executor.copy_to_host(a.ctypes.data_as(ctypes.c_void_p).value, ptr, a.nbytes)
        return a

    assert np.array_equal(bits(dC.cpu().numpy()), bits(ref["C"]))
    assert np.array_equal(grab(ws.get_shift_A(), (M,), np.int32), ref["shift_A"])
    assert np.array_equal(grab(ws.get_A_slices(), (S, M, K), np.int8), ref["A_slices"])
    assert np.array_equal(grab(ws.get_C_tc(), (1, M, N), np.int32), ref["C_tc"])
