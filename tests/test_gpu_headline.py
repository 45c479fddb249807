"""Bit-exact parity at the benchmarked sizes.

* 8192^3, Scheme II, 16 moduli, phi = 0.5, generator seeds 42/43 -- the
  default bench workload -- and 8192^3, Scheme I, 8 slices (its equal-error
  point): shifts, slices/residues, INT32 products and C against the
  reference's own GPU pipeline (baseline/_ref: its unmodified cuBLAS-backed
  src/cuda/pipeline.cu:40-265), compared on the device.  The bench's path (the
  fused coefficient epilogue for Scheme II) must give the same C as the
  reference; the intermediates come from a materialising workspace.
* The two precision-targeted shapes (16384 x 16384 x 1024 and 1024 x 1024 x
  65536, phi = 4, 5% zeros, rows and columns scaled by 2^+-300), at the slice
  counts their autotuning picks: the reference's 32-bit indices overflow
  there, so seeded 128 x 128 blocks of C are compared with the CPU oracle
  run on the gathered rows of A and columns of B (step 1 is per row of A and
  per column of B, so the gathered product reproduces those entries of the
  full run exactly).
"""
import numpy as np
import pytest

from tests import ref_gpu

pytestmark = pytest.mark.gpu


def _oz():
    import ozablas_b200 as oz
    return oz


def _dev(executor, ptr, shape, dtype):
    import torch
    t = torch.empty(shape, dtype=dtype, device="cuda")
    executor.copy_device_to_device(t.data_ptr(), ptr, t.numel() * t.element_size())
    return t


def _ours_device(executor, scheme, dA, dB, S, materialize):
    import torch
    oz = _oz()
    M, K = dA.shape
    N = dB.shape[1]
    ws = (oz.WorkspaceScheme2 if scheme == 2 else oz.WorkspaceScheme1)(executor, M, N, K, S, materialize=materialize)
    dC = torch.full((M, N), float("nan"), dtype=torch.float64, device="cuda")
    (oz.ozaki_scheme2_gemm if scheme == 2 else oz.ozaki_scheme1_gemm)(ws, dA, dB, dC)
    torch.cuda.synchronize()
    assert ws.device_error() == 0
    out = dict(C=dC)
    if materialize:
        i = ws.info
        Mp, Np, Kp, G = i["Mp"], i["Np"], i["Kp"], i["groups"]
        out["shift_A"] = _dev(executor, ws.get_shift_A(), (M,), torch.int32)
        out["shift_B"] = _dev(executor, ws.get_shift_B(), (N,), torch.int32)
        out["A_planes"] = _dev(executor, ws.get_A_slices(), (S, Mp, Kp), torch.int8)
        out["B_planes"] = _dev(executor, ws.get_B_slices(), (S, Np, Kp), torch.int8)
        out["C_planes"] = _dev(executor, ws.get_C_tc(), (G, Mp, Np), torch.int32)
    return out


def _same_bits(a, b):
    import torch
    return torch.equal(a.contiguous().view(torch.int64), b.contiguous().view(torch.int64))


@pytest.mark.skipif(not ref_gpu.available(), reason="reference GPU build (baseline/_ref) missing")
@pytest.mark.parametrize("scheme,S", [(2, 16), (1, 8)])
def test_8192_cubed_matches_reference_gpu_bit_for_bit(executor, scheme, S):
    import torch
    oz = _oz()
    n = 8192
    dA = torch.from_numpy(oz.generate_matrix(n, n, 0.5, 42)).cuda()
    dB = torch.from_numpy(oz.generate_matrix(n, n, 0.5, 43)).cuda()
    ref = ref_gpu.run_device(executor, scheme, dA, dB, S)
    if scheme == 2:
        fused = _ours_device(executor, 2, dA, dB, S, materialize=False)   # the bench's path
        assert _same_bits(fused["C"], ref["C"]), "C of the fused path"
        del fused
    got = _ours_device(executor, scheme, dA, dB, S, materialize=True)
    assert torch.equal(got["shift_A"], ref["shift_A"]), "shift_A"
    assert torch.equal(got["shift_B"], ref["shift_B"]), "shift_B"
    for s in range(S):   # plane by plane: the padded K-major layouts against [S][M][K] / [S][K][N]
        assert torch.equal(got["A_planes"][s, :n, :n], ref["A_slices"][s]), f"A plane {s}"
        assert torch.equal(got["B_planes"][s, :n, :n].t(), ref["B_slices"][s]), f"B plane {s}"
    if scheme == 2:
        for s in range(S):
            assert torch.equal(got["C_planes"][s, :n, :n], ref["C_tc"][s]), f"INT32 product {s}"
    else:   # the reference keeps only the last group, g = S + 1
        assert torch.equal(got["C_planes"][S - 1, :n, :n], ref["C_tc"][0]), "last INT32 group"
    assert _same_bits(got["C"], ref["C"]), "C"


def _precision_inputs(M, N, K):
    import importlib.util
    import os
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    spec = importlib.util.spec_from_file_location("bench_inputs", os.path.join(root, "bench.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    return b.precision_inputs(M, N, K)


@pytest.mark.parametrize("shape,scheme,S", [((16384, 16384, 1024), 2, 20), ((16384, 16384, 1024), 1, 11),
                                            ((1024, 1024, 65536), 2, 20), ((1024, 1024, 65536), 1, 11)])
def test_precision_shapes_blocks_match_oracle(executor, shape, scheme, S):
    import torch
    from oracle import Oracle
    M, N, K = shape
    A, B, rows, cols = _precision_inputs(M, N, K)
    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    got = _ours_device(executor, scheme, dA, dB, S, materialize=False)["C"]
    rng = np.random.default_rng(11)
    I = np.unique(np.concatenate([rng.choice(M, 124, replace=False), rows]))   # the scaled rows included
    J = np.unique(np.concatenate([rng.choice(N, 124, replace=False), cols]))
    Ab, Bb = np.ascontiguousarray(A[I]), np.ascontiguousarray(B[:, J])
    ref = (Oracle.scheme2 if scheme == 2 else Oracle.scheme1)(Ab, Bb, S)["C"]
    blk = got[torch.from_numpy(I).cuda()][:, torch.from_numpy(J).cuda()].cpu().numpy()
    diff = blk.view(np.int64) != ref.view(np.int64)
    assert not diff.any(), f"{int(diff.sum())} of {diff.size} sampled entries differ from the oracle"
