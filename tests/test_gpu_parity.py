"""GPU parity: every stage of the sm_100a pipeline against the CPU oracle,
bit for bit (shifts, INT8 slices/residues, INT32 products, FP64 C), on seeded
inputs and on the edge cases the reference's arithmetic has."""
import numpy as np
import pytest

from tests.gpu_helpers import bits, run_pipeline

pytestmark = pytest.mark.gpu


def _oz():
    import ozablas_b200 as oz
    return oz


def _check_all(got, ref):
    assert np.array_equal(got["shift_A"], ref["shift_A"]), "shift_A"
    assert np.array_equal(got["shift_B"], ref["shift_B"]), "shift_B"
    assert np.array_equal(got["A_slices"], ref["A_slices"]), "A slices"
    assert np.array_equal(got["B_slices"], ref["B_slices"]), "B slices"
    if "C_tc" in got:
        assert np.array_equal(got["C_tc"], ref["C_tc"]), "INT32 products"
    diff = bits(got["C"]) != bits(ref["C"])
    assert not diff.any(), f"C differs in {int(diff.sum())} entries"


def _padding_zero(got):
    """The K padding of every real row of the A and B^T planes is zero (it
    enters the sums); rows past M and N are left unwritten, since the products
    they feed are never read."""
    i = got["ws"].info
    M, N, K = i["M"], i["N"], i["K"]
    assert not got["A_planes"][:, :M, K:].any()
    assert not got["B_planes"][:, :N, K:].any()


@pytest.mark.parametrize("S", [1, 2, 3, 4, 5, 7, 8, 9, 11, 12, 13, 15, 16, 17, 18, 20])
def test_scheme2_stages_bitexact(executor, S):
    oz = _oz()
    from oracle import Oracle
    A = oz.generate_matrix(160, 256, 0.5, 42)
    B = oz.generate_matrix(256, 300, 0.5, 43)
    got = run_pipeline(oz, executor, 2, A, B, S)
    _check_all(got, Oracle.scheme2(A, B, S))
    _padding_zero(got)


@pytest.mark.parametrize("S", [1, 2, 3, 5, 8, 10, 13])
def test_scheme1_stages_bitexact(executor, S):
    oz = _oz()
    from oracle import Oracle
    A = oz.generate_matrix(130, 200, 1.0, 42)
    B = oz.generate_matrix(200, 260, 1.0, 43)
    got = run_pipeline(oz, executor, 1, A, B, S)
    _check_all(got, Oracle.scheme1(A, B, S))
    _padding_zero(got)


@pytest.mark.parametrize("scheme,S", [(2, 8), (2, 16), (1, 6)])
@pytest.mark.parametrize("shape", [(1, 1, 1), (7, 5, 3), (129, 257, 129), (64, 33, 1000), (300, 17, 64)])
def test_ragged_shapes(executor, scheme, S, shape):
    oz = _oz()
    from oracle import Oracle
    M, N, K = shape
    A = oz.generate_matrix(M, K, 2.0, 11)
    B = oz.generate_matrix(K, N, 2.0, 12)
    got = run_pipeline(oz, executor, scheme, A, B, S)
    ref = Oracle.scheme2(A, B, S) if scheme == 2 else Oracle.scheme1(A, B, S)
    _check_all(got, ref)


@pytest.mark.parametrize("scheme,S", [(2, 8), (2, 19), (1, 7)])
def test_exponent_edge_cases(executor, scheme, S):
    """All-zero rows/columns, exact zeros, subnormals, powers of two, values just
    below a power of two, rows and columns scaled by 2^+-300."""
    oz = _oz()
    from oracle import Oracle
    M, N, K = 96, 80, 128
    A = oz.generate_matrix(M, K, 4.0, 5)
    B = oz.generate_matrix(K, N, 4.0, 6)
    rng = np.random.default_rng(1234)
    A[rng.random(A.shape) < 0.05] = 0.0
    B[rng.random(B.shape) < 0.05] = 0.0
    A[3, :] = 0.0
    B[:, 7] = 0.0
    A[1, :] *= 2.0 ** 300
    A[5, :] *= 2.0 ** -300
    B[:, 17] *= 2.0 ** 300
    B[:, 33] *= 2.0 ** -300
    A[9, :] = np.ldexp(1.0, np.arange(K) % 9 - 4)
    A[10, :] = np.nextafter(np.ldexp(1.0, np.arange(K) % 5), 0.0)
    A[11, :] = 5e-324 * (np.arange(K) + 1)          # subnormals
    B[:, 40] = -2.2250738585072014e-308 * np.arange(K)
    got = run_pipeline(oz, executor, scheme, A, B, S)
    ref = Oracle.scheme2(A, B, S) if scheme == 2 else Oracle.scheme1(A, B, S)
    _check_all(got, ref)


def test_1024_cubed_8_moduli_vs_oracle(executor):
    """1024^3, phi = 0.5, Scheme II with 8 moduli, bit-exact end to end."""
    oz = _oz()
    from oracle import Oracle
    A = oz.generate_matrix(1024, 1024, 0.5, 42)
    B = oz.generate_matrix(1024, 1024, 0.5, 43)
    got = run_pipeline(oz, executor, 2, A, B, 8)
    _check_all(got, Oracle.scheme2(A, B, 8))


def test_repeat_calls_identical(executor):
    """Workspaces are reusable: a second call gives identical results."""
    import torch
    oz = _oz()
    A = oz.generate_matrix(256, 384, 0.5, 1)
    B = oz.generate_matrix(384, 512, 0.5, 2)
    ws = oz.WorkspaceScheme2(executor, 256, 512, 384, 12)
    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    c1 = torch.empty(256, 512, dtype=torch.float64, device="cuda")
    c2 = torch.empty_like(c1)
    oz.ozaki_scheme2_gemm(ws, dA, dB, c1)
    oz.ozaki_scheme2_gemm(ws, dA, dB, c2)
    torch.cuda.synchronize()
    assert torch.equal(c1.view(torch.int64), c2.view(torch.int64))
    assert ws.device_error() == 0


@pytest.mark.parametrize("S", [1, 3, 4, 5, 8, 9, 12, 13, 16, 17, 20])
@pytest.mark.parametrize("shape", [(160, 300, 256), (7, 5, 3), (129, 257, 129), (300, 17, 64), (256, 512, 1000)])
def test_scheme2_fused_epilogue_bitexact(executor, S, shape):
    """Scheme II with the CRT inside the GEMM epilogue: C bit-exact vs the oracle."""
    oz = _oz()
    from oracle import Oracle
    M, N, K = shape
    A = oz.generate_matrix(M, K, 1.0, 21)
    B = oz.generate_matrix(K, N, 1.0, 22)
    got = run_pipeline(oz, executor, 2, A, B, S, materialize=False)
    assert "C_tc" not in got
    _check_all(got, Oracle.scheme2(A, B, S))


@pytest.mark.parametrize("S", [8, 16])
def test_scheme2_fused_equals_materialized(executor, S):
    oz = _oz()
    A = oz.generate_matrix(640, 384, 2.0, 31)
    B = oz.generate_matrix(384, 700, 2.0, 32)
    fused = run_pipeline(oz, executor, 2, A, B, S, materialize=False)
    mat = run_pipeline(oz, executor, 2, A, B, S, materialize=True)
    assert np.array_equal(bits(fused["C"]), bits(mat["C"]))


def test_scheme2_fused_edge_cases(executor):
    oz = _oz()
    from oracle import Oracle
    M, N, K = 96, 80, 128
    A = oz.generate_matrix(M, K, 4.0, 5)
    B = oz.generate_matrix(K, N, 4.0, 6)
    A[3, :] = 0.0
    B[:, 7] = 0.0
    A[1, :] *= 2.0 ** 300
    B[:, 33] *= 2.0 ** -300
    A[11, :] = 5e-324 * (np.arange(K) + 1)
    for S in (8, 19):
        got = run_pipeline(oz, executor, 2, A, B, S, materialize=False)
        _check_all(got, Oracle.scheme2(A, B, S))


@pytest.mark.parametrize("scheme,S", [(2, 16), (1, 5)])
def test_gemm_configurations_are_bit_identical(executor, scheme, S):
    """Every step-3 configuration (rasterisation band, wait hint, overlapped
    stages) gives the same bits; the autotuner keeps one of them."""
    import torch
    import ozablas_b200 as oz
    M, N, K = 700, 520, 900
    A = torch.from_numpy(oz.generate_matrix(M, K, 1.0, 1)).cuda()
    B = torch.from_numpy(oz.generate_matrix(K, N, 1.0, 2)).cuda()
    W = (oz.WorkspaceScheme2 if scheme == 2 else oz.WorkspaceScheme1)(executor, M, N, K, S)
    gemm = oz.ozaki_scheme2_gemm if scheme == 2 else oz.ozaki_scheme1_gemm
    ref = torch.empty(M, N, dtype=torch.float64, device="cuda")
    gemm(W, A, B, ref)
    for band, hint in ((8, 0), (32, 0), (16, 200), (1, 0)):
        W.set_gemm_config(band=band, wait_hint_ns=hint)
        C = torch.empty_like(ref)
        gemm(W, A, B, C)
        assert torch.equal(C.view(torch.int64), ref.view(torch.int64)), (band, hint)
    if scheme == 2:
        for chunks in (1, 2, 3, 16):   # steps in order and overlapped stages: same bits
            W.set_gemm_config(overlap_chunks=chunks)
            for _ in range(3):
                C = torch.full_like(ref, float("nan"))
                gemm(W, A, B, C)
                assert torch.equal(C.view(torch.int64), ref.view(torch.int64)), chunks
    W.set_gemm_config()
    cfg, ms = W.autotune_gemm(A, B, torch.empty_like(ref))
    assert ms > 0 and W.get_gemm_config() == cfg
    with pytest.raises(ValueError):
        W.set_gemm_config(band=-1)


@pytest.mark.parametrize("scheme,S", [(2, 7), (2, 16), (2, 19), (1, 4)])
def test_all_zero_chunks_bit_exact(executor, scheme, S):
    """Chunks whose values are all zero (padding, zero rows, zeroed blocks,
    -0.0) skip the residue arithmetic; every stage stays bit-identical."""
    oz = _oz()
    from oracle import Oracle
    M, N, K = 300, 270, 400
    A = oz.generate_matrix(M, K, 1.0, 61)
    B = oz.generate_matrix(K, N, 1.0, 62)
    A[5] = 0.0
    A[:, 16:48] = 0.0
    A[40:60, 200:216] = -0.0
    A[7, 3] = -0.0
    B[:, 9] = 0.0
    B[128:256, 100:140] = 0.0
    B[300:, :] = 0.0
    got = run_pipeline(oz, executor, scheme, A, B, S)
    ref = (Oracle.scheme2 if scheme == 2 else Oracle.scheme1)(A, B, S)
    _check_all(got, ref)
    _padding_zero(got)


def test_scheme1_split_groups_vs_oracle(executor):
    """Scheme I at K = 65536, S = 9: the groups of 8 and 9 slice pairs are
    split over two INT32 planes each (at most 7 pairs per plane keep every
    INT32 sum exact) and added exactly in step 4; C, shifts and slices equal
    the oracle's, which accumulates each group in one INT32 as the reference
    does (random data: no overflow)."""
    oz = _oz()
    from oracle import Oracle
    M, N, K, S = 32, 48, 65536, 9
    A = oz.generate_matrix(M, K, 1.0, 7)
    B = oz.generate_matrix(K, N, 1.0, 8)
    got = run_pipeline(oz, executor, 1, A, B, S)
    assert got["ws"].info["groups"] == 11
    ref = Oracle.scheme1(A, B, S)
    assert np.array_equal(got["shift_A"], ref["shift_A"])
    assert np.array_equal(got["shift_B"], ref["shift_B"])
    assert np.array_equal(got["A_slices"], ref["A_slices"])
    assert np.array_equal(got["B_slices"], ref["B_slices"])
    # group g's planes add up to the oracle's INT32 group plane
    first = [0, 1, 2, 3, 4, 5, 6, 7, 9, 11]
    for g in range(S):
        summed = got["C_tc"][first[g]:first[g + 1]].astype(np.int64).sum(axis=0)
        assert np.array_equal(summed, ref["C_tc"][g].astype(np.int64))
    assert np.array_equal(bits(got["C"]), bits(ref["C"]))
