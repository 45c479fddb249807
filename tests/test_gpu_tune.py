"""Accuracy tools on the GPU: the double-double block reference, the sampled
block error, and the slice-count autotuner (oza_block_error,
oza_autotune_slices), checked against the oracle's FP128 and double-double
GEMMs (the reference's accuracy oracle is FP128, utils/matrix_reference.hpp:22-50)."""
import numpy as np
import pytest

import ozablas_b200 as oz
from oracle import Oracle, error_metrics

pytestmark = pytest.mark.gpu


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x, np.float64)).cuda()


def _run(executor, scheme, A, B, S):
    import torch
    M, K = A.shape
    N = B.shape[1]
    ws_cls = oz.WorkspaceScheme2 if scheme == 2 else oz.WorkspaceScheme1
    fn = oz.ozaki_scheme2_gemm if scheme == 2 else oz.ozaki_scheme1_gemm
    ws = ws_cls(executor, M, N, K, S)
    dA, dB = _dev(A), _dev(B)
    dC = torch.empty((M, N), dtype=torch.float64, device="cuda")
    fn(ws, dA, dB, dC, oz.OzaTimings())
    return dC.cpu().numpy()


def test_block_error_of_exact_product_is_rounding_only(executor):
    """The DD reference agrees with the FP128 oracle to within one rounding."""
    A = oz.generate_matrix(70, 333, phi=2.0, seed=5)
    B = oz.generate_matrix(333, 50, phi=2.0, seed=6)
    C = Oracle.gemm_fp128(A, B)
    err = oz.block_error(executor, _dev(A), _dev(B), _dev(C), 70, 50, 333, block=1000, seed=1)
    assert err <= 2.0 ** -52


@pytest.mark.parametrize("scheme,S", [(2, 6), (2, 12), (1, 3), (1, 6)])
def test_block_error_covering_all_entries_matches_oracle(executor, scheme, S):
    """With a block covering every row and column, the sampled error is the
    full max relative error against the FP128 oracle (within a rounding of
    the reference value)."""
    M, N, K = 64, 48, 200
    A = oz.generate_matrix(M, K, phi=1.0, seed=11)
    B = oz.generate_matrix(K, N, phi=1.0, seed=12)
    C = _run(executor, scheme, A, B, S)
    want = error_metrics(Oracle.gemm_fp128(A, B), C)["max_rel"]
    got = oz.block_error(executor, _dev(A), _dev(B), _dev(C), M, N, K, block=max(M, N), seed=3)
    assert got == pytest.approx(want, rel=1e-6, abs=2.0 ** -52)


@pytest.mark.parametrize("scheme,S", [(2, 9), (1, 5)])
def test_gathered_block_reproduces_full_run_entries(executor, scheme, S):
    """The property the autotuner rests on: the pipeline on A[I,:] x B[:,J]
    returns exactly the (I, J) entries of the full run (shifts are per row of
    A and per column of B)."""
    M, N, K = 300, 260, 410
    A = oz.generate_matrix(M, K, phi=2.0, seed=21)
    B = oz.generate_matrix(K, N, phi=2.0, seed=22)
    A[7] *= 2.0 ** 200
    B[:, 3] *= 2.0 ** -150
    C = _run(executor, scheme, A, B, S)
    rng = np.random.default_rng(0)
    I = np.sort(rng.choice(M, 37, replace=False))
    J = np.sort(rng.choice(N, 29, replace=False))
    I[0], J[0] = 7, 3
    I.sort(); J.sort()
    Cb = _run(executor, scheme, A[I], B[:, J], S)
    assert np.array_equal(Cb.view(np.int64), C[np.ix_(I, J)].view(np.int64))


@pytest.mark.parametrize("scheme", [2, 1])
def test_autotune_meets_target_with_smallest_slices(executor, scheme):
    M, N, K = 512, 384, 1024
    A = oz.generate_matrix(M, K, phi=1.0, seed=31)
    B = oz.generate_matrix(K, N, phi=1.0, seed=32)
    exact = Oracle.gemm_fp128(A, B)
    target = 10.0 * error_metrics(exact, A @ B)["max_rel"]
    S, err = oz.autotune_slices(executor, scheme, _dev(A), _dev(B), M, N, K, target, block=128, seed=9)
    assert 1 <= S <= 20 and err <= target
    # the chosen S meets the target on the sampled block, S - 1 does not
    dA, dB = _dev(A), _dev(B)
    CS = _run(executor, scheme, A, B, S)
    assert oz.block_error(executor, dA, dB, _dev(CS), M, N, K, block=128, seed=9) == pytest.approx(err, abs=0)
    if S > 1:
        Cm = _run(executor, scheme, A, B, S - 1)
        assert oz.block_error(executor, dA, dB, _dev(Cm), M, N, K, block=128, seed=9) > target
    # and the full run at S is within an order of magnitude of the target
    assert error_metrics(exact, CS)["max_rel"] <= 10.0 * target


def test_autotune_unreachable_target_raises(executor):
    A = oz.generate_matrix(64, 64, phi=4.0, seed=41)
    B = oz.generate_matrix(64, 64, phi=4.0, seed=42)
    with pytest.raises(oz.OzaError, match="not reached"):
        oz.autotune_slices(executor, 2, _dev(A), _dev(B), 64, 64, 64, 1e-300, block=32)


def test_autotune_argument_checks(executor):
    A = _dev(np.ones((4, 4)))
    with pytest.raises(ValueError):
        oz.autotune_slices(executor, 3, A, A, 4, 4, 4, 1e-10)
    with pytest.raises(ValueError):
        oz.autotune_slices(executor, 2, A, A, 4, 4, 4, 0.0)
    with pytest.raises(ValueError):
        oz.block_error(executor, A, A, A, 4, 4, 4, block=0)


@pytest.mark.parametrize("K,phi,target", [(16384, 4.0, 1e-14), (140000, 1.0, 1e-12), (2048, 0.5, 1e-12)])
def test_autotune_scheme_choice(executor, K, phi, target):
    """oza_autotune_scheme takes Scheme II where its moduli meet the target on
    both sampled blocks, Scheme I where they do not -- for a wide exponent
    range with a tight target, and always beyond Scheme II's INT32 bound
    (K > 137438) -- and its count then meets the target on both blocks."""
    M, N = 128, 128
    A = oz.generate_matrix(M, K, phi=phi, seed=51)
    B = oz.generate_matrix(K, N, phi=phi, seed=52)
    dA, dB = _dev(A), _dev(B)
    scheme, S, err = oz.autotune_scheme(executor, dA, dB, M, N, K, target, block=64, seed=3)
    assert 1 <= S <= 20 and err <= target
    C = _run(executor, scheme, A, B, S)
    for sd in (3, 3 ^ 0x5bd1e995):
        assert oz.block_error(executor, dA, dB, _dev(C), M, N, K, block=64, seed=sd) <= target
    if K > 137438:
        assert scheme == 1
        return
    # Scheme II on the same two blocks decides which scheme is due
    def e2(S2):
        C2 = _run(executor, 2, A, B, S2)
        return max(oz.block_error(executor, dA, dB, _dev(C2), M, N, K, block=64, seed=sd)
                   for sd in (3, 3 ^ 0x5bd1e995))
    if e2(20) > target:
        assert scheme == 1
    elif e2(19) <= target:   # Scheme II below its cap: taken unless Scheme I is cheaper
        assert scheme == 2 or S * (S + 1) // 2 < 19
    # else Scheme II only at its cap, where the knob checks more blocks: either scheme


@pytest.mark.parametrize("K,phi", [(2048, 0.5), (16384, 4.0)])
def test_autotune_scheme_like_dgemm(executor, K, phi):
    """oza_autotune_scheme_like: the chosen count's error is at most native
    DGEMM's on each sampled block (the ratio it reports is <= 1), and at that
    count the scheme's result does meet DGEMM's error on the knob's first
    block."""
    import torch
    M, N = 128, 128
    A = oz.generate_matrix(M, K, phi=phi, seed=61)
    B = oz.generate_matrix(K, N, phi=phi, seed=62)
    dA, dB = _dev(A), _dev(B)
    D = torch.matmul(dA, dB)
    scheme, S, ratio = oz.autotune_scheme_like(executor, dA, dB, M, N, K, D, 1.0, block=64, seed=5)
    assert scheme in (1, 2) and 1 <= S <= 20 and ratio <= 1.0
    C = _run(executor, scheme, A, B, S)
    ours = oz.block_error(executor, dA, dB, _dev(C), M, N, K, block=64, seed=5)
    dgemm = oz.block_error(executor, dA, dB, D, M, N, K, block=64, seed=5)
    assert ours <= max(dgemm, 2.0 ** -53)


@pytest.mark.parametrize("phi", [0.5, 2.0, 4.0])
def test_estimate_phi(executor, phi):
    """oza_estimate_phi recovers the generator's phi from sampled rows and
    columns, and row/column scaling (which the step-1 shifts absorb) does not
    move it; the scheme lookup then takes the estimate."""
    M, N, K = 256, 192, 4096
    A = oz.generate_matrix(M, K, phi=phi, seed=71)
    B = oz.generate_matrix(K, N, phi=phi, seed=72)
    est = oz.estimate_phi(executor, _dev(A), _dev(B), M, N, K)
    assert abs(est - phi) <= 0.1 * phi
    A[3, :] *= 2.0 ** 300
    B[:, 5] *= 2.0 ** -300
    A[:, 7] = 0.0
    est2 = oz.estimate_phi(executor, _dev(A), _dev(B), M, N, K)
    assert abs(est2 - phi) <= 0.1 * phi
    scheme, S = oz.scheme_for_target(1e-12, K, est2)
    assert scheme in (1, 2) and 1 <= S <= 21
