"""Grouped Scheme II GEMM (oza_group_*): every problem's C is bit-identical to
the single-GEMM path (oza_gemm) on the same inputs, which is itself pinned to
the oracle and the reference; graph replay, direct launches, mixed slice
counts, pointer changes between calls and ragged shapes."""
import numpy as np
import pytest

import ozablas_b200 as oz
from oracle import Oracle

pytestmark = pytest.mark.gpu


def _problems(shapes, phi=1.0, seed=100):
    import torch
    As, Bs = [], []
    for i, (M, N, K) in enumerate(shapes):
        As.append(torch.from_numpy(oz.generate_matrix(M, K, phi, seed + 2 * i)).cuda())
        Bs.append(torch.from_numpy(oz.generate_matrix(K, N, phi, seed + 2 * i + 1)).cuda())
    return As, Bs


def _single(executor, A, B, S):
    import torch
    M, K = A.shape
    N = B.shape[1]
    C = torch.empty(M, N, dtype=torch.float64, device="cuda")
    oz.ozaki_scheme2_gemm(oz.WorkspaceScheme2(executor, M, N, K, S), A, B, C)
    return C


def _bits(t):
    return t.cpu().numpy().view(np.int64)


def _random_shapes(n, lo, hi, seed):
    rng = np.random.default_rng(seed)
    return [tuple(int(round(x)) for x in np.exp(rng.uniform(np.log(lo), np.log(hi), 3))) for _ in range(n)]


@pytest.mark.parametrize("graph", [True, False])
def test_group_matches_single_calls(executor, graph):
    import torch
    shapes = _random_shapes(24, 17, 700, seed=5) + [(1, 1, 1), (129, 257, 129), (300, 5, 1000)]
    S = 14
    As, Bs = _problems(shapes)
    Cs = [torch.full((M, N), float("nan"), dtype=torch.float64, device="cuda") for M, N, K in shapes]
    g = oz.GroupGemm(executor, shapes, S, graph=graph)
    assert g.info["graph"] == (1 if graph else 0)
    assert g.info["launches"] == 6
    for _ in range(2):   # capture + replay
        g(As, Bs, Cs)
    torch.cuda.synchronize()
    assert g.device_error() == 0
    for A, B, C in zip(As, Bs, Cs):
        assert np.array_equal(_bits(C), _bits(_single(executor, A, B, S)))


def test_group_mixed_slice_counts_and_wide_residues(executor):
    """Slice counts 17-20 at small K take the wide residue path (K_param > 62)."""
    import torch
    shapes = [(200, 300, 64), (64, 64, 2048), (130, 70, 33), (256, 512, 256), (90, 260, 500), (40, 40, 40)]
    slices = [20, 16, 8, 17, 12, 19]
    assert any(oz.scheme2_k_param(s, K) > 62 for s, (_, _, K) in zip(slices, shapes))
    As, Bs = _problems(shapes, phi=2.0, seed=300)
    Cs = [torch.empty(M, N, dtype=torch.float64, device="cuda") for M, N, K in shapes]
    g = oz.GroupGemm(executor, shapes, slices)
    assert g.info["launches"] == 3 + 3 * len(set(slices))
    g(As, Bs, Cs)
    torch.cuda.synchronize()
    for A, B, C, S in zip(As, Bs, Cs, slices):
        assert np.array_equal(_bits(C), _bits(_single(executor, A, B, S)))


def test_group_against_oracle(executor):
    import torch
    shapes = [(70, 90, 110), (128, 256, 128), (33, 257, 65)]
    As, Bs = _problems(shapes, phi=0.5, seed=7)
    Cs = [torch.empty(M, N, dtype=torch.float64, device="cuda") for M, N, K in shapes]
    oz.GroupGemm(executor, shapes, 9)(As, Bs, Cs)
    torch.cuda.synchronize()
    for A, B, C in zip(As, Bs, Cs):
        want = Oracle.scheme2(A.cpu().numpy(), B.cpu().numpy(), 9)["C"]
        assert np.array_equal(_bits(C), want.view(np.int64))


def test_group_pointer_change_between_replays(executor):
    import torch
    shapes = [(100, 120, 140), (64, 300, 90)]
    As1, Bs1 = _problems(shapes, seed=11)
    As2, Bs2 = _problems(shapes, seed=51)
    C1 = [torch.empty(M, N, dtype=torch.float64, device="cuda") for M, N, K in shapes]
    C2 = [torch.empty(M, N, dtype=torch.float64, device="cuda") for M, N, K in shapes]
    g = oz.GroupGemm(executor, shapes, 12)
    g(As1, Bs1, C1)
    g(As2, Bs2, C2)
    g(As1, Bs1, C1)
    torch.cuda.synchronize()
    for A, B, C in list(zip(As1, Bs1, C1)) + list(zip(As2, Bs2, C2)):
        assert np.array_equal(_bits(C), _bits(_single(executor, A, B, 12)))


def test_group_timings(executor):
    import torch
    shapes = _random_shapes(8, 64, 512, seed=9)
    As, Bs = _problems(shapes)
    Cs = [torch.empty(M, N, dtype=torch.float64, device="cuda") for M, N, K in shapes]
    t = oz.OzaTimings()
    oz.GroupGemm(executor, shapes, 10)(As, Bs, Cs, t)
    assert t.total_ms > 0 and t.step3_ms > 0
    assert abs(t.step1_ms + t.step2_ms + t.step3_ms + t.step4_ms - t.total_ms) < 0.05 * t.total_ms + 0.01


def test_group_argument_checks(executor):
    with pytest.raises(ValueError):
        oz.GroupGemm(executor, [(4, 0, 4)], 8)
    with pytest.raises(ValueError):
        oz.GroupGemm(executor, [(4, 4, 4)], 21)
    with pytest.raises(ValueError):
        oz.GroupGemm(executor, [], 8)
    g = oz.GroupGemm(executor, [(4, 4, 4)], 8)
    with pytest.raises(ValueError):
        g([], [], [])
