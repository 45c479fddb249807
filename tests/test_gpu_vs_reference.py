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
