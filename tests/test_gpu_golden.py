"""The sm_100a pipeline against the committed fixtures the reference itself
produced (tests/golden/pipeline_*.npz): every intermediate and C, bit for bit."""
import glob
import os

import numpy as np
import pytest

from tests.gpu_helpers import bits, run_pipeline

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "pipeline_*.npz"))),
                         ids=lambda p: os.path.basename(p)[9:-4])
def test_gpu_matches_reference_fixtures(executor, path):
    import ozablas_b200 as oz
    g = np.load(path)
    got = run_pipeline(oz, executor, int(g["scheme"]), g["A"], g["B"], int(g["S"]))
    for k in ("shift_A", "shift_B", "A_slices", "B_slices", "C_tc"):
        assert np.array_equal(got[k], g[k]), k
    assert np.array_equal(bits(got["C"]), bits(g["C"]))
