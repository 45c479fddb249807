"""Failure detection on the GPU without a fault: a bounded device wait that
nothing satisfies gives up after its limit, the kernel returns, the host reads
the error code, and the context keeps working (a GEMM afterwards is exact)."""
import numpy as np
import pytest

import ozablas_b200 as oz

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("limit_s", [0.05, 0.3])
def test_bounded_wait_expires_and_reports(executor, limit_s):
    code, elapsed = oz.selftest_wait_timeout(executor, limit_s)
    assert code == 1                       # kErrWaitTimeout
    assert limit_s <= elapsed < limit_s + 1.0


def test_context_usable_after_expired_wait(executor):
    import torch
    from oracle import Oracle
    oz.selftest_wait_timeout(executor, 0.05)
    A = oz.generate_matrix(96, 130, 0.5, 5)
    B = oz.generate_matrix(130, 70, 0.5, 6)
    ws = oz.WorkspaceScheme2(executor, 96, 70, 130, 8)
    C = torch.empty(96, 70, dtype=torch.float64, device="cuda")
    oz.ozaki_scheme2_gemm(ws, torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda(), C, oz.OzaTimings())
    assert ws.device_error() == 0
    want = Oracle.scheme2(A, B, 8)["C"]
    assert np.array_equal(C.cpu().numpy().view(np.int64), want.view(np.int64))


def test_selftest_rejects_bad_limits(executor):
    with pytest.raises(ValueError):
        oz.selftest_wait_timeout(executor, 0.0)
    with pytest.raises(ValueError):
        oz.selftest_wait_timeout(executor, 60.0)
