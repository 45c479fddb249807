"""Request loop with continuous batching (oza_server_*): each result is
bit-identical to oza_gemm on the same request alone, whatever it was batched
with; admission respects the workspace budget; concurrent submitters."""
import threading

import numpy as np
import pytest

import ozablas_b200 as oz

pytestmark = pytest.mark.gpu


def _req(M, N, K, phi, seed):
    import torch
    A = torch.from_numpy(oz.generate_matrix(M, K, phi, seed)).cuda()
    B = torch.from_numpy(oz.generate_matrix(K, N, phi, seed + 1)).cuda()
    C = torch.full((M, N), float("nan"), dtype=torch.float64, device="cuda")
    return A, B, C


def _alone(executor, A, B, S):
    import torch
    M, K = A.shape
    N = B.shape[1]
    C = torch.empty(M, N, dtype=torch.float64, device="cuda")
    oz.ozaki_scheme2_gemm(oz.WorkspaceScheme2(executor, M, N, K, S), A, B, C)
    torch.cuda.synchronize()
    return C


def _same(x, y):
    return np.array_equal(x.cpu().numpy().view(np.int64), y.cpu().numpy().view(np.int64))


def _mix(n, seed, lo=40, hi=700):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        M, N, K = (int(v) for v in np.exp(rng.uniform(np.log(lo), np.log(hi), 3)))
        out.append((M, N, K, int(rng.choice([8, 12, 16, 18, 20])), float(rng.choice([0.5, 2.0]))))
    return out


def test_results_identical_alone_and_in_the_mix(executor):
    reqs = _mix(30, seed=1)
    data = [_req(M, N, K, phi, 1000 + 2 * i) for i, (M, N, K, S, phi) in enumerate(reqs)]
    with oz.Server(executor, 2 << 30, max_inflight=2, max_batch=16) as srv:
        ids = [srv.submit(A, B, C, S) for (A, B, C), (_, _, _, S, _) in zip(data, reqs)]
        stats = [srv.wait(i, timeout=120) for i in ids]
        sst = srv.stats()
    assert sst["completed"] == len(reqs) and sst["queued"] == 0
    assert sst["max_batch_seen"] > 1           # requests really were batched
    assert sst["arena_peak"] <= 2 << 30
    for st in stats:
        assert st["status"] == 0 and st["submit_s"] <= st["admit_s"] <= st["done_s"]
    for (A, B, C), (_, _, _, S, _) in zip(data, reqs):
        assert _same(C, _alone(executor, A, B, S))


def test_budget_limits_admission(executor):
    """A budget that holds about one large request at a time: admission waits
    for memory, results stay exact, peak usage stays under the budget."""
    big = (700, 650, 900, 16)
    need = oz.Server.request_bytes(*big)
    budget = int(need * 1.5) + (8 << 20)
    data = [(_req(big[0], big[1], big[2], 0.5, 50 + 2 * i), big[3]) for i in range(5)]
    with oz.Server(executor, budget, max_inflight=3, max_batch=8) as srv:
        ids = [srv.submit(A, B, C, S) for (A, B, C), S in data]
        for i in ids:
            srv.wait(i, timeout=120)
        sst = srv.stats()
    assert sst["arena_peak"] <= budget
    assert sst["batches"] == 5                 # one request per batch: the budget admits one at a time
    for (A, B, C), S in data:
        assert _same(C, _alone(executor, A, B, S))


def test_request_over_budget_is_rejected(executor):
    import torch
    A = torch.zeros(2048, 2048, dtype=torch.float64, device="cuda")
    with oz.Server(executor, 64 << 20) as srv:
        with pytest.raises(MemoryError):
            srv.submit(A, A, A, 20)
        with pytest.raises(ValueError):
            srv.submit(A, A, A, 21)


def test_concurrent_submitters(executor):
    reqs = _mix(24, seed=7, lo=64, hi=400)
    data = [_req(M, N, K, phi, 5000 + 2 * i) for i, (M, N, K, S, phi) in enumerate(reqs)]
    errors = []
    with oz.Server(executor, 1 << 30, max_inflight=2, max_batch=8) as srv:
        def client(part):
            try:
                ids = [(j, srv.submit(*data[j], reqs[j][3])) for j in part]
                for j, i in ids:
                    srv.wait(i, timeout=120)
            except Exception as e:  # noqa: BLE001
                errors.append(e)
        threads = [threading.Thread(target=client, args=(range(k, len(reqs), 4),)) for k in range(4)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
    assert not errors
    for (A, B, C), (_, _, _, S, _) in zip(data, reqs):
        assert _same(C, _alone(executor, A, B, S))


def test_wait_timeout_then_completion(executor):
    A, B, C = _req(1536, 1536, 1536, 0.5, 77)
    with oz.Server(executor, 1 << 30) as srv:
        rid = srv.submit(A, B, C, 16)
        with pytest.raises(oz.OzaTimeoutError):
            srv.wait(rid, timeout=0.0)
        st = srv.wait(rid, timeout=120)
        assert st["status"] == 0 and st["slices"] == 16
    assert _same(C, _alone(executor, A, B, 16))


def _alone_scheme(executor, scheme, A, B, S):
    import torch
    M, K = A.shape
    N = B.shape[1]
    C = torch.empty(M, N, dtype=torch.float64, device="cuda")
    if scheme == 2:
        oz.ozaki_scheme2_gemm(oz.WorkspaceScheme2(executor, M, N, K, S), A, B, C)
    else:
        oz.ozaki_scheme1_gemm(oz.WorkspaceScheme1(executor, M, N, K, S), A, B, C)
    torch.cuda.synchronize()
    return C


def test_scheme_i_requests_in_the_mix(executor):
    """Requests for which the accuracy knob chose Scheme I run as batches of
    their own among batched Scheme II requests; every result equals its
    scheme's oza_gemm alone, bit for bit."""
    reqs = [(300, 200, 500, 2, 16), (257, 129, 1000, 1, 11), (90, 400, 300, 2, 18), (128, 256, 640, 2, 12),
            (500, 70, 2000, 1, 8), (64, 64, 64, 2, 20), (200, 300, 400, 1, 13), (330, 220, 110, 2, 9)]
    data = [_req(M, N, K, 2.0, 9000 + 2 * i) for i, (M, N, K, _, _) in enumerate(reqs)]
    with oz.Server(executor, 2 << 30, max_inflight=2, max_batch=8) as srv:
        ids = [srv.submit(A, B, C, S, scheme=sc) for (A, B, C), (_, _, _, sc, S) in zip(data, reqs)]
        stats = [srv.wait(i, timeout=120) for i in ids]
    for st, (_, _, _, sc, _) in zip(stats, reqs):
        assert st["status"] == 0
        if sc == 1:
            assert st["batch_size"] == 1
    for (A, B, C), (_, _, _, sc, S) in zip(data, reqs):
        assert _same(C, _alone_scheme(executor, sc, A, B, S)), (sc, S)
