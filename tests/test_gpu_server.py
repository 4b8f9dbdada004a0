"""GPU tests of the serving loop: requests submitted concurrently from several
threads, in host and device memory, with mixed sizes and k, are batched on the
fly; every result must equal the same search alone and match the oracle."""
import threading

import numpy as np
import pytest

import oracle
from tests.knn_check import assert_knn_matches

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cb():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import curplsh_b200
    return curplsh_b200


@pytest.fixture(scope="module")
def res(cb):
    r = cb.DeviceResources(0)
    yield r
    r.close()


def _alone(ix, q, k, precision):
    import torch
    qd = torch.as_tensor(np.asarray(q.cpu() if hasattr(q, "cpu") else q), device="cuda")
    idx = torch.empty((qd.shape[0], k), dtype=torch.int32, device="cuda")
    dist = torch.empty((qd.shape[0], k), dtype=torch.float32, device="cuda")
    ix.search_ex(qd.shape[0], qd, k, idx, dist, precision)
    torch.cuda.synchronize()
    return idx.cpu().numpy(), dist.cpu().numpy()


@pytest.mark.parametrize("precision", [0, 1])
def test_server_results_equal_search_alone(cb, res, precision):
    import torch
    rng = np.random.default_rng(21 + precision)
    n, d = 40000, 128
    base = rng.standard_normal((n, d), dtype=np.float32)
    ix = cb.IndexBF(res, d, cb.IndexBFConfig(precision=precision))
    ix.add(n, base)
    srv = cb.Server(ix, max_inflight=3, max_step_queries=384, memory_budget=512 << 20)
    reqs = []
    for j in range(48):
        nq = int(np.exp(rng.uniform(0, np.log(256))))
        k = int(rng.choice([1, 10, 50, 100]))
        q = rng.standard_normal((nq, d), dtype=np.float32)
        if j % 3 == 0:  # device memory
            reqs.append((torch.tensor(q, device="cuda"), k, torch.empty((nq, k), dtype=torch.int32, device="cuda"),
                         torch.empty((nq, k), dtype=torch.float32, device="cuda"), q))
        else:  # host memory
            reqs.append((q, k, np.empty((nq, k), np.int32), np.empty((nq, k), np.float32), q))
    torch.cuda.synchronize()
    tickets = [None] * len(reqs)

    def submitter(lo):
        for j in range(lo, len(reqs), 2):
            q, k, oi, od, _ = reqs[j]
            tickets[j] = srv.submit(q, k, oi, od)

    th = [threading.Thread(target=submitter, args=(lo,)) for lo in (0, 1)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    lat = [srv.wait(t, timeout=60.0) for t in tickets]
    assert all(x >= 0 for x in lat)
    st = srv.stats()
    assert st["requests_done"] == len(reqs)
    assert st["steps"] >= 2 and st["peak_bytes_in_use"] <= 512 << 20
    for j, (q, k, oi, od, qh) in enumerate(reqs):
        gi = oi.cpu().numpy() if hasattr(oi, "cpu") else oi
        gd = od.cpu().numpy() if hasattr(od, "cpu") else od
        ai, ad = _alone(ix, qh, k, precision)
        np.testing.assert_array_equal(gi, ai, err_msg=f"request {j}: indices differ from the search alone")
        np.testing.assert_array_equal(gd, ad, err_msg=f"request {j}: distances differ from the search alone")
        if j % 6 == 0:
            rd, ri = oracle.knn(base, qh, k + 1)
            assert_knn_matches(base, qh, gd, gi, rd, ri)
    srv.close()
    ix.close()


def test_server_admission_by_memory(cb, res):
    """A tight budget admits at most two 64-query steps at a time (each needs
    ~72 MB of candidate pools); a request whose working memory alone exceeds
    the budget is rejected at submit."""
    rng = np.random.default_rng(3)
    n, d = 20000, 64
    base = rng.standard_normal((n, d), dtype=np.float32)
    ix = cb.IndexBF(res, d, cb.IndexBFConfig(precision=1))
    ix.add(n, base)
    srv = cb.Server(ix, max_inflight=4, max_step_queries=64, memory_budget=160 << 20)
    with pytest.raises(cb.CurplshError):
        big = rng.standard_normal((64, d), dtype=np.float32)
        srv.submit(big, 1024, np.empty((64, 1024), np.int32), np.empty((64, 1024), np.float32))
    reqs = []
    for _ in range(20):
        q = rng.standard_normal((64, d), dtype=np.float32)
        reqs.append((q, np.empty((64, 10), np.int32), np.empty((64, 10), np.float32)))
    ts = [srv.submit(q, 10, oi, od) for q, oi, od in reqs]
    for t in ts:
        srv.wait(t, timeout=60.0)
    st = srv.stats()
    assert st["requests_done"] == 20 and st["peak_bytes_in_use"] <= 160 << 20
    for q, oi, od in reqs[:3]:
        ai, ad = _alone(ix, q, 10, 1)
        np.testing.assert_array_equal(oi, ai)
        np.testing.assert_array_equal(od, ad)
    srv.close()
    ix.close()
