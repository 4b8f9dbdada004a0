"""GPU: the sampled bound estimate inside a captured batch graph and inside the
serving loop.  There the estimate is verified on the device, and a fallback
chain enqueued behind each fused launch (bounds reset, the launch and its
merges again without the estimate) runs only when some query of that launch
failed.  On data built so that the estimate fails for half the queries, and
on benign data, every result must equal the same search alone (which
re-searches failed queries from the host)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, D = 1 << 20, 32


@pytest.fixture(scope="module")
def cb():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import curplsh_b200
    # these tests compare paths that differ only in the estimate: the coarse
    # check (host searches only) stays off so that it cannot tell them apart
    curplsh_b200.set_coarse_check(False)
    yield curplsh_b200
    curplsh_b200.set_bound_estimate(True)
    curplsh_b200.set_coarse_check(True)


@pytest.fixture(scope="module")
def res(cb):
    r = cb.DeviceResources(0)
    yield r
    r.close()


def _forced_failure_index(cb, res, rng, nq, k, precision):
    """Every sample row of the estimate sits in a cluster at the origin, every
    other row in a cluster far away: a query at the origin finds its j-th
    block minimum admitting fewer than k' rows, so its estimate fails."""
    ix = cb.IndexBF(res, D, cb.IndexBFConfig(precision=precision))
    ix.add(N, rng.normal(0.0, 1.0, (N, D)).astype(np.float32))
    rows, step, r = ix.estimate_plan(nq, k, precision)
    assert rows > 0
    far = np.full(D, 6.0, np.float32)
    base = (far + rng.normal(0.0, 2.0, (N, D))).astype(np.float32)
    base[np.arange(rows, dtype=np.int64) * step] = rng.normal(0.0, 0.5, (rows, D)).astype(np.float32)
    n_near = nq // 2
    queries = np.concatenate([rng.normal(0.0, 0.5, (n_near, D)),
                              far + rng.normal(0.0, 2.0, (nq - n_near, D))]).astype(np.float32)
    ix.reset()
    ix.add(N, base)
    return ix, queries, n_near


def _alone(ix, q, k, precision):
    import torch
    qd = torch.as_tensor(q, device="cuda")
    idx = torch.empty((q.shape[0], k), dtype=torch.int32, device="cuda")
    dist = torch.empty((q.shape[0], k), dtype=torch.float32, device="cuda")
    ix.search_ex(q.shape[0], qd, k, idx, dist, precision)
    torch.cuda.synchronize()
    return idx.cpu().numpy(), dist.cpu().numpy()


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_graph_with_failing_estimates(cb, res, precision):
    import torch
    rng = np.random.default_rng(41 + precision)
    k = 300 if precision == 0 else 100
    nq = 2048
    ix, queries, n_near = _forced_failure_index(cb, res, rng, nq, k, precision)
    before = ix.fallback_count()
    ref_i, ref_d = _alone(ix, queries, k, precision)
    assert ix.fallback_count() - before == n_near  # the host path saw the failures
    # two requests against the failing index (one fused item) and one against
    # a small index that uses no estimate
    small = cb.IndexBF(res, D, cb.IndexBFConfig(precision=precision))
    sdata = rng.normal(0.0, 1.0, (5000, D)).astype(np.float32)
    small.add(5000, sdata)
    sq = rng.normal(0.0, 1.0, (37, D)).astype(np.float32)
    halves = [queries[:nq // 4 * 3], queries[nq // 4 * 3:]]
    items = []
    for q, index, kk in ((halves[0], ix, k), (halves[1], ix, k), (sq, small, 10)):
        items.append((index, torch.as_tensor(q, device="cuda"), kk,
                      torch.full((q.shape[0], kk), -5, dtype=torch.int32, device="cuda"),
                      torch.full((q.shape[0], kk), -5.0, dtype=torch.float32, device="cuda")))
    batch = cb.SearchBatch(items, precision=precision)
    for _ in range(2):  # the graph replays: the failure counts start at zero every time
        batch.run()
        got_i = np.concatenate([items[0][3].cpu().numpy(), items[1][3].cpu().numpy()])
        got_d = np.concatenate([items[0][4].cpu().numpy(), items[1][4].cpu().numpy()])
        np.testing.assert_array_equal(got_i, ref_i)
        np.testing.assert_array_equal(got_d, ref_d)
        si, sd = _alone(small, sq, 10, precision)
        np.testing.assert_array_equal(items[2][3].cpu().numpy(), si)
        np.testing.assert_array_equal(items[2][4].cpu().numpy(), sd)
    batch.close()
    # benign queries (no failure): the fallback chain is skipped, same results
    far_q = queries[n_near:]
    ref2 = _alone(ix, far_q, k, precision)
    it2 = [(ix, torch.as_tensor(far_q, device="cuda"), k,
            torch.empty((far_q.shape[0], k), dtype=torch.int32, device="cuda"),
            torch.empty((far_q.shape[0], k), dtype=torch.float32, device="cuda"))]
    b2 = cb.SearchBatch(it2, precision=precision)
    b2.run()
    np.testing.assert_array_equal(it2[0][3].cpu().numpy(), ref2[0])
    np.testing.assert_array_equal(it2[0][4].cpu().numpy(), ref2[1])
    b2.close()
    small.close()
    ix.close()


def test_server_with_failing_estimates(cb, res):
    rng = np.random.default_rng(77)
    k, precision = 100, 1
    nq = 1024
    ix, queries, n_near = _forced_failure_index(cb, res, rng, nq, k, precision)
    ref_i, ref_d = _alone(ix, queries, k, precision)
    srv = cb.Server(ix, precision=precision, max_inflight=2, max_step_queries=1024, memory_budget=2 << 30)
    cuts = [0, 100, 612, 700, nq]
    outs = []
    for a, b in zip(cuts[:-1], cuts[1:]):
        oi = np.empty((b - a, k), np.int32)
        od = np.empty((b - a, k), np.float32)
        t = srv.submit(np.ascontiguousarray(queries[a:b]), k, oi, od)
        outs.append((t, oi, od))
    got_i = []
    got_d = []
    for t, oi, od in outs:
        srv.wait(t, timeout=120.0)
        got_i.append(oi)
        got_d.append(od)
    srv.close()
    np.testing.assert_array_equal(np.concatenate(got_i), ref_i)
    np.testing.assert_array_equal(np.concatenate(got_d), ref_d)
    ix.close()
