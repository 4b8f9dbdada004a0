"""GPU: the sampled bound estimate.  A search that starts its candidate pools
from the j-th smallest block minimum of a strided database sample must return
exactly what the search without it returns, on benign data (the estimate
holds) and on data built so that it fails for chosen queries (those are
searched again).  Run with -m gpu on a B200."""
import numpy as np
import pytest

import oracle
from tests.knn_check import assert_knn_matches

pytestmark = pytest.mark.gpu

N, D, NQ = 1 << 20, 32, 8192
# (precision, k): k' = 416 for BF16/FP8 at k = 100, 320 for FP32-exact at k = 300;
# both shapes are large enough for the estimate to be used
CASES = [(1, 100), (2, 100), (0, 300)]


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


def mixture(rng, n, centers):
    c = centers[rng.integers(0, centers.shape[0], n)]
    return (c + rng.normal(0.0, 1.0, (n, D))).astype(np.float32)


def search_both(cb, ix, queries, k, precision):
    """(results with the estimate, results without, fallback count delta)."""
    before = ix.fallback_count()
    cb.set_bound_estimate(True)
    d1, i1 = ix.search_array(queries, k, precision=precision)
    delta = ix.fallback_count() - before
    cb.set_bound_estimate(False)
    d0, i0 = ix.search_array(queries, k, precision=precision)
    cb.set_bound_estimate(True)
    return (d1, i1), (d0, i0), delta


@pytest.mark.parametrize("precision,k", CASES)
def test_estimate_matches_plain_search(cb, res, precision, k):
    rng = np.random.default_rng(11 + precision)
    centers = rng.normal(0.0, 4.0, (512, D))
    base = mixture(rng, N, centers)
    queries = mixture(rng, NQ, centers)
    ix = cb.IndexBF(res, D, cb.IndexBFConfig(precision=precision, rerankFactor=4))
    ix.add(N, base)
    rows, step, r = ix.estimate_plan(NQ, k, precision)
    assert rows > 0 and rows % 256 == 0 and step >= 10 and 1 <= r, (rows, step, r)
    assert (rows - 1) * step < N
    (d1, i1), (d0, i0), delta = search_both(cb, ix, queries, k, precision)
    np.testing.assert_array_equal(i1, i0)
    np.testing.assert_array_equal(d1, d0)
    # a uniform sample fails a query with probability ~1e-6
    assert delta <= 4, delta
    check_sample(base, queries, d1, i1, rng.choice(NQ, 16, replace=False), k, precision)
    ix.close()


def check_sample(base, queries, got_d, got_i, sel, k, precision, min_recall=1.0):
    """Against the FP64 oracle: exact results for the exact form (and for BF16
    when min_recall is 1), else the recall of the coarse form's candidates."""
    rd, ri = oracle.knn(base, queries[sel], k + 1)
    if precision == 0 or (precision == 1 and min_recall >= 1.0):
        assert_knn_matches(base, queries[sel], got_d[sel], got_i[sel], rd, ri[:, :k])
    else:
        rec, _ = oracle.recall_at_k(base, queries[sel], got_i[sel], rd[:, :k])
        assert rec >= (0.5 if precision == 2 else min_recall), rec


@pytest.mark.parametrize("precision,k", CASES)
def test_estimate_failure_is_searched_again(cb, res, precision, k):
    """Every sample row (0, step, 2 step, ...) sits in a cluster at the origin and
    every other row in a cluster far away: for a query at the origin the j-th
    smallest block minimum of the sample admits about j < k' rows, so its
    estimate fails and it must be searched again; queries of the far cluster
    keep theirs."""
    rng = np.random.default_rng(23 + precision)
    ix = cb.IndexBF(res, D, cb.IndexBFConfig(precision=precision, rerankFactor=4))
    ix.add(N, rng.normal(0.0, 1.0, (N, D)).astype(np.float32))
    rows, step, r = ix.estimate_plan(NQ, k, precision)
    assert rows > 0
    # far enough that no far row passes a near query's estimate; the far
    # cluster's spread keeps its neighbours apart at BF16 precision (ulp 1/32 at 6)
    far = np.full(D, 6.0, np.float32)
    base = (far + rng.normal(0.0, 2.0, (N, D))).astype(np.float32)
    sample = np.arange(rows, dtype=np.int64) * step
    base[sample] = rng.normal(0.0, 0.5, (rows, D)).astype(np.float32)
    n_near = NQ // 2
    queries = np.concatenate([rng.normal(0.0, 0.5, (n_near, D)),
                              far + rng.normal(0.0, 2.0, (NQ - n_near, D))]).astype(np.float32)
    ix.reset()
    ix.add(N, base)
    assert ix.estimate_plan(NQ, k, precision) == (rows, step, r)
    (d1, i1), (d0, i0), delta = search_both(cb, ix, queries, k, precision)
    np.testing.assert_array_equal(i1, i0)
    np.testing.assert_array_equal(d1, d0)
    assert delta == n_near, (delta, n_near)
    sel = np.concatenate([rng.choice(n_near, 6, replace=False), n_near + rng.choice(NQ - n_near, 6, replace=False)])
    # the far cluster's offset costs the BF16 coarse pass accuracy (the folded
    # norms are exact, the rounded dot product is not): BF16 is held to recall
    check_sample(base, queries, d1, i1, sel, k, precision, min_recall=0.99)
    ix.close()


def test_estimate_switch(cb):
    cb.set_bound_estimate(False)
    assert cb.get_bound_estimate() is False
    cb.set_bound_estimate(True)
    assert cb.get_bound_estimate() is True


@pytest.mark.parametrize("precision,k", CASES)
def test_estimate_failure_checked_on_the_stream(cb, res, precision, k):
    """The same forced failures with queries and results in device memory (and
    the coarse check off): the check runs on the stream -- the whole pass runs
    again from no bound -- and the results still equal the search without the
    estimate; the failed queries are counted on the device."""
    import torch
    rng = np.random.default_rng(31 + precision)
    ix = cb.IndexBF(res, D, cb.IndexBFConfig(precision=precision, rerankFactor=4))
    ix.add(N, rng.normal(0.0, 1.0, (N, D)).astype(np.float32))
    rows, step, _ = ix.estimate_plan(NQ, k, precision)
    assert rows > 0
    far = np.full(D, 6.0, np.float32)
    base = (far + rng.normal(0.0, 2.0, (N, D))).astype(np.float32)
    base[np.arange(rows, dtype=np.int64) * step] = rng.normal(0.0, 0.5, (rows, D)).astype(np.float32)
    n_near = NQ // 2
    queries = np.concatenate([rng.normal(0.0, 0.5, (n_near, D)),
                              far + rng.normal(0.0, 2.0, (NQ - n_near, D))]).astype(np.float32)
    ix.reset()
    ix.add(N, base)
    qd = torch.tensor(queries, device="cuda")
    oi = torch.empty((NQ, k), dtype=torch.int32, device="cuda")
    od = torch.empty((NQ, k), dtype=torch.float32, device="cuda")
    st = torch.cuda.Stream()
    before = ix.fallback_count()
    cb.set_bound_estimate(True)
    ix.search_ex(NQ, qd, k, oi, od, precision, -1, stream=st)
    st.synchronize()
    delta = ix.fallback_count() - before
    cb.set_bound_estimate(False)
    d0, i0 = ix.search_array(queries, k, precision=precision)
    cb.set_bound_estimate(True)
    np.testing.assert_array_equal(oi.cpu().numpy(), i0)
    np.testing.assert_array_equal(od.cpu().numpy(), d0)
    assert delta == n_near, (delta, n_near)
    ix.close()
