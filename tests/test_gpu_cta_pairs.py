"""CTA pairs (clusters of two CTAs sharing one 256-row tcgen05 MMA over two
query blocks): the fused pass must return exactly what the single-CTA pass
returns, for every form, for odd and even query-block counts, for the batch
graph, and both must match the FP64 oracle."""
import numpy as np
import pytest

import oracle
from tests.knn_check import assert_knn_matches

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import curplsh_b200 as cb
    res = cb.DeviceResources(0)
    default = cb.get_cta_pairs()
    yield cb, res
    cb.set_cta_pairs(default)
    res.close()


def _bf16_values(rng, shape):
    import torch
    return torch.tensor(rng.standard_normal(shape, dtype=np.float32)).bfloat16().float().numpy()


def _search(cb, res, base, queries, k, form, pairs):
    cb.set_cta_pairs(pairs)
    ix = cb.IndexBF(res, base.shape[1], cb.IndexBFConfig(precision=form))
    ix.add(base.shape[0], base)
    d, i = ix.search_array(queries, k)
    ix.close()
    cb.set_cta_pairs(True)
    return np.asarray(d), np.asarray(i)


def test_switch_round_trips(env):
    cb, _ = env
    cb.set_cta_pairs(False)
    assert cb.get_cta_pairs() is False
    cb.set_cta_pairs(True)
    assert cb.get_cta_pairs() is True
    cb.set_cta_pairs("auto")
    assert cb.get_cta_pairs() == "auto"


# (rows, queries, dim, k): 8 query blocks; 17 blocks (the last group of two is
# half empty); 5 blocks (one odd block in five is too many: single CTAs either
# way); d = 96 and 64 (a streamed or narrow K tail)
@pytest.mark.parametrize("n,nq,d,k", [(30000, 1000, 128, 10), (60000, 2100, 96, 50), (20000, 600, 256, 100),
                                      (45000, 1024, 64, 20)])
@pytest.mark.parametrize("form", [0, 1, 2])
def test_pairs_match_single_cta(env, n, nq, d, k, form):
    cb, res = env
    rng = np.random.default_rng(1000 + n + form)
    base = _bf16_values(rng, (n, d))
    queries = _bf16_values(rng, (nq, d))
    d1, i1 = _search(cb, res, base, queries, k, form, pairs=False)
    d2, i2 = _search(cb, res, base, queries, k, form, pairs=True)
    np.testing.assert_array_equal(i1, i2)
    np.testing.assert_array_equal(d1, d2)
    sub = np.arange(0, nq, max(1, nq // 64))
    rd, ri = oracle.knn(base, queries[sub], k + 1)
    assert_knn_matches(base, queries[sub], d2[sub], i2[sub], rd, ri)


def test_pairs_in_the_batch_graph(env):
    """A batch over two indexes with several query batches each (the graph's
    fused launches run as CTA pairs) equals each search alone."""
    import torch
    cb, res = env
    rng = np.random.default_rng(7)
    dbs = []
    for n in (40000, 25000):
        data = _bf16_values(rng, (n, 128))
        ix = cb.IndexBF(res, 128, cb.IndexBFConfig(precision=1))
        ix.add(n, data)
        dbs.append((ix, data))
    items, expect = [], []
    for j, nq in enumerate((700, 300, 1100, 513)):
        ix, data = dbs[j % 2]
        q = torch.tensor(_bf16_values(rng, (nq, 128)), device="cuda")
        idx = torch.empty((nq, 10), dtype=torch.int32, device="cuda")
        dist = torch.empty((nq, 10), device="cuda")
        items.append((ix, q, 10, idx, dist))
        cb.set_cta_pairs(False)
        d_alone, i_alone = ix.search_array(q.cpu().numpy(), 10)
        expect.append((np.asarray(d_alone), np.asarray(i_alone)))
    cb.set_cta_pairs(True)
    batch = cb.SearchBatch(items, precision=1)
    batch.run()
    for (ix, q, k, idx, dist), (de, ie) in zip(items, expect):
        np.testing.assert_array_equal(idx.cpu().numpy(), ie)
        np.testing.assert_array_equal(dist.cpu().numpy(), de)
    batch.close()
    for ix, _ in dbs:
        ix.close()


@pytest.mark.parametrize("form,d", [(1, 384), (0, 256)])
def test_automatic_pairs_with_estimate(env, form, d):
    """The automatic mode pairs BF16 passes from d = 320 and FP32-exact passes
    from d = 192; with 70,000 rows the sampled bound estimate runs as well.
    Results equal the single-CTA pass and the oracle."""
    cb, res = env
    rng = np.random.default_rng(31 + d)
    n, nq, k = 70000, 1024, 10
    base = _bf16_values(rng, (n, d))
    queries = _bf16_values(rng, (nq, d))
    d1, i1 = _search(cb, res, base, queries, k, form, pairs=False)
    d2, i2 = _search(cb, res, base, queries, k, form, pairs="auto")
    np.testing.assert_array_equal(i1, i2)
    np.testing.assert_array_equal(d1, d2)
    sub = np.arange(0, nq, 16)
    rd, ri = oracle.knn(base, queries[sub], k + 1)
    assert_knn_matches(base, queries[sub], d2[sub], i2[sub], rd, ri)
