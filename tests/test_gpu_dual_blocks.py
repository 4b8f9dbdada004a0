"""Dual query blocks (two resident query blocks per CTA, each 128-row database
tile feeding two 128 x 128 tcgen05 MMAs; used by the FP8 form): the fused pass
must return exactly what the one-block pass returns, for odd and even
query-block counts and for the batch graph, and match the FP64 oracle.  The
other forms must be unaffected by the switch."""
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
    default = cb.get_dual_blocks()
    yield cb, res
    cb.set_dual_blocks(default)
    res.close()


def _bf16_values(rng, shape):
    import torch
    return torch.tensor(rng.standard_normal(shape, dtype=np.float32)).bfloat16().float().numpy()


def _search(cb, res, base, queries, k, form, dual):
    cb.set_dual_blocks(dual)
    ix = cb.IndexBF(res, base.shape[1], cb.IndexBFConfig(precision=form))
    ix.add(base.shape[0], base)
    d, i = ix.search_array(queries, k)
    ix.close()
    cb.set_dual_blocks(True)
    return np.asarray(d), np.asarray(i)


def test_switch_round_trips(env):
    cb, _ = env
    cb.set_dual_blocks(False)
    assert cb.get_dual_blocks() is False
    cb.set_dual_blocks(True)
    assert cb.get_dual_blocks() is True


# (rows, queries, dim, k): 8 query blocks; 17 blocks (the last group of two is
# half empty); 5 blocks (one odd block in five is too many: one block per CTA
# either way); d = 96 and 64
@pytest.mark.parametrize("n,nq,d,k", [(30000, 1000, 128, 10), (60000, 2100, 96, 50), (20000, 600, 256, 100),
                                      (45000, 1024, 64, 20)])
@pytest.mark.parametrize("form", [0, 1, 2])
def test_dual_matches_single_block(env, n, nq, d, k, form):
    cb, res = env
    rng = np.random.default_rng(1000 + n + form)
    base = _bf16_values(rng, (n, d))
    queries = _bf16_values(rng, (nq, d))
    d1, i1 = _search(cb, res, base, queries, k, form, dual=False)
    d2, i2 = _search(cb, res, base, queries, k, form, dual=True)
    np.testing.assert_array_equal(i1, i2)
    np.testing.assert_array_equal(d1, d2)
    sub = np.arange(0, nq, max(1, nq // 64))
    rd, ri = oracle.knn(base, queries[sub], k + 1)
    assert_knn_matches(base, queries[sub], d2[sub], i2[sub], rd, ri)


def test_dual_in_the_batch_graph(env):
    """An FP8 batch over two indexes with several query batches each: the
    graph planned with dual blocks returns exactly what the graph planned
    without them returns."""
    import torch
    cb, res = env
    rng = np.random.default_rng(7)
    dbs = []
    for n in (40000, 25000):
        data = _bf16_values(rng, (n, 128))
        ix = cb.IndexBF(res, 128, cb.IndexBFConfig(precision=2))
        ix.add(n, data)
        dbs.append(ix)
    queries = [torch.tensor(_bf16_values(rng, (nq, 128)), device="cuda") for nq in (700, 300, 1100, 513)]
    outs = []
    for dual in (False, True):
        cb.set_dual_blocks(dual)
        items = []
        for j, q in enumerate(queries):
            idx = torch.empty((q.shape[0], 10), dtype=torch.int32, device="cuda")
            dist = torch.empty((q.shape[0], 10), device="cuda")
            items.append((dbs[j % 2], q, 10, idx, dist))
        batch = cb.SearchBatch(items, precision=2)
        batch.run()
        outs.append([(it[3].cpu().numpy(), it[4].cpu().numpy()) for it in items])
        batch.close()
    cb.set_dual_blocks(True)
    for (i0, d0), (i1, d1) in zip(outs[0], outs[1]):
        np.testing.assert_array_equal(i0, i1)
        np.testing.assert_array_equal(d0, d1)
    for ix in dbs:
        ix.close()
