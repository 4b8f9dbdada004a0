"""GPU tests of the batched search (one captured graph over several indexes):
every item must return exactly what the same search returns alone, and match
the FP64 oracle."""
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


def _bf16_values(rng, shape):
    """N(0,1) values rounded to BF16 and stored as FP32."""
    import torch
    return torch.tensor(rng.standard_normal(shape, dtype=np.float32)).bfloat16().float().numpy()


def _make_dbs(cb, res, rng, specs, precision):
    dbs = []
    for n, d in specs:
        data = _bf16_values(rng, (n, d))
        ix = cb.IndexBF(res, d, cb.IndexBFConfig(precision=precision))
        if n:
            ix.add(n, data)
        dbs.append((ix, data))
    return dbs


def _check_oracle(data, q, k, got_i, got_d):
    rd, ri = oracle.knn(data, q, k + 1)
    assert_knn_matches(data, q, got_d, got_i, rd, ri)


def _alone(ix, q, k, precision):
    import torch
    idx = torch.empty((q.shape[0], k), dtype=torch.int32, device="cuda")
    dist = torch.empty((q.shape[0], k), dtype=torch.float32, device="cuda")
    ix.search_ex(q.shape[0], q, k, idx, dist, precision)
    torch.cuda.synchronize()
    return idx.cpu().numpy(), dist.cpu().numpy()


@pytest.mark.parametrize("precision", [0, 1, 2])
def test_batch_matches_alone_and_oracle(cb, res, precision):
    import torch
    rng = np.random.default_rng(1234 + precision)
    specs = [(3000, 64), (20000, 128), (7000, 128), (1500, 256), (0, 64), (900, 100)]
    dbs = _make_dbs(cb, res, rng, specs, precision)
    sizes = [1, 300, 17, 129, 5, 64, 1, 250, 40, 3, 0, 77]
    ks = [1, 10, 100, 10, 1024, 1, 10, 100, 10, 1, 10, 50]
    items, host = [], []
    for j, (nq, k) in enumerate(zip(sizes, ks)):
        ix, data = dbs[j % len(dbs)]
        d = data.shape[1]
        q = _bf16_values(rng, (nq, d))
        qd = torch.tensor(q, device="cuda")
        idx = torch.full((nq, k), -7, dtype=torch.int32, device="cuda")
        dist = torch.full((nq, k), -7.0, dtype=torch.float32, device="cuda")
        items.append((ix, qd, k, idx, dist))
        host.append((q, data))
    batch = cb.SearchBatch(items, precision=precision)
    batch.run()
    launches, ws = batch.info()
    assert launches >= 3 and ws > 0
    for j, (ix, qd, k, idx, dist) in enumerate(items):
        if qd.shape[0] == 0:
            continue
        bi, bd = idx.cpu().numpy(), dist.cpu().numpy()
        ai, ad = _alone(ix, qd, k, precision)
        np.testing.assert_array_equal(bi, ai, err_msg=f"item {j}: indices differ from the search alone")
        np.testing.assert_array_equal(bd, ad, err_msg=f"item {j}: distances differ from the search alone")
        q, data = host[j]
        _check_oracle(data, q, k, bi, bd)
    # replay after overwriting the queries in place
    for j, (ix, qd, k, idx, dist) in enumerate(items):
        if qd.shape[0]:
            qd.copy_(torch.tensor(_bf16_values(rng, tuple(qd.shape)), device="cuda"))
    batch.run()
    for j, (ix, qd, k, idx, dist) in enumerate(items):
        if qd.shape[0] == 0:
            continue
        ai, ad = _alone(ix, qd, k, precision)
        np.testing.assert_array_equal(idx.cpu().numpy(), ai, err_msg=f"replay item {j}")
        np.testing.assert_array_equal(dist.cpu().numpy(), ad, err_msg=f"replay item {j}")
    batch.close()
    for ix, _ in dbs:
        ix.close()


def test_batch_replans_after_add(cb, res):
    import torch
    rng = np.random.default_rng(99)
    data = _bf16_values(rng, (5000, 128))
    ix = cb.IndexBF(res, 128, cb.IndexBFConfig(precision=1))
    ix.add(5000, data)
    q = torch.tensor(_bf16_values(rng, (33, 128)), device="cuda")
    idx = torch.empty((33, 10), dtype=torch.int32, device="cuda")
    dist = torch.empty((33, 10), dtype=torch.float32, device="cuda")
    batch = cb.SearchBatch([(ix, q, 10, idx, dist)])
    batch.run()
    more = _bf16_values(rng, (3000, 128))
    ix.add(3000, more)
    batch.run()
    full = np.concatenate([data, more])
    _check_oracle(full, q.cpu().numpy(), 10, idx.cpu().numpy(), dist.cpu().numpy())
    ai, ad = _alone(ix, q, 10, 1)
    np.testing.assert_array_equal(idx.cpu().numpy(), ai)
    batch.close()
    ix.close()


def test_batch_rejects_host_memory_and_mixed_args(cb, res):
    rng = np.random.default_rng(5)
    data = _bf16_values(rng, (1000, 64))
    ix = cb.IndexBF(res, 64, cb.IndexBFConfig())
    ix.add(1000, data)
    q = np.zeros((4, 64), np.float32)
    idx = np.zeros((4, 10), np.int32)
    dist = np.zeros((4, 10), np.float32)
    with pytest.raises(cb.CurplshError):
        cb.SearchBatch([(ix, q, 10, idx, dist)])
    import torch
    qd = torch.zeros((4, 64), device="cuda")
    with pytest.raises(cb.CurplshError):
        cb.SearchBatch([(ix, qd, 0, torch.zeros((4, 1), dtype=torch.int32, device="cuda"),
                         torch.zeros((4, 1), device="cuda"))])
    ix.close()
