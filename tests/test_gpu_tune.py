"""GPU tests of the launch-parameter table and the autotuner: every split and
pool headroom gives bit-identical results, which match the FP64 oracle."""
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


@pytest.mark.parametrize("precision,k", [(0, 10), (1, 100), (2, 32)])
def test_every_tuning_gives_identical_results(cb, res, precision, k):
    import torch
    rng = np.random.default_rng(7 + precision)
    n, nq, d = 60000, 300, 128
    base = rng.standard_normal((n, d), dtype=np.float32)
    q = rng.standard_normal((nq, d), dtype=np.float32)
    ix = cb.IndexBF(res, d, cb.IndexBFConfig(precision=precision))
    ix.add(n, base)
    qd = torch.tensor(q, device="cuda")
    ref_i = torch.empty((nq, k), dtype=torch.int32, device="cuda")
    ref_d = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    cb.tuning_clear()
    ix.search_ex(nq, qd, k, ref_i, ref_d, precision)
    torch.cuda.synchronize()
    if precision != 2:  # FP8 accuracy on unit-variance data is covered by the parity tests
        rd, ri = oracle.knn(base, q, k + 1)
        assert_knn_matches(base, q, ref_d.cpu().numpy(), ref_i.cpu().numpy(), rd, ri)
    oi = torch.empty_like(ref_i)
    od = torch.empty_like(ref_d)
    for split in (1, 2, 3, 8):
        for head in (128, 1024):
            cb.tuning_set(precision, d, k, nq, split, head)
            ix.search_ex(nq, qd, k, oi, od, precision)
            torch.cuda.synchronize()
            assert torch.equal(oi, ref_i) and torch.equal(od, ref_d), f"split {split} headroom {head}"
    cb.tuning_clear()
    ix.close()


def test_autotune_installs_and_caches(cb, res, tmp_path):
    import torch

    from curplsh_b200 import autotune
    rng = np.random.default_rng(11)
    base = rng.standard_normal((40000, 64), dtype=np.float32)
    ix = cb.IndexBF(res, 64, cb.IndexBFConfig(precision=1))
    ix.add(40000, base)
    qd = torch.tensor(rng.standard_normal((500, 64), dtype=np.float32), device="cuda")
    cb.tuning_clear()
    rec = autotune.tune(ix, qd, 10, reps=1)
    assert cb.tuning_get(1, 64, 10, 500) == (rec["split_q4"], rec["pool_headroom"])
    assert rec["ms"] <= rec["default_ms"]
    path = autotune.save([rec], str(tmp_path / "tune.json"))
    cb.tuning_clear()
    assert autotune.load(path) == 1
    assert cb.tuning_get(1, 64, 10, 500) == (rec["split_q4"], rec["pool_headroom"])
    cb.tuning_clear()
    ix.close()


def test_tuned_batch_matches_alone(cb, res):
    import torch

    from curplsh_b200 import autotune
    rng = np.random.default_rng(13)
    dbs = []
    for n, d in [(30000, 64), (12000, 256)]:
        x = rng.standard_normal((n, d), dtype=np.float32)
        ix = cb.IndexBF(res, d, cb.IndexBFConfig(precision=1))
        ix.add(n, x)
        dbs.append(ix)
    items = []
    for j, (nq, k) in enumerate([(200, 10), (37, 100), (900, 1), (5, 10)]):
        ix = dbs[j % 2]
        d = ix.getDimension()
        items.append((ix, torch.tensor(rng.standard_normal((nq, d), dtype=np.float32), device="cuda"), k,
                      torch.empty((nq, k), dtype=torch.int32, device="cuda"),
                      torch.empty((nq, k), dtype=torch.float32, device="cuda")))
    cb.tuning_clear()
    autotune.tune_batch(items, reps=1)
    batch = cb.SearchBatch(items)
    batch.run()
    cb.tuning_clear()
    for ix, q, k, oi, od in items:
        ai = torch.empty_like(oi)
        ad = torch.empty_like(od)
        ix.search_ex(q.shape[0], q, k, ai, ad, 1)
        torch.cuda.synchronize()
        assert torch.equal(ai, oi) and torch.equal(ad, od)
    batch.close()
    for ix in dbs:
        ix.close()
