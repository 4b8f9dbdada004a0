"""GPU test of the shard merge kernel (curplsh_merge_shard_results): a
database split into shards, each searched on its own, merges to the same
top-k as one search over the whole database."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cb():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import curplsh_b200
    return curplsh_b200


@pytest.mark.parametrize("k,cuts", [(10, [0, 7000, 7001, 20000]), (100, [0, 50, 12000, 20000]),
                                    (1024, [0, 300, 900, 20000])])
def test_shard_merge_equals_single_search(cb, k, cuts):
    import torch
    rng = np.random.default_rng(k)
    n, nq, d = cuts[-1], 97, 64
    base = rng.standard_normal((n, d), dtype=np.float32)
    q = torch.tensor(rng.standard_normal((nq, d), dtype=np.float32), device="cuda")
    res = cb.DeviceResources(0)
    full = cb.IndexBF(res, d, cb.IndexBFConfig(precision=0))
    full.add(n, base)
    ri = torch.empty((nq, k), dtype=torch.int32, device="cuda")
    rd = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    full.search_ex(nq, q, k, ri, rd, 0)
    G = len(cuts) - 1
    gd = torch.empty((G, nq, k), dtype=torch.float32, device="cuda")
    gi = torch.empty((G, nq, k), dtype=torch.int32, device="cuda")
    shards = []
    for s in range(G):
        ix = cb.IndexBF(res, d, cb.IndexBFConfig(precision=0))
        ix.add(cuts[s + 1] - cuts[s], base[cuts[s]:cuts[s + 1]])
        ix.search_ex(nq, q, k, gi[s], gd[s], 0)
        shards.append(ix)
    bases = torch.tensor(cuts[:-1], dtype=torch.int64, device="cuda")
    oi = torch.empty((nq, k), dtype=torch.int32, device="cuda")
    od = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    cb.merge_shard_results(gd, gi, bases, oi, od)
    torch.cuda.synchronize()
    assert torch.equal(oi, ri), "indices differ from the single search"
    assert torch.equal(od, rd), "distances differ from the single search"
    for ix in shards:
        ix.close()
    full.close()
    res.close()
