"""FP8 row scales.  The FP8 copy takes one common scale when the nonzero rows'
own scales (max |x| / 448) lie within a factor 16 of each other, else one
scale per row; both must give the exact k nearest rows (coarse check on), and
all-zero rows (scale 0) must be handled."""
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
    yield cb, res
    res.close()


def _check(cb, res, base, queries, k):
    ix = cb.IndexBF(res, base.shape[1], cb.IndexBFConfig(precision=2))
    ix.add(base.shape[0], base)
    d, i = ix.search_array(queries, k)
    ix.close()
    rd, ri = oracle.knn(base, queries, k + 1)
    assert_knn_matches(base, queries, np.asarray(d), np.asarray(i), rd, ri)


@pytest.mark.parametrize("spread", [1.0, 4.0, 1000.0])
def test_fp8_rows_of_mixed_magnitude(env, spread):
    """Rows drawn at magnitudes 1 and `spread` (1 and 4: one common scale;
    1000: a scale per row), with a few all-zero rows."""
    cb, res = env
    rng = np.random.default_rng(int(spread) + 5)
    n, nq, d, k = 60000, 300, 96, 10
    base = rng.normal(0.0, 1.0, (n, d)).astype(np.float32)
    big = rng.random(n) < 0.5
    base[big] *= np.float32(spread)
    base[rng.choice(n, 7, replace=False)] = 0.0
    queries = base[rng.choice(n, nq, replace=False)] + rng.normal(0.0, 0.05, (nq, d)).astype(np.float32)
    _check(cb, res, base, queries.astype(np.float32), k)


def test_fp8_zero_query_and_zero_rows(env):
    cb, res = env
    rng = np.random.default_rng(3)
    n, d, k = 20000, 64, 5
    base = rng.normal(0.0, 1.0, (n, d)).astype(np.float32)
    base[:3] = 0.0
    queries = np.zeros((4, d), np.float32)
    queries[1:] = rng.normal(0.0, 1.0, (3, d))
    _check(cb, res, base, queries, k)
