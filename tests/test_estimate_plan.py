"""CPU: sizing of the sampled bound estimate (host logic, no device needed).

The plan is restated here from its model: a strided sample holding mu <= 12 of a
query's k' nearest rows on average, at most a tenth of the database's 256-row
tiles, none below mu = 8 or for N < 2^16 or N < 64 k'; the sample's 128-row
block minima below the query's k'-th distance are Binomial(B, 1 - (1 - k'/N)^128),
and the rank j is the smallest whose upper tail is <= 1e-6 (j <= B / 2)."""
import math

import pytest
from scipy.stats import binom

import curplsh_b200 as cb

SHAPES = [(10**6, 416), (10**6, 128), (10**6, 64), (10**7, 40), (10**7, 416), (5 * 10**6, 224),
          (5 * 10**6, 96), (2**20, 416), (2**20, 320), (65536, 128), (65535, 128), (50000, 100),
          (3 * 10**7, 4096), (2 * 10**6, 1024)]


def model(n, kp):
    if n < (1 << 16) or n < 64 * kp:
        return None
    T = -(-n // 256)
    tiles = min(math.ceil(12.0 * n / kp / 256), T // 10)
    if kp * tiles * 256 / n < 8.0:
        return None
    rows = tiles * 256
    return rows, n // rows, rows // 128, -math.expm1(128 * math.log1p(-kp / n))


@pytest.mark.parametrize("n,kp", SHAPES)
def test_plan_follows_the_model(n, kp):
    rows, step, j = cb.estimate_plan_shape(n, 10000, kp, 148)
    m = model(n, kp)
    if m is None:
        assert rows == 0
        return
    m_rows, m_step, blocks, q0 = m
    if rows == 0:  # only when no rank <= B/2 reaches the tail target
        assert binom.sf(blocks // 2 - 1, blocks, q0) > 1e-6
        return
    assert (rows, step) == (m_rows, m_step)
    assert rows % 256 == 0 and (rows - 1) * step < n  # every sample row exists
    assert 1 <= j <= blocks // 2
    # the smallest rank whose tail is <= 1e-6 (a relative slack for the two
    # independent evaluations of the binomial tail)
    assert binom.sf(j - 1, blocks, q0) <= 1e-6 * 1.001
    if j > 1:
        assert binom.sf(j - 2, blocks, q0) > 1e-6 * 0.999


def test_plan_independent_of_queries():
    assert cb.estimate_plan_shape(10**6, 1, 416) == cb.estimate_plan_shape(10**6, 10**6, 416)


def test_plan_rejects_bad_shapes():
    with pytest.raises(cb.CurplshError):
        cb.estimate_plan_shape(-1, 10, 100)
    with pytest.raises(cb.CurplshError):
        cb.estimate_plan_shape(10**6, 10, 100, num_sms=0)
