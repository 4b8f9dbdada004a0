"""The coarse-margin check of the BF16/FP8 forms (merge pass + exact re-search).

The coarse forms choose k' candidates by BF16 or FP8-E4M3 distances; when the
data is finer than the form (FP8 on integer-valued rows in [0, 255]: a 3-bit
mantissa cannot order neighbours a few units apart), the check lists the
query and the search returns the FP32-exact answer for it instead."""
import importlib.util
import os

import numpy as np
import pytest

import oracle
from tests.knn_check import assert_knn_matches

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _synth():
    spec = importlib.util.spec_from_file_location("curplsh_synth", os.path.join(ROOT, "curplsh_b200", "synth.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="module")
def env():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import curplsh_b200 as cb
    res = cb.DeviceResources(0)
    yield cb, res
    cb.set_coarse_check(True)
    res.close()


def _search(cb, res, base, queries, k, form, which="coarse", rf=-1):
    """(distances, indices, queries searched again): by the coarse check, or
    (which="any") by the coarse check or the estimate's verification."""
    ix = cb.IndexBF(res, base.shape[1], cb.IndexBFConfig(precision=form))
    ix.add(base.shape[0], base)
    d, i = ix.search_array(queries, k, rerank_factor=rf)
    fb = ix.coarse_fallback_count() + (ix.fallback_count() if which == "any" else 0)
    ix.close()
    return d, i, fb


def test_fp8_on_integer_mixture_is_exact_with_the_check(env):
    """The 1M-row integer Gaussian mixture (its first 256 queries): ~1,000
    rows per cluster, so a query's 100th and 400th neighbours lie ~5,000
    apart while FP8's coarse error is ~10,000."""
    cb, res = env
    s = _synth()
    base, queries, _ = s.make("mixture_int_1m", q=256)
    k = 100
    rd, ri = oracle.knn(base, queries, k + 1)
    cb.set_coarse_check(True)
    # k' = 4k: FP8's coarse error swamps the gap between the 100th and 400th neighbours
    d8, i8, fb = _search(cb, res, base, queries, k, 2, which="any", rf=4)
    # the queries the coarse form cannot resolve are searched again (a query
    # whose estimate failed is listed by that check first)
    assert fb > 0, "FP8 on integer-valued rows should be searched again for some queries"
    assert_knn_matches(base, queries, d8, i8, rd, ri)
    de, ie, _ = _search(cb, res, base, queries, k, 0)
    np.testing.assert_array_equal(i8, ie)
    np.testing.assert_array_equal(d8, de)


def test_bf16_on_integer_mixture_never_falls_back(env):
    """BF16 represents integers up to 256 exactly: coarse = exact, margin always holds."""
    cb, res = env
    s = _synth()
    base, queries = s.mixture_int(200_000, 256)
    k = 100
    cb.set_coarse_check(True)
    d, i, fb = _search(cb, res, base, queries, k, 1)
    assert fb == 0
    rd, ri = oracle.knn(base, queries, k + 1)
    assert_knn_matches(base, queries, d, i, rd, ri)


def test_fp8_on_unit_sphere_mixture(env):
    """The unit-sphere mixture of the 10M-row workload (d = 96, k = 10, k' = 40) at N = 500,000."""
    cb, res = env
    s = _synth()
    base, queries = s.sphere_mixture(500_000, 256)
    k = 10
    rd, ri = oracle.knn(base, queries, k + 1)
    for on in (True, False):
        cb.set_coarse_check(on)
        d8, i8, fb = _search(cb, res, base, queries, k, 2)
        if on:
            assert_knn_matches(base, queries, d8, i8, rd, ri)
            assert fb < queries.shape[0] // 4, f"{fb} of {queries.shape[0]} queries fell back"
    cb.set_coarse_check(True)


def test_check_switch_and_data_finer_than_bf16(env):
    """Rows at 4 + N(0, 0.05^2): BF16 rounds every value by up to 1/64, so its
    coarse distances (error ~1) cannot order neighbours 0.01 apart, while the
    FP32-exact form resolves them.  With the check, BF16 returns the exact
    form's answer."""
    cb, res = env
    rng = np.random.default_rng(123)
    base = (4.0 + rng.standard_normal((60_000, 64)) * 0.05).astype(np.float32)
    queries = (4.0 + rng.standard_normal((200, 64)) * 0.05).astype(np.float32)
    k = 20
    rd, ri = oracle.knn(base, queries, k + 1)
    cb.set_coarse_check(True)
    assert cb.get_coarse_check()
    de, ie, _ = _search(cb, res, base, queries, k, 0)
    assert_knn_matches(base, queries, de, ie, rd, ri)
    d, i, fb = _search(cb, res, base, queries, k, 1)
    assert fb > 0
    assert_knn_matches(base, queries, d, i, rd, ri)
    np.testing.assert_array_equal(i, ie)
    cb.set_coarse_check(False)
    assert not cb.get_coarse_check()
    _, _, fb_off = _search(cb, res, base, queries, k, 1)
    assert fb_off == 0
    cb.set_coarse_check(True)
