"""The host FP64 oracle, pinned against the reference's own known answers.

The reference ships no assertion-based tests; its two smoke programs print
outputs for fixed patterns (test/test_search.cpp:12-36, test/test_norm.cpp:9-22).
tests/golden/ref_smoke_patterns.npz holds their analytic answers (see
gen_golden.py); the oracle must reproduce them exactly.
"""
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _smoke():
    return np.load(os.path.join(GOLDEN, "ref_smoke_patterns.npz"))


def search_pattern_inputs(g):
    n, nq, d = int(g["search_n"]), int(g["search_nq"]), int(g["search_d"])
    base = np.repeat(np.minimum(np.arange(n), 10).astype(np.float32)[:, None], d, axis=1)
    queries = np.ones((nq, d), dtype=np.float32)
    return base, queries


def test_oracle_matches_reference_search_pattern():
    g = _smoke()
    base, queries = search_pattern_inputs(g)
    k = int(g["search_k"])
    dist, idx = oracle.knn(base, queries, k)
    np.testing.assert_array_equal(idx, g["search_idx"])
    np.testing.assert_array_equal(dist, g["search_dist_exact"])
    # the reference program itself prints the relative form (computeExactDistances=false)
    qn = oracle.l2_norms(queries)[:, None]
    np.testing.assert_array_equal(dist - qn, g["search_dist_relative"])


def test_search_pattern_expected_values():
    g = _smoke()
    # (1, 0, 2, 3, ..., 9) with the lower-index tie rule; 128*(m-1)^2 exact
    assert list(g["search_idx"][0]) == [1, 0, 2, 3, 4, 5, 6, 7, 8, 9]
    assert list(g["search_dist_exact"][0]) == [0, 128, 128, 512, 1152, 2048, 3200, 4608, 6272, 8192]
    assert list(g["search_dist_relative"][0]) == [-128, 0, 0, 384, 1024, 1920, 3072, 4480, 6144, 8064]


@pytest.mark.parametrize("shape_i", range(7))
def test_oracle_matches_reference_norm_pattern(shape_i):
    g = _smoke()
    num, dim = (int(v) for v in g["norm_shapes"][shape_i])
    norms = oracle.l2_norms(np.ones((num, dim), dtype=np.float32))
    np.testing.assert_array_equal(norms, np.full(num, float(dim)))


def test_oracle_random_fixture_regenerates():
    f = np.load(os.path.join(GOLDEN, "random_small.npz"))
    dist, idx = oracle.knn(f["base"], f["queries"], int(f["k"]) + 1)
    np.testing.assert_array_equal(idx, f["idx"])
    np.testing.assert_allclose(dist, f["dist"], rtol=0, atol=0)


def test_oracle_against_numpy_bruteforce():
    rng = np.random.default_rng(7)
    base = rng.standard_normal((500, 24)).astype(np.float32)
    queries = rng.standard_normal((13, 24)).astype(np.float32)
    k = 17
    dist, idx = oracle.knn(base, queries, k)
    full = ((queries.astype(np.float64)[:, None, :] - base.astype(np.float64)[None]) ** 2).sum(-1)
    for q in range(13):
        order = np.lexsort((np.arange(500), full[q]))[:k]
        np.testing.assert_array_equal(idx[q], order)
        np.testing.assert_allclose(dist[q], full[q][order], rtol=1e-12)


def test_oracle_tie_rule_lower_index_first():
    base = np.zeros((6, 4), dtype=np.float32)
    base[[1, 3, 4]] = 1.0  # rows 0,2,5 tie at distance 0 from the zero query
    dist, idx = oracle.knn(base, np.zeros((1, 4), np.float32), 5)
    assert list(idx[0]) == [0, 2, 5, 1, 3]
    assert list(dist[0]) == [0, 0, 0, 4, 4]


def test_oracle_k_larger_than_n_pads():
    base = np.arange(12, dtype=np.float32).reshape(3, 4)
    dist, idx = oracle.knn(base, base[:1], 5)
    assert list(idx[0]) == [0, 1, 2, -1, -1]
    assert dist[0, 3] == np.float32(np.finfo(np.float32).max)


def test_oracle_empty_database():
    # search.cu:94-101: FLT_MAX / -1 everywhere
    dist, idx = oracle.knn(np.zeros((0, 8), np.float32), np.ones((3, 8), np.float32), 4)
    assert (idx == -1).all()
    assert (dist == np.float32(np.finfo(np.float32).max)).all()


def test_ref_formula_model():
    rng = np.random.default_rng(3)
    base = rng.random((50, 32), dtype=np.float32)
    q = rng.random((4, 32), dtype=np.float32)
    qi = np.repeat(np.arange(4), 50)
    bi = np.tile(np.arange(50), 4)
    got = oracle.ref_formula(base, q, qi, bi)
    exact = oracle.exact_distances(base, q, qi, bi)
    np.testing.assert_allclose(got, exact, rtol=1e-4, atol=1e-4)


def test_recall_metric_is_tie_aware():
    base = np.zeros((6, 4), dtype=np.float32)
    base[[1, 3, 4]] = 1.0
    q = np.zeros((1, 4), np.float32)
    dist, idx = oracle.knn(base, q, 3)
    # any two of the tied rows {0,2,5} plus the third tie: still perfect recall
    r, _ = oracle.recall_at_k(base, q, np.array([[5, 0, 2]]), dist)
    assert r == 1.0
    r, _ = oracle.recall_at_k(base, q, np.array([[0, 1, 2]]), dist)
    assert abs(r - 2 / 3) < 1e-12
    r, _ = oracle.recall_at_k(base, q, np.array([[0, 0, 2]]), dist)  # duplicates are wrong
    assert r == 0.0
