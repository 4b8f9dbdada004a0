"""Shared parity assertions for the GPU tests (CUDA result vs the FP64 oracle)."""
import numpy as np

import oracle

FLT_MAX = np.float32(np.finfo(np.float32).max)

# Distances: the engine returns sum (q-x)^2 evaluated in FP32 after an exact
# rerank; the tolerance is relative 1e-4 (plus a tiny absolute floor for
# distances at or near zero).
DIST_RTOL = 1e-4
DIST_ATOL_FRAC = 1e-6   # of the mean squared norm scale
# Indices: strict positional equality wherever the oracle's neighbouring
# distances are separated by more than this (relative); tie-aware recall 1.0
# everywhere.
SEP_RTOL = 1e-5


def assert_knn_matches(base, queries, got_d, got_i, ref_d, ref_i, min_recall=1.0, strict=True):
    base = np.asarray(base, np.float32)
    queries = np.asarray(queries, np.float32)
    got_d = np.asarray(got_d, np.float64)
    got_i = np.asarray(got_i, np.int64)
    nq, k = got_i.shape
    ref_d = ref_d[:, :k + 1] if ref_d.shape[1] > k else ref_d
    ref_i = ref_i[:, :k]
    rk = ref_d[:, :k]
    scale = float(np.mean(np.sum(base.astype(np.float64) ** 2, 1))) if base.size else 1.0
    atol = DIST_ATOL_FRAC * max(scale, 1e-30)
    pad = ref_i < 0
    assert np.array_equal(got_i < 0, pad), "padding slots differ"
    assert (got_d[pad] == FLT_MAX).all(), "padding distances must be FLT_MAX"
    real = ~pad
    # distances at each rank
    err = np.abs(got_d[real] - rk[real])
    lim = DIST_RTOL * np.abs(rk[real]) + atol
    assert (err <= lim).all(), f"distance error max {err.max():.3e} (limit {lim[np.argmax(err - lim)]:.3e})"
    # returned distance belongs to the returned index
    qidx = np.repeat(np.arange(nq), k).reshape(nq, k)
    own = oracle.exact_distances(base, queries, qidx, got_i)
    e2 = np.abs(got_d[real] - own[real])
    assert (e2 <= DIST_RTOL * np.abs(own[real]) + atol).all(), "returned distance does not match its index"
    # ascending order
    for q in range(nq):
        row = got_d[q][real[q]]
        assert (np.diff(row) >= 0).all(), f"results of query {q} not sorted"
    # recall (tie-aware)
    rec, per = oracle.recall_at_k(base, queries, got_i, rk)
    assert rec >= min_recall, f"recall {rec:.6f} < {min_recall} (worst query {per.min():.3f})"
    if strict and min_recall >= 1.0:
        full = np.concatenate([ref_d, np.full((nq, max(0, k + 1 - ref_d.shape[1])), np.inf)], axis=1)[:, :k + 1]
        lo = np.concatenate([np.full((nq, 1), -np.inf), full[:, :k - 1]], axis=1)
        sep = ((full[:, :k] - lo) > SEP_RTOL * np.abs(full[:, :k])) & \
              ((full[:, 1:k + 1] - full[:, :k]) > SEP_RTOL * np.abs(full[:, :k]))
        sep &= real
        bad = sep & (got_i != ref_i)
        assert not bad.any(), f"{int(bad.sum())} well-separated positions differ, first at {np.argwhere(bad)[0]}"
    return rec


def assert_matches_reference(got_d, got_i, ref_d, ref_i, sep_rtol=SEP_RTOL, dist_rtol=DIST_RTOL):
    """Compare a result with the reference's own output (cuRPLSH
    searchL2Distance with exact distances), rank by rank.

    The reference computes ||q||^2 + ||x||^2 - 2 q.x in FP32 and breaks ties in
    no particular order, so: distances must agree within `dist_rtol` at every
    rank; indices must be equal wherever the reference's distance at that rank
    is separated from both neighbours by more than `sep_rtol` (relative); and,
    per query, the set of indices strictly inside the k-th distance's tie group
    (distance below kth * (1 - sep_rtol)) must be the same set.  Returns the
    number of positions compared strictly."""
    got_d = np.asarray(got_d, np.float64)
    got_i = np.asarray(got_i, np.int64)
    ref_d = np.asarray(ref_d, np.float64)
    ref_i = np.asarray(ref_i, np.int64)
    assert got_d.shape == ref_d.shape and got_i.shape == ref_i.shape, (got_d.shape, ref_d.shape)
    nq, k = ref_i.shape
    err = np.abs(got_d - ref_d)
    lim = dist_rtol * np.abs(ref_d) + 1e-6 * max(float(np.mean(np.abs(ref_d))), 1e-30)
    assert (err <= lim).all(), f"distance differs from the reference by {err.max():.3e} at {np.unravel_index(np.argmax(err - lim), err.shape)}"
    gap = sep_rtol * np.abs(ref_d)
    lo = np.concatenate([np.full((nq, 1), -np.inf), ref_d[:, :-1]], axis=1)
    hi = np.concatenate([ref_d[:, 1:], np.full((nq, 1), np.inf)], axis=1)
    sep = ((ref_d - lo) > gap) & ((hi - ref_d) > gap)
    # the last rank is compared only if it is separated from the reference's
    # (unknown) k+1-th distance, which the inside-set rule below covers instead
    sep[:, -1] = False
    bad = sep & (got_i != ref_i)
    assert not bad.any(), f"{int(bad.sum())} separated positions differ from the reference, first {np.argwhere(bad)[0]}"
    for q in range(nq):
        thr = ref_d[q, -1] * (1 - sep_rtol) if ref_d[q, -1] > 0 else -np.inf
        a = set(ref_i[q][ref_d[q] < thr].tolist())
        b = set(got_i[q][got_d[q] < thr].tolist())
        assert a == b, f"query {q}: indices inside the k-th distance differ from the reference ({sorted(a ^ b)[:5]})"
    return int(sep.sum())
