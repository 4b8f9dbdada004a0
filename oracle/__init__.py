"""Host FP64 brute-force kNN oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's ``cpu_baseline`` /
``--impl reference`` legs import this package.  The curplsh_b200 product never
does: its search path is the CUDA library, and it fails loudly when that
library is missing instead of falling back here.

The C restatement lives in ``knn_oracle.c`` (see its header for the reference
files and lines it follows).  This module loads ``libknn_oracle.so`` (built by
``build()``), and adds the tie-aware recall metric used by the parity tests.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libknn_oracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile knn_oracle.c into libknn_oracle.so (gcc + OpenMP)."""
    src = os.path.join(_HERE, "knn_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE, "libknn_oracle.so"])
    return _LIB_PATH


def _load():
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(_LIB_PATH)
        f32p = ctypes.POINTER(ctypes.c_float)
        f64p = ctypes.POINTER(ctypes.c_double)
        i64p = ctypes.POINTER(ctypes.c_int64)
        lib.oracle_knn.argtypes = [f32p, ctypes.c_int64, f32p, ctypes.c_int64, ctypes.c_int32,
                                   ctypes.c_int32, i64p, f64p, ctypes.c_int]
        lib.oracle_knn.restype = ctypes.c_int
        lib.oracle_l2_norms.argtypes = [f32p, ctypes.c_int64, ctypes.c_int32, f64p]
        lib.oracle_l2_norms.restype = None
        lib.oracle_ref_formula.argtypes = [f32p, f32p, ctypes.c_int32, i64p, i64p, ctypes.c_int64, f32p]
        lib.oracle_ref_formula.restype = None
        lib.oracle_num_threads.argtypes = []
        lib.oracle_num_threads.restype = ctypes.c_int
        _lib = lib
    return _lib


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr(a, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def num_threads() -> int:
    return int(_load().oracle_num_threads())


def l2_norms(x) -> np.ndarray:
    """Squared L2 norms of the rows of x, in FP64."""
    x = _f32(x)
    n, d = x.shape
    out = np.empty(n, dtype=np.float64)
    _load().oracle_l2_norms(_ptr(x, ctypes.c_float), n, d, _ptr(out, ctypes.c_double))
    return out


def knn(base, queries, k: int, threads: int = 0):
    """Exact kNN in FP64.  Returns (distances[nq,k] float64, indices[nq,k] int64),
    ascending by (distance, index); (-1, FLT_MAX) padding when k > N."""
    base = _f32(base)
    queries = _f32(queries)
    if base.ndim != 2 or queries.ndim != 2:
        raise ValueError("base and queries must be 2-D")
    n = base.shape[0]
    d = queries.shape[1]
    if n and base.shape[1] != d:
        raise ValueError("dimension mismatch")
    nq = queries.shape[0]
    idx = np.empty((nq, k), dtype=np.int64)
    dist = np.empty((nq, k), dtype=np.float64)
    rc = _load().oracle_knn(_ptr(base, ctypes.c_float), n, _ptr(queries, ctypes.c_float), nq, d, k,
                            _ptr(idx, ctypes.c_int64), _ptr(dist, ctypes.c_double), int(threads))
    if rc != 0:
        raise RuntimeError("oracle_knn failed")
    return dist, idx


def ref_formula(base, queries, qi, bi) -> np.ndarray:
    """The reference's FP32 distance formula ||q||^2 + (||x||^2 - 2 q.x) for pairs."""
    base = _f32(base)
    queries = _f32(queries)
    qi = np.ascontiguousarray(qi, dtype=np.int64)
    bi = np.ascontiguousarray(bi, dtype=np.int64)
    out = np.empty(qi.shape[0], dtype=np.float32)
    _load().oracle_ref_formula(_ptr(base, ctypes.c_float), _ptr(queries, ctypes.c_float), queries.shape[1],
                               _ptr(qi, ctypes.c_int64), _ptr(bi, ctypes.c_int64), qi.shape[0],
                               _ptr(out, ctypes.c_float))
    return out


def exact_distances(base, queries, qidx, bidx) -> np.ndarray:
    """FP64 squared distances of explicit (query, base) pairs; bidx < 0 gives inf."""
    base = np.asarray(base, dtype=np.float64)
    queries = np.asarray(queries, dtype=np.float64)
    qidx = np.asarray(qidx)
    bidx = np.asarray(bidx)
    out = np.full(bidx.shape, np.inf)
    ok = bidx >= 0
    diff = queries[qidx[ok]] - base[bidx[ok]]
    out[ok] = np.einsum("ij,ij->i", diff, diff)
    return out


def recall_at_k(base, queries, got_idx, ref_dist, rel_eps: float = 1e-6):
    """Tie-aware recall@k.

    Returned index j counts as a hit for query q when its FP64 distance is
    within (1 + rel_eps) of the oracle's k-th distance (so any member of a tie
    group straddling the k-th position is accepted), and indices are not
    repeated.  Returns (mean recall, per-query recall)."""
    got_idx = np.asarray(got_idx, dtype=np.int64)
    nq, k = got_idx.shape
    kth = ref_dist[:, k - 1]
    qidx = np.repeat(np.arange(nq), k).reshape(nq, k)
    d = exact_distances(base, queries, qidx, got_idx)
    tol = np.abs(kth) * rel_eps + 1e-12
    hit = (d <= (kth + tol)[:, None]) & (got_idx >= 0)
    # padding slots (oracle has -1 / FLT_MAX too) count as hits
    pad = (got_idx < 0) & (ref_dist >= np.finfo(np.float32).max)
    hit |= pad
    per = np.empty(nq)
    for q in range(nq):
        row = got_idx[q]
        valid = row[row >= 0]
        dup = valid.size != np.unique(valid).size
        per[q] = 0.0 if dup else hit[q].mean()
    return float(per.mean()), per


def well_separated(ref_dist, rel_gap: float) -> np.ndarray:
    """Mask of queries whose k-th and (k+1)-th oracle distances differ by more
    than rel_gap (relative) -- pass k+1 columns of ref_dist."""
    a = ref_dist[:, -2]
    b = ref_dist[:, -1]
    return (b - a) > rel_gap * np.maximum(np.abs(a), 1e-30)
