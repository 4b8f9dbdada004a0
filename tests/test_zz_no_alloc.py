"""The allocation-free search (curplsh_index_search_noalloc).

It serves callers that cannot allocate device memory while answering queries
(a process whose GPU memory belongs to another allocator, or a latency-critical
loop that must not hit cudaMalloc/cudaFree and their device-wide
synchronisation).  It must return the same neighbours as the regular search
while working out of the library's fixed scratch array.  This file is named to
be collected last, so a run that stops at the first failure has already run
every other test.
"""
import ctypes

import numpy as np
import pytest

from tests.knn_check import DIST_RTOL

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import curplsh_b200 as cb
    res = cb.DeviceResources(0)
    yield cb, torch, res
    res.close()


def _regular(cb, torch, ix, q, k):
    nq = q.shape[0]
    idx = torch.empty((nq, k), dtype=torch.int32, device="cuda")
    dist = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    ix.search_ex(nq, q, k, idx, dist)
    torch.cuda.synchronize()
    return idx.cpu().numpy(), dist.cpu().numpy()


def _noalloc_c_abi(cb, torch, ix, q, k):
    """Call the entry point through the C ABI directly (ctypes on the library)."""
    nq = q.shape[0]
    idx = torch.full((nq, k), -7, dtype=torch.int32, device="cuda")
    dist = torch.full((nq, k), -7.0, dtype=torch.float32, device="cuda")
    lib = ctypes.CDLL(cb.lib_path())
    fn = lib.curplsh_index_search_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_void_p]
    rc = fn(ix._h, nq, ctypes.c_void_p(q.data_ptr()), k, ctypes.c_void_p(idx.data_ptr()),
            ctypes.c_void_p(dist.data_ptr()), None)
    assert rc == 0, cb._lib.curplsh_last_error().decode()
    return idx.cpu().numpy(), dist.cpu().numpy()


@pytest.mark.parametrize("form", [0, 1, 2])
def test_noalloc_matches_regular_search_twice(env, form):
    cb, torch, res = env
    rng = np.random.default_rng(31 + form)
    base = torch.tensor(rng.standard_normal((20000, 96)).astype(np.float32)).cuda()
    queries = torch.tensor(rng.standard_normal((300, 96)).astype(np.float32)).cuda()
    k = 25
    ix = cb.IndexBF(res, 96, cb.IndexBFConfig(precision=form))
    ix.add(base.shape[0], base)
    ref_i, ref_d = _regular(cb, torch, ix, queries, k)  # also builds the FP8 copy for form 2
    for _ in range(2):  # the scratch keeps the previous call's contents: results must not depend on it
        got_i, got_d = _noalloc_c_abi(cb, torch, ix, queries, k)
        np.testing.assert_array_equal(got_i, ref_i)
        np.testing.assert_allclose(got_d, ref_d, rtol=DIST_RTOL, atol=0)
    ix.close()


def test_noalloc_after_a_different_shape(env):
    """A smaller call after a larger one reuses stale scratch contents safely."""
    cb, torch, res = env
    rng = np.random.default_rng(77)
    base = torch.tensor(rng.random((5000, 64), dtype=np.float32)).cuda()
    ix = cb.IndexBF(res, 64, cb.IndexBFConfig(precision=1))
    ix.add(5000, base)
    for nq, k in ((500, 100), (7, 3), (500, 100)):
        q = torch.tensor(rng.random((nq, 64), dtype=np.float32)).cuda()
        ref = _regular(cb, torch, ix, q, k)
        got = _noalloc_c_abi(cb, torch, ix, q, k)
        np.testing.assert_array_equal(got[0], ref[0])
        np.testing.assert_allclose(got[1], ref[1], rtol=DIST_RTOL, atol=0)
    ix.close()


def test_noalloc_rejects_oversized_requests(env):
    cb, torch, res = env
    base = torch.rand((3000, 32), device="cuda")
    ix = cb.IndexBF(res, 32, cb.IndexBFConfig(precision=1))
    ix.add(3000, base)
    nq, k = 60000, 1024  # candidate pools far beyond the fixed scratch
    q = torch.rand((nq, 32), device="cuda")
    idx = torch.empty((nq, k), dtype=torch.int32, device="cuda")
    dist = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    with pytest.raises(cb.CurplshError) as e:
        ix.search_noalloc(nq, q, k, idx, dist)
    assert e.value.code == cb.ERR_INVALID_ARG
    assert "scratch" in str(e.value)
    # host buffers would need staging memory: rejected
    qh = np.ones((4, 32), np.float32)
    with pytest.raises(cb.CurplshError):
        ix.search_noalloc(4, qh, 3, np.empty((4, 3), np.int32), np.empty((4, 3), np.float32))
    ix.close()
