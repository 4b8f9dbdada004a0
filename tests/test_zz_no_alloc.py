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


def test_noalloc_waits_for_an_async_fp8_build(env):
    """The FP8 copy is built by the index's first regular FP8 search, on that
    search's stream and without a host sync (device buffers, no estimate below
    2^16 rows).  A no-alloc call issued right after it on another stream (here
    the legacy default stream) must still read the finished copy."""
    cb, torch, res = env
    rng = np.random.default_rng(404)
    n, d, nq, k = 60000, 256, 400, 10
    base = torch.tensor(rng.standard_normal((n, d)).astype(np.float32)).cuda()
    queries = torch.tensor(rng.standard_normal((nq, d)).astype(np.float32)).cuda()
    ix = cb.IndexBF(res, d, cb.IndexBFConfig(precision=2))
    ix.add(n, base)
    side = torch.cuda.Stream()
    idx_a = torch.empty((nq, k), dtype=torch.int32, device="cuda")
    dist_a = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    ix.search_ex(nq, queries, k, idx_a, dist_a, stream=side)  # asynchronous: builds the FP8 copy on `side`
    got_i, got_d = _noalloc_c_abi(cb, torch, ix, queries, k)  # no host sync in between
    torch.cuda.synchronize()
    np.testing.assert_array_equal(got_i, idx_a.cpu().numpy())
    np.testing.assert_allclose(got_d, dist_a.cpu().numpy(), rtol=DIST_RTOL, atol=0)
    ix.close()


def test_noalloc_allocates_nothing(env):
    """After the first call on the device (which looks up the scratch array),
    calls of any shape leave the device's free memory unchanged."""
    cb, torch, res = env
    rng = np.random.default_rng(5)
    base = torch.tensor(rng.random((30000, 128), dtype=np.float32)).cuda()
    ix = cb.IndexBF(res, 128, cb.IndexBFConfig(precision=1))
    ix.add(30000, base)
    shapes = [(1, 1), (100, 10), (1000, 100), (37, 1024), (4096, 50)]
    bufs = []
    for nq, k in shapes:
        q = torch.tensor(rng.random((nq, 128), dtype=np.float32)).cuda()
        bufs.append((q, torch.empty((nq, k), dtype=torch.int32, device="cuda"),
                     torch.empty((nq, k), dtype=torch.float32, device="cuda"), k))
    ix.search_noalloc(bufs[0][0].shape[0], bufs[0][0], bufs[0][3], bufs[0][1], bufs[0][2])  # warm-up
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        for q, i, dd, k in bufs:
            ix.search_noalloc(q.shape[0], q, k, i, dd)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    ix.close()


def test_noalloc_concurrent_callers(env):
    """Two host threads, each on its own stream, call the entry point at once;
    calls on one device are serialised over the shared scratch, so each thread
    gets the same results as the regular search."""
    import threading
    cb, torch, res = env
    rng = np.random.default_rng(9)
    base = torch.tensor(rng.standard_normal((25000, 64)).astype(np.float32)).cuda()
    ix = cb.IndexBF(res, 64, cb.IndexBFConfig(precision=0))
    ix.add(25000, base)
    work = []
    for nq, k in ((700, 32), (333, 7)):
        q = torch.tensor(rng.standard_normal((nq, 64)).astype(np.float32)).cuda()
        work.append((q, k, _regular(cb, torch, ix, q, k)))
    errors = []

    def run(q, k, ref):
        try:
            s = torch.cuda.Stream()
            i = torch.empty((q.shape[0], k), dtype=torch.int32, device="cuda")
            dd = torch.empty((q.shape[0], k), dtype=torch.float32, device="cuda")
            for _ in range(5):
                i.fill_(-3)
                s.wait_stream(torch.cuda.current_stream())
                ix.search_noalloc(q.shape[0], q, k, i, dd, stream=s)
                np.testing.assert_array_equal(i.cpu().numpy(), ref[0])
                np.testing.assert_allclose(dd.cpu().numpy(), ref[1], rtol=DIST_RTOL, atol=0)
        except Exception as e:  # noqa: BLE001  (reported by the main thread)
            errors.append(e)

    threads = [threading.Thread(target=run, args=w) for w in work]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    ix.close()
