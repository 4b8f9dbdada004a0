"""Searches on one index from several host threads at once (each on its own
stream, plus two threads sharing a stream) return exactly what the same
searches return one after another; an add() waits for them."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import curplsh_b200 as cb
    res = cb.DeviceResources(0)
    yield cb, res
    res.close()


@pytest.mark.parametrize("form", [0, 1, 2])
def test_concurrent_searches_match_sequential(env, form):
    import torch
    cb, res = env
    rng = np.random.default_rng(40 + form)
    n, d, k, nq = 200_000, 96, 20, 1500
    base = rng.normal(0.0, 1.0, (n, d)).astype(np.float32)
    ix = cb.IndexBF(res, d, cb.IndexBFConfig(precision=form))
    ix.add(n, base)
    batches = [rng.normal(0.0, 1.0, (nq, d)).astype(np.float32) for _ in range(6)]
    expect = [ix.search_array(q, k) for q in batches]
    shared = torch.cuda.Stream()
    got = [None] * len(batches)
    errors = []

    def worker(i):
        try:
            # threads 0-3 on their own streams with device buffers (asynchronous
            # where the form allows), 4-5 on one shared stream
            st = shared if i >= 4 else torch.cuda.Stream()
            qd = torch.tensor(batches[i], device="cuda")
            oi = torch.empty((nq, k), dtype=torch.int32, device="cuda")
            od = torch.empty((nq, k), dtype=torch.float32, device="cuda")
            for _ in range(3):
                ix.search_ex(nq, qd, k, oi, od, stream=st)
            st.synchronize()
            got[i] = (od.cpu().numpy(), oi.cpu().numpy())
        except Exception as e:  # reported on the main thread
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(i,)) for i in range(len(batches))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for (d0, i0), (d1, i1) in zip(expect, got):
        np.testing.assert_array_equal(np.asarray(i0), i1)
        np.testing.assert_array_equal(np.asarray(d0), d1)
    ix.close()


def test_add_waits_for_searches(env):
    """An append while other threads search: every search sees either the old
    or the new database whole, and the final state equals one index built from
    both parts."""
    cb, res = env
    rng = np.random.default_rng(9)
    d, k = 64, 10
    a = rng.normal(0.0, 1.0, (50_000, d)).astype(np.float32)
    b = rng.normal(0.0, 1.0, (30_000, d)).astype(np.float32)
    q = rng.normal(0.0, 1.0, (700, d)).astype(np.float32)
    ix = cb.IndexBF(res, d, cb.IndexBFConfig(precision=0))
    ix.add(a.shape[0], a)
    old = ix.search_array(q, k)
    both = np.concatenate([a, b])
    ref = cb.IndexBF(res, d, cb.IndexBFConfig(precision=0))
    ref.add(both.shape[0], both)
    new = ref.search_array(q, k)
    ref.close()
    seen, errors = [], []

    def searcher():
        try:
            for _ in range(8):
                seen.append(ix.search_array(q, k))
        except Exception as e:
            errors.append(e)

    threads = [threading.Thread(target=searcher) for _ in range(2)]
    for t in threads:
        t.start()
    ix.add(b.shape[0], b)
    for t in threads:
        t.join()
    assert not errors, errors
    for dd, ii in seen:
        ok_old = np.array_equal(np.asarray(ii), np.asarray(old[1]))
        ok_new = np.array_equal(np.asarray(ii), np.asarray(new[1]))
        assert ok_old or ok_new
    np.testing.assert_array_equal(np.asarray(ix.search_array(q, k)[1]), np.asarray(new[1]))
    ix.close()
