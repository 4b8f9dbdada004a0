"""GPU parity: the CUDA path (through the C ABI) against the FP64 oracle and
the reference's known-answer patterns.  Run with -m gpu on a B200."""
import os

import numpy as np
import pytest

import oracle
from tests.knn_check import FLT_MAX, assert_knn_matches

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
FORMS = [0, 1, 2]  # FP32-exact, BF16+rerank, FP8+rerank


@pytest.fixture(scope="module")
def cb():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import curplsh_b200
    return curplsh_b200


@pytest.fixture(scope="module")
def res(cb):
    r = cb.DeviceResources(0)
    yield r
    r.close()


def make_index(cb, res, data, precision=0, **kw):
    ix = cb.IndexBF(res, data.shape[1], cb.IndexBFConfig(precision=precision, **kw))
    if data.shape[0]:
        ix.add(data.shape[0], data)
    return ix


# ---------------------------------------------------------------- golden patterns
def test_reference_search_pattern(cb, res):
    """test/test_search.cpp:12-36 through IndexBF (exact distances, index_bf.cpp:68-69)."""
    g = np.load(os.path.join(GOLDEN, "ref_smoke_patterns.npz"))
    n, nq, d, k = (int(g[f"search_{s}"]) for s in "n nq d k".split())
    base = np.repeat(np.minimum(np.arange(n), 10).astype(np.float32)[:, None], d, axis=1)
    queries = np.ones((nq, d), np.float32)
    for form in FORMS:
        ix = make_index(cb, res, base, precision=form)
        dist, idx = ix.search_array(queries, k)
        np.testing.assert_array_equal(idx, g["search_idx"], err_msg=f"form {form}")
        np.testing.assert_array_equal(dist, g["search_dist_exact"].astype(np.float32), err_msg=f"form {form}")
        ix.close()


def test_reference_search_pattern_relative_form(cb, res):
    """The smoke program's own call: searchL2Distance(..., computeExactDistances=false)."""
    import torch
    g = np.load(os.path.join(GOLDEN, "ref_smoke_patterns.npz"))
    n, nq, d, k = (int(g[f"search_{s}"]) for s in "n nq d k".split())
    base = torch.tensor(np.repeat(np.minimum(np.arange(n), 10).astype(np.float32)[:, None], d, axis=1)).cuda()
    queries = torch.ones((nq, d), dtype=torch.float32, device="cuda")
    idx = torch.empty((nq, k), dtype=torch.int32, device="cuda")
    dist = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    cb.search_l2_distance(res, base, None, queries, k, idx, dist, exact_distances=False)
    np.testing.assert_array_equal(idx.cpu().numpy(), g["search_idx"])
    np.testing.assert_array_equal(dist.cpu().numpy(), g["search_dist_relative"].astype(np.float32))


@pytest.mark.parametrize("shape_i", range(7))
def test_reference_norm_pattern(cb, shape_i):
    """test/test_norm.cpp:15-22: all-ones rows have squared norm == dim."""
    import torch
    g = np.load(os.path.join(GOLDEN, "ref_smoke_patterns.npz"))
    num, dim = (int(v) for v in g["norm_shapes"][shape_i])
    x = torch.ones((num, dim), dtype=torch.float32, device="cuda")
    out = torch.empty(num, dtype=torch.float32, device="cuda")
    cb.compute_l2_norm(x, out, squared=True)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), np.full(num, dim, np.float32))
    cb.compute_l2_norm(x, out, squared=False)
    torch.cuda.synchronize()
    np.testing.assert_allclose(out.cpu().numpy(), np.full(num, np.sqrt(dim), np.float32), rtol=1e-6)


def test_l2_norm_random_vs_oracle(cb):
    import torch
    rng = np.random.default_rng(11)
    x = rng.standard_normal((1000, 96)).astype(np.float32)
    out = torch.empty(1000, dtype=torch.float32, device="cuda")
    cb.compute_l2_norm(torch.tensor(x).cuda(), out, squared=True)
    torch.cuda.synchronize()
    np.testing.assert_allclose(out.cpu().numpy(), oracle.l2_norms(x), rtol=2e-6)


# ---------------------------------------------------------------- random fixture
@pytest.mark.parametrize("form", FORMS)
def test_random_fixture(cb, res, form):
    f = np.load(os.path.join(GOLDEN, "random_small.npz"))
    k = int(f["k"])
    ix = make_index(cb, res, f["base"], precision=form)
    dist, idx = ix.search_array(f["queries"], k)
    assert_knn_matches(f["base"], f["queries"], dist, idx, f["dist"], f["idx"])


# ---------------------------------------------------------------- shapes and edges
SHAPES = [
    # (n, nq, d, k)
    (1, 1, 8, 1),
    (5, 3, 16, 10),        # k > n: (-1, FLT_MAX) padding
    (255, 127, 32, 7),
    (257, 129, 64, 64),
    (1000, 200, 96, 10),
    (3000, 130, 100, 33),  # d not a multiple of 8
    (4097, 300, 128, 100),
    (2000, 50, 256, 1),
    (2500, 150, 160, 20),  # FP8 norm tail in the second K chunk (byte 160)
    (1200, 90, 200, 12),   # FP8 norm tail at byte 224 (the last step of chunk 2)
    (1500, 64, 512, 200),
    (600, 10, 1000, 5),    # very high d: query chunks stream with the database
]


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "n%d_q%d_d%d_k%d" % s)
def test_shapes_vs_oracle(cb, res, shape, form):
    n, nq, d, k = shape
    rng = np.random.default_rng(hash(shape) % 2**32)
    base = rng.standard_normal((n, d)).astype(np.float32)
    queries = rng.standard_normal((nq, d)).astype(np.float32)
    ix = make_index(cb, res, base, precision=form)
    dist, idx = ix.search_array(queries, k)
    rd, ri = oracle.knn(base, queries, k + 1)
    assert_knn_matches(base, queries, dist, idx, rd, ri)


def test_integer_data_ties(cb, res):
    """Integer-valued data (the c1 distribution in miniature): many exact ties,
    resolved by lower row index -- must match the oracle position by position."""
    rng = np.random.default_rng(5)
    cent = rng.integers(0, 4, size=(8, 32)).astype(np.float32)
    base = cent[rng.integers(0, 8, 3000)] + rng.integers(-1, 2, size=(3000, 32))
    queries = cent[rng.integers(0, 8, 70)] + rng.integers(-1, 2, size=(70, 32))
    base = base.astype(np.float32)
    queries = queries.astype(np.float32)
    rd, ri = oracle.knn(base, queries, 50)
    for form in FORMS:
        ix = make_index(cb, res, base, precision=form)
        dist, idx = ix.search_array(queries, 50)
        np.testing.assert_array_equal(idx, ri, err_msg=f"form {form}")
        np.testing.assert_array_equal(dist, rd.astype(np.float32), err_msg=f"form {form}")


def test_empty_database(cb, res):
    ix = cb.IndexBF(res, 16)
    dist, idx = ix.search_array(np.ones((4, 16), np.float32), 3)
    assert (idx == -1).all() and (dist == FLT_MAX).all()


def test_k_limits(cb, res):
    ix = make_index(cb, res, np.random.default_rng(0).random((50, 8), dtype=np.float32))
    with pytest.raises(cb.CurplshError):
        ix.search_array(np.ones((1, 8), np.float32), 1025)
    with pytest.raises(cb.CurplshError):
        ix.search_array(np.ones((1, 8), np.float32), 0)


def test_k1024(cb, res):
    rng = np.random.default_rng(9)
    base = rng.standard_normal((5000, 64)).astype(np.float32)
    queries = rng.standard_normal((20, 64)).astype(np.float32)
    rd, ri = oracle.knn(base, queries, 1025)
    for form in FORMS:
        ix = make_index(cb, res, base, precision=form)
        dist, idx = ix.search_array(queries, 1024)
        assert_knn_matches(base, queries, dist, idx, rd, ri)


def test_device_and_host_pointers_agree(cb, res):
    import torch
    rng = np.random.default_rng(2)
    base = rng.random((3000, 64), dtype=np.float32)
    queries = rng.random((77, 64), dtype=np.float32)
    ix = make_index(cb, res, base)
    d_h, i_h = ix.search_array(queries, 12)
    dq = torch.tensor(queries).cuda()
    d_d, i_d = ix.search_array(dq, 12)
    np.testing.assert_array_equal(i_h, i_d.cpu().numpy())
    np.testing.assert_array_equal(d_h, d_d.cpu().numpy())
    # device database rows, borrowed (the reference's aliasing) and copied
    xb = torch.tensor(base).cuda()
    for borrow in (False, True):
        ix2 = cb.IndexBF(res, 64, cb.IndexBFConfig(borrowDeviceData=borrow))
        ix2.add(3000, xb)
        d2, i2 = ix2.search_array(queries, 12)
        np.testing.assert_array_equal(i_h, i2)
        np.testing.assert_array_equal(d_h, d2)


def test_append_and_reset(cb, res):
    rng = np.random.default_rng(4)
    base = rng.standard_normal((2500, 48)).astype(np.float32)
    queries = rng.standard_normal((40, 48)).astype(np.float32)
    ix = cb.IndexBF(res, 48)
    ix.add(1000, base[:1000])
    ix.add(1500, base[1000:])
    assert ix.getNumData() == 2500 and ix.getDimension() == 48 and ix.getDevice() == 0
    dist, idx = ix.search_array(queries, 20)
    rd, ri = oracle.knn(base, queries, 21)
    assert_knn_matches(base, queries, dist, idx, rd, ri)
    ix.reset()
    assert ix.getNumData() == 0
    dist, idx = ix.search_array(queries, 3)
    assert (idx == -1).all()


def test_deterministic_repeat(cb, res):
    rng = np.random.default_rng(8)
    base = rng.integers(0, 3, size=(20000, 32)).astype(np.float32)  # heavy ties
    queries = rng.integers(0, 3, size=(300, 32)).astype(np.float32)
    for form in FORMS:
        ix = make_index(cb, res, base, precision=form)
        a = ix.search_array(queries, 64)
        b = ix.search_array(queries, 64)
        np.testing.assert_array_equal(a[1], b[1])
        np.testing.assert_array_equal(a[0], b[0])


@pytest.mark.parametrize("form", FORMS)
def test_bf16_exact_rows_rerank_identically(cb, res, form):
    """An index whose values are all exactly BF16 reranks from its BF16 copy;
    the same rows in an index that also holds one non-BF16 row (far away, so
    never a neighbour) rerank from FP32.  Both must give identical results."""
    import torch
    rng = np.random.default_rng(31 + form)
    n, nq, d, k = 5000, 64, 96, 20
    base = torch.tensor(rng.standard_normal((n, d), dtype=np.float32)).bfloat16().float().numpy()
    q = rng.standard_normal((nq, d), dtype=np.float32)
    far = np.full((1, d), 1000.0, np.float32)
    far[0, 0] = 1000.1  # not a BF16 value
    a = make_index(cb, res, base, precision=form)
    b = make_index(cb, res, np.concatenate([base, far]), precision=form)
    da, ia = a.search_array(q, k)
    db, ib = b.search_array(q, k)
    np.testing.assert_array_equal(ia, ib)
    np.testing.assert_array_equal(da, db)
    rd, ri = oracle.knn(base, q, k + 1)
    assert_knn_matches(base, q, da, ia, rd, ri)
    a.close()
    b.close()
