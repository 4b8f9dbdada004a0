"""TEXMEX file I/O and recall evaluation (curplsh_b200.dataset), on CPU."""
import numpy as np
import pytest

from curplsh_b200 import dataset


def test_fvecs_layout_and_roundtrip(tmp_path):
    x = np.arange(12, dtype=np.float32).reshape(3, 4)
    p = str(tmp_path / "a.fvecs")
    dataset.save_xvecs(p, x)
    raw = np.fromfile(p, dtype=np.int32)
    # every row: int32 dimension, then the values (include/dataset.h:14-45)
    assert raw.size == 3 * 5 and (raw.reshape(3, 5)[:, 0] == 4).all()
    np.testing.assert_array_equal(raw.reshape(3, 5)[:, 1:].view(np.float32), x)
    np.testing.assert_array_equal(dataset.load_xvecs(p), x)


def test_ivecs_bvecs_roundtrip(tmp_path):
    gt = np.array([[5, 1, 3], [0, 2, 4]], dtype=np.int32)
    p = str(tmp_path / "g.ivecs")
    dataset.save_xvecs(p, gt)
    np.testing.assert_array_equal(dataset.load_xvecs(p), gt)
    b = np.arange(10, dtype=np.uint8).reshape(2, 5)
    pb = str(tmp_path / "b.bvecs")
    dataset.save_xvecs(pb, b)
    np.testing.assert_array_equal(dataset.load_xvecs(pb), b)


def test_trailing_partial_row_ignored(tmp_path):
    # the row count is file size // row size, as in the reference
    x = np.ones((2, 3), np.float32)
    p = str(tmp_path / "t.fvecs")
    dataset.save_xvecs(p, x)
    with open(p, "ab") as f:
        f.write(b"\x03\x00")
    assert dataset.load_xvecs(p).shape == (2, 3)


def test_bad_files_rejected(tmp_path):
    p = tmp_path / "bad.fvecs"
    p.write_bytes(b"\x00\x00")
    with pytest.raises(ValueError):
        dataset.load_xvecs(str(p))
    rows = np.concatenate([np.array([[2]], np.int32).view(np.uint8), np.ones((1, 2), np.float32).view(np.uint8)], 1)
    rows2 = np.concatenate([np.array([[3]], np.int32).view(np.uint8), np.ones((1, 2), np.float32).view(np.uint8)], 1)
    (tmp_path / "mixed.fvecs").write_bytes(rows.tobytes() + rows2.tobytes())
    with pytest.raises(ValueError):
        dataset.load_xvecs(str(tmp_path / "mixed.fvecs"))


def test_recall_is_sorted_multiset_intersection():
    gt = np.array([[1, 2, 3, 4], [7, 8, 9, 10]])
    res = np.array([[4, 3, 2, 1], [10, 11, 12, 7]])
    diff = np.zeros(2, np.int64)
    assert dataset.recall(res, gt, diff) == pytest.approx((1.0 + 0.5) / 2)
    assert diff.tolist() == [0, 2]
    # repeated results count once per matching ground-truth entry
    assert dataset.recall(np.array([[1, 1, 1, 1]]), np.array([[1, 2, 3, 4]])) == pytest.approx(0.25)
    # inputs are not modified
    assert res.tolist() == [[4, 3, 2, 1], [10, 11, 12, 7]]


def test_irisa_directory(tmp_path):
    rng = np.random.default_rng(0)
    base = rng.random((50, 8), dtype=np.float32)
    query = rng.random((5, 8), dtype=np.float32)
    d = ((query[:, None, :] - base[None]) ** 2).sum(-1)
    gt = np.argsort(d, axis=1, kind="stable")[:, :10].astype(np.int32)
    dataset.save_xvecs(str(tmp_path / "sift_base.fvecs"), base)
    dataset.save_xvecs(str(tmp_path / "sift_query.fvecs"), query)
    dataset.save_xvecs(str(tmp_path / "sift_groundtruth.ivecs"), gt)
    ds = dataset.DatasetSIFT(str(tmp_path))
    assert (ds.getNumBase(), ds.getNumQuery(), ds.getDimension(), ds.getGroundTruthK()) == (50, 5, 8, 10)
    assert ds.getName() == "sift"
    assert ds.evaluate(gt) == 1.0
