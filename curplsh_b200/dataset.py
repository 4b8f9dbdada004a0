"""TEXMEX ``.fvecs`` / ``.ivecs`` / ``.bvecs`` files and recall evaluation,
mirroring cuRPLSH's dataset helpers (include/dataset.h).

File format (the reference's reader, include/dataset.h:14-45): every row is a
4-byte little-endian integer dimension followed by the row's values (float32
for .fvecs, int32 for .ivecs, uint8 for .bvecs); the dimension is read from
the first row and the row count is file size / (dim * sizeof(value) + 4).

``Dataset.evaluate`` follows ``Dataset::evaluate`` (include/dataset.h:135-152,
src/internal/algorithms.cu:10-28):
recall = mean over queries of |result ∩ ground truth| / gtK, the intersection
taken as sorted multisets.  Unlike the reference, which sorts the caller's
result and ground-truth rows in place, the inputs are left untouched.

No dataset files ship with either project; these load user-supplied SIFT1M /
GIST1M style directories (``<name>_base.fvecs``, ``<name>_query.fvecs``,
``<name>_groundtruth.ivecs``).
"""
from __future__ import annotations

import os

import numpy as np

_DTYPES = {".fvecs": np.float32, ".ivecs": np.int32, ".bvecs": np.uint8}


def load_xvecs(path: str, dtype=None) -> np.ndarray:
    """Reads a TEXMEX file into a [num, dim] array (helper::loadXvecsData,
    include/dataset.h:14-45).  `dtype` defaults from the file extension."""
    if dtype is None:
        dtype = _DTYPES[os.path.splitext(path)[1]]
    dtype = np.dtype(dtype)
    raw = np.fromfile(path, dtype=np.uint8)
    if raw.size < 4:
        raise ValueError(f"{path}: shorter than one row header")
    dim = int(raw[:4].view(np.int32)[0])
    if dim <= 0:
        raise ValueError(f"{path}: bad dimension {dim}")
    row_bytes = 4 + dim * dtype.itemsize
    num = raw.size // row_bytes
    rows = raw[:num * row_bytes].reshape(num, row_bytes)
    dims = rows[:, :4].copy().view(np.int32).reshape(num)
    if num and not (dims == dim).all():
        raise ValueError(f"{path}: rows of different dimensions")
    return rows[:, 4:].copy().view(dtype).reshape(num, dim)


def save_xvecs(path: str, data: np.ndarray) -> None:
    """Writes a [num, dim] array in the TEXMEX layout (the reference leaves
    saveXvecsData a TODO, include/dataset.h:47)."""
    data = np.ascontiguousarray(data)
    num, dim = data.shape
    header = np.full((num, 1), dim, dtype=np.int32).view(np.uint8)
    body = data.view(np.uint8).reshape(num, dim * data.dtype.itemsize)
    np.concatenate([header, body], axis=1).tofile(path)


def recall(indices: np.ndarray, groundtruth: np.ndarray, diff: np.ndarray | None = None) -> float:
    """Dataset::evaluate: mean over queries of |sorted-multiset intersection| / gtK."""
    indices = np.asarray(indices)
    groundtruth = np.asarray(groundtruth)
    nq, gtk = groundtruth.shape
    if indices.shape[0] != nq or indices.shape[1] < gtk:
        raise ValueError("indices must hold at least gtK results per query")
    total = 0.0
    for q in range(nq):
        a = np.sort(indices[q, :gtk])
        b = np.sort(groundtruth[q])
        i = j = hits = 0
        while i < gtk and j < gtk:
            if a[i] < b[j]:
                i += 1
            elif b[j] < a[i]:
                j += 1
            else:
                hits += 1
                i += 1
                j += 1
        if diff is not None:
            diff[q] = gtk - hits
        total += hits / gtk
    return total / nq if nq else 0.0


class Dataset:
    """Dataset<T, IndexT> (include/dataset.h:50-167), host arrays."""

    def __init__(self, base=None, query=None, groundtruth=None, name: str = ""):
        self.base, self.query, self.groundtruth, self.name = base, query, groundtruth, name

    def getDimension(self) -> int:
        return int(self.base.shape[1]) if self.base is not None else 0

    def getGroundTruthK(self) -> int:
        return int(self.groundtruth.shape[1]) if self.groundtruth is not None else 0

    def getNumBase(self) -> int:
        return int(self.base.shape[0]) if self.base is not None else 0

    def getNumQuery(self) -> int:
        return int(self.query.shape[0]) if self.query is not None else 0

    def getBase(self):
        return self.base

    def getQuery(self):
        return self.query

    def getGroundTruth(self):
        return self.groundtruth

    def getName(self) -> str:
        return self.name

    def evaluate(self, indices, diff=None) -> float:
        return recall(indices, self.groundtruth, diff)


class DatasetIrisa(Dataset):
    """DatasetIrisa (include/dataset.h:169-192): <dir>/<name>_{base,query}.fvecs
    and <name>_groundtruth.ivecs."""

    def __init__(self, name: str, datadir: str):
        super().__init__(load_xvecs(os.path.join(datadir, f"{name}_base.fvecs")),
                         load_xvecs(os.path.join(datadir, f"{name}_query.fvecs")),
                         load_xvecs(os.path.join(datadir, f"{name}_groundtruth.ivecs")), name)


class DatasetSIFT(DatasetIrisa):
    """include/dataset.h:194-198"""

    def __init__(self, basedir: str):
        super().__init__("sift", basedir)


class DatasetGIST(DatasetIrisa):
    """include/dataset.h:200-204"""

    def __init__(self, basedir: str):
        super().__init__("gist", basedir)
