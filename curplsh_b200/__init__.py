"""curplsh_b200 -- B200-native exact L2 k-nearest-neighbour engine.

Python mirror of cuRPLSH's host interface (``Index`` / ``IndexBF`` /
``DeviceResources``, include/index.h, include/index_bf.h,
include/device_resources.h), bound with ctypes to the C ABI of
``libcurplsh_b200.so`` (include/curplsh_b200.h).  The compute path is the
CUDA library; if it is missing this module raises on import -- there is no
CPU fallback.

Arrays may be numpy arrays (host memory) or torch tensors (host or CUDA);
float32, C-contiguous.  Methods named like the reference take the same
arguments (``add(num, data)``, ``search(num, queries, k, indices,
distances)``); ``add_array`` / ``search_array`` are the convenience forms
returning new arrays.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

__all__ = [
    "DeviceResources", "IndexBF", "IndexBFConfig", "MemorySpace", "Precision", "CurplshError",
    "compute_l2_norm", "search_l2_distance", "lib_path", "get_num_devices", "SearchBatch", "Server",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
# CURPLSH_B200_LIB selects another build of the library (e.g. an instrumented one).
_LIB_PATH = os.environ.get("CURPLSH_B200_LIB") or os.path.join(_HERE, "libcurplsh_b200.so")


class CurplshError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"curplsh error {code}: {msg}")
        self.code = code


OK, ERR_INVALID_ARG, ERR_CUDA, ERR_OOM, ERR_UNSUPPORTED, ERR_DEVICE, ERR_STATE = range(7)


class MemorySpace:
    """include/memory_space.h:12-17"""
    Device = 0
    Unified = 1


class Precision:
    FP32_EXACT = 0
    BF16_RERANK = 1
    FP8_RERANK = 2


class _Cfg(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("memory_space", ctypes.c_int32),
                ("store_transposed", ctypes.c_int32), ("compute_exact_distances", ctypes.c_int32),
                ("precision", ctypes.c_int32), ("rerank_factor", ctypes.c_int32),
                ("borrow_device_data", ctypes.c_int32)]


class _BatchItem(ctypes.Structure):
    _fields_ = [("index", ctypes.c_void_p), ("num", ctypes.c_int64), ("queries", ctypes.c_void_p),
                ("k", ctypes.c_int32), ("pad0", ctypes.c_int32), ("indices", ctypes.c_void_p),
                ("distances", ctypes.c_void_p)]


class _ServerCfg(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int32), ("rerank_factor", ctypes.c_int32),
                ("max_inflight", ctypes.c_int32), ("max_step_queries", ctypes.c_int32),
                ("memory_budget", ctypes.c_int64)]


class _ServerStats(ctypes.Structure):
    _fields_ = [("requests_done", ctypes.c_int64), ("queries_done", ctypes.c_int64), ("steps", ctypes.c_int64),
                ("kernel_launches", ctypes.c_int64), ("max_step_queries", ctypes.c_int64),
                ("peak_bytes_in_use", ctypes.c_int64), ("max_inflight_seen", ctypes.c_int32),
                ("pad0", ctypes.c_int32), ("busy_seconds", ctypes.c_double)]


def lib_path() -> str:
    return _LIB_PATH


def _load():
    if not os.path.exists(_LIB_PATH):
        raise ImportError(f"{_LIB_PATH} is missing: run `python curplsh_b200/build.py` "
                          "(there is no CPU fallback)")
    lib = ctypes.CDLL(_LIB_PATH)
    vp, i32, i64, f32p, i32p = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p
    sig = {
        "curplsh_bf_config_init": (None, [ctypes.POINTER(_Cfg)]),
        "curplsh_last_error": (ctypes.c_char_p, []),
        "curplsh_version": (ctypes.c_char_p, []),
        "curplsh_get_num_devices": (i32, [ctypes.POINTER(ctypes.c_int)]),
        "curplsh_resources_create": (i32, [ctypes.POINTER(vp)]),
        "curplsh_resources_destroy": (i32, [vp]),
        "curplsh_resources_initialize_for_device": (i32, [vp, i32]),
        "curplsh_resources_get_default_stream": (i32, [vp, i32, ctypes.POINTER(vp)]),
        "curplsh_resources_set_default_stream": (i32, [vp, i32, vp]),
        "curplsh_resources_get_alternate_streams": (i32, [vp, i32, ctypes.POINTER(vp), ctypes.POINTER(ctypes.c_int)]),
        "curplsh_resources_get_async_copy_stream": (i32, [vp, i32, ctypes.POINTER(vp)]),
        "curplsh_resources_sync_default_stream": (i32, [vp, i32]),
        "curplsh_index_bf_create": (i32, [vp, i32, ctypes.POINTER(_Cfg), ctypes.POINTER(vp)]),
        "curplsh_index_destroy": (i32, [vp]),
        "curplsh_index_train": (i32, [vp, i64, f32p]),
        "curplsh_index_add": (i32, [vp, i64, f32p]),
        "curplsh_index_search": (i32, [vp, i64, f32p, i32, i32p, f32p]),
        "curplsh_index_search_ex": (i32, [vp, i64, f32p, i32, i32, i32, i32p, f32p, vp]),
        "curplsh_index_search_profiled": (i32, [vp, i64, f32p, i32, i32, i32, i32p, f32p, vp,
                                                ctypes.POINTER(ctypes.c_float)]),
        "curplsh_index_reset": (i32, [vp]),
        "curplsh_index_get_dimension": (i32, [vp, ctypes.POINTER(ctypes.c_int)]),
        "curplsh_index_get_num_data": (i32, [vp, ctypes.POINTER(ctypes.c_int64)]),
        "curplsh_index_get_device": (i32, [vp, ctypes.POINTER(ctypes.c_int)]),
        "curplsh_compute_l2_norm": (i32, [f32p, i64, i32, f32p, i32, vp]),
        "curplsh_search_l2_distance": (i32, [vp, f32p, i64, f32p, f32p, i64, i32, i32, i32p, f32p, i32]),
        "curplsh_index_search_noalloc": (i32, [vp, i64, f32p, i32, i32p, f32p, vp]),
        "curplsh_batch_create": (i32, [ctypes.POINTER(_BatchItem), i32, i32, i32, ctypes.POINTER(vp)]),
        "curplsh_batch_run": (i32, [vp, vp, i32]),
        "curplsh_batch_get_info": (i32, [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int64)]),
        "curplsh_batch_destroy": (i32, [vp]),
        "curplsh_tuning_set": (i32, [i32, i32, i32, i64, i32, i32]),
        "curplsh_tuning_get": (i32, [i32, i32, i32, i64, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
        "curplsh_tuning_clear": (i32, []),
        "curplsh_server_config_init": (None, [ctypes.POINTER(_ServerCfg)]),
        "curplsh_server_create": (i32, [vp, ctypes.POINTER(_ServerCfg), ctypes.POINTER(vp)]),
        "curplsh_server_submit": (i32, [vp, i64, f32p, i32, i32p, f32p, ctypes.POINTER(ctypes.c_int64)]),
        "curplsh_server_wait": (i32, [vp, i64, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]),
        "curplsh_server_wait_phases": (i32, [vp, i64, ctypes.c_double, ctypes.POINTER(ctypes.c_double),
                                             ctypes.POINTER(ctypes.c_double)]),
        "curplsh_server_get_stats": (i32, [vp, ctypes.POINTER(_ServerStats)]),
        "curplsh_server_destroy": (i32, [vp]),
        "curplsh_merge_shard_results": (i32, [i64, i32, i32, f32p, i32p, vp, i32p, f32p, vp]),
        "curplsh_set_bound_estimate": (i32, [i32]),
        "curplsh_get_bound_estimate": (i32, [ctypes.POINTER(ctypes.c_int)]),
        "curplsh_set_coarse_check": (i32, [i32]),
        "curplsh_index_get_coarse_fallback_count": (i32, [vp, ctypes.POINTER(ctypes.c_int64)]),
        "curplsh_get_coarse_check": (i32, [ctypes.POINTER(ctypes.c_int)]),
        "curplsh_set_cta_pairs": (i32, [i32]),
        "curplsh_get_cta_pairs": (i32, [ctypes.POINTER(ctypes.c_int)]),
        "curplsh_set_dual_blocks": (i32, [i32]),
        "curplsh_get_dual_blocks": (i32, [ctypes.POINTER(ctypes.c_int)]),
        "curplsh_index_estimate_plan": (i32, [vp, i64, i32, i32, i32, ctypes.POINTER(ctypes.c_int),
                                              ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
        "curplsh_index_get_fallback_count": (i32, [vp, ctypes.POINTER(ctypes.c_int64)]),
        "curplsh_estimate_plan_shape": (i32, [i64, i64, i32, i32, ctypes.POINTER(ctypes.c_int),
                                              ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_lib = _load()

# Every symbol the C header declares; tests check the library exports them all.
EXPORTED_SYMBOLS = (
    "curplsh_bf_config_init", "curplsh_last_error", "curplsh_version", "curplsh_get_num_devices",
    "curplsh_resources_create", "curplsh_resources_destroy", "curplsh_resources_initialize_for_device",
    "curplsh_resources_get_default_stream", "curplsh_resources_set_default_stream",
    "curplsh_resources_get_alternate_streams", "curplsh_resources_get_async_copy_stream",
    "curplsh_resources_sync_default_stream", "curplsh_index_bf_create", "curplsh_index_destroy",
    "curplsh_index_train", "curplsh_index_add", "curplsh_index_search", "curplsh_index_search_ex",
    "curplsh_index_search_profiled", "curplsh_index_reset", "curplsh_index_get_dimension",
    "curplsh_index_get_num_data", "curplsh_index_get_device", "curplsh_compute_l2_norm",
    "curplsh_search_l2_distance", "curplsh_index_search_noalloc", "curplsh_batch_create", "curplsh_batch_run",
    "curplsh_batch_get_info", "curplsh_batch_destroy", "curplsh_tuning_set", "curplsh_tuning_get",
    "curplsh_tuning_clear", "curplsh_server_config_init", "curplsh_server_create", "curplsh_server_submit",
    "curplsh_server_wait", "curplsh_server_wait_phases", "curplsh_server_get_stats", "curplsh_server_destroy", "curplsh_merge_shard_results",
    "curplsh_set_bound_estimate", "curplsh_get_bound_estimate", "curplsh_index_estimate_plan",
    "curplsh_index_get_fallback_count", "curplsh_estimate_plan_shape", "curplsh_set_coarse_check",
    "curplsh_get_coarse_check", "curplsh_index_get_coarse_fallback_count", "curplsh_set_cta_pairs",
    "curplsh_get_cta_pairs", "curplsh_set_dual_blocks", "curplsh_get_dual_blocks",
)


def _check(rc: int):
    if rc != OK:
        raise CurplshError(rc, _lib.curplsh_last_error().decode(errors="replace"))


def version() -> str:
    return _lib.curplsh_version().decode()


def get_num_devices() -> int:
    n = ctypes.c_int(0)
    _check(_lib.curplsh_get_num_devices(ctypes.byref(n)))
    return n.value


# ------------------------------------------------------------------ arrays
def _ptr(a, dtype, writable=False):
    """Raw pointer of a float32/int32 C-contiguous numpy array or torch tensor."""
    if a is None:
        return None
    if hasattr(a, "data_ptr") and hasattr(a, "is_contiguous"):  # torch tensor
        import torch
        want = {np.float32: torch.float32, np.int32: torch.int32}[dtype]
        if a.dtype != want or not a.is_contiguous():
            raise TypeError(f"expected a contiguous {want} tensor")
        return ctypes.c_void_p(a.data_ptr())
    if not isinstance(a, np.ndarray):
        raise TypeError("expected a numpy array or torch tensor")
    if a.dtype != dtype or not a.flags.c_contiguous or (writable and not a.flags.writeable):
        raise TypeError(f"expected a C-contiguous {np.dtype(dtype)} array")
    return ctypes.c_void_p(a.ctypes.data)


def _stream_ptr(stream):
    if stream is None:
        return None
    if hasattr(stream, "cuda_stream"):
        return ctypes.c_void_p(stream.cuda_stream)
    return ctypes.c_void_p(int(stream))


# ------------------------------------------------------------------ resources
class DeviceResources:
    """include/device_resources.h:60-263 (streams per device; no cuBLAS/cuRAND handles are needed)."""

    def __init__(self, devices=None):
        h = ctypes.c_void_p()
        _check(_lib.curplsh_resources_create(ctypes.byref(h)))
        self._h = h
        if devices is not None:
            for d in ([devices] if isinstance(devices, int) else devices):
                self.initializeForDevice(d)

    def close(self):
        if getattr(self, "_h", None):
            _lib.curplsh_resources_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def initializeForDevice(self, device: int):
        _check(_lib.curplsh_resources_initialize_for_device(self._h, device))

    def getDefaultStream(self, device: int) -> int:
        s = ctypes.c_void_p()
        _check(_lib.curplsh_resources_get_default_stream(self._h, device, ctypes.byref(s)))
        return s.value or 0

    def setDefaultStream(self, device: int, stream) -> None:
        _check(_lib.curplsh_resources_set_default_stream(self._h, device, _stream_ptr(stream)))

    def getAlternateStreams(self, device: int):
        arr = (ctypes.c_void_p * 2)()
        n = ctypes.c_int(2)
        _check(_lib.curplsh_resources_get_alternate_streams(self._h, device, arr, ctypes.byref(n)))
        return [arr[i] or 0 for i in range(n.value)]

    def getAsyncCopyStream(self, device: int) -> int:
        s = ctypes.c_void_p()
        _check(_lib.curplsh_resources_get_async_copy_stream(self._h, device, ctypes.byref(s)))
        return s.value or 0

    def syncDefaultStream(self, device: int) -> None:
        _check(_lib.curplsh_resources_sync_default_stream(self._h, device))


class IndexBFConfig:
    """IndexBFConfig (include/index_bf.h:8-19) + IndexConfig (include/index.h:8-16) + precision controls."""

    def __init__(self, device=0, memorySpace=MemorySpace.Device, storeTransposed=False,
                 computeExactDistances=False, precision=Precision.FP32_EXACT, rerankFactor=0,
                 borrowDeviceData=False):
        self.device = device
        self.memorySpace = memorySpace
        self.storeTransposed = storeTransposed
        self.computeExactDistances = computeExactDistances
        self.precision = precision
        self.rerankFactor = rerankFactor
        self.borrowDeviceData = borrowDeviceData

    def _c(self) -> _Cfg:
        c = _Cfg()
        _lib.curplsh_bf_config_init(ctypes.byref(c))
        c.device = self.device
        c.memory_space = self.memorySpace
        c.store_transposed = int(bool(self.storeTransposed))
        c.compute_exact_distances = int(bool(self.computeExactDistances))
        c.precision = self.precision
        c.rerank_factor = self.rerankFactor
        c.borrow_device_data = int(bool(self.borrowDeviceData))
        return c


class IndexBF:
    """Brute-force exact L2 index (include/index_bf.h:21-46, src/index_bf.cpp)."""

    def __init__(self, resources: DeviceResources, dim: int, config: IndexBFConfig | None = None):
        self._res = resources
        self.config = config or IndexBFConfig()
        h = ctypes.c_void_p()
        cfg = self.config._c()
        _check(_lib.curplsh_index_bf_create(resources._h, int(dim), ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self._keep = None  # borrowed device rows must outlive the index

    def close(self):
        if getattr(self, "_h", None):
            _lib.curplsh_index_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- reference-shaped methods (include/index.h:29-64)
    def train(self, num: int, data) -> None:
        _check(_lib.curplsh_index_train(self._h, int(num), _ptr(data, np.float32) if data is not None else None))

    def add(self, num: int, data) -> None:
        if self.config.borrowDeviceData:
            self._keep = data
        _check(_lib.curplsh_index_add(self._h, int(num), _ptr(data, np.float32)))

    def search(self, num: int, queries, k: int, indices, distances) -> None:
        _check(_lib.curplsh_index_search(self._h, int(num), _ptr(queries, np.float32), int(k),
                                         _ptr(indices, np.int32, True), _ptr(distances, np.float32, True)))

    def search_ex(self, num: int, queries, k: int, indices, distances, precision: int = -1,
                  rerank_factor: int = -1, stream=None) -> None:
        """search with an explicit precision form, rerank factor and stream.  With device
        buffers the call is asynchronous on `stream`, except when the BF16/FP8 coarse-margin
        check applies (it then returns synchronised, after searching again in the exact
        form any query the check lists).  A sampled bound estimate is verified on the
        stream in the asynchronous case and by the host otherwise."""
        _check(_lib.curplsh_index_search_ex(self._h, int(num), _ptr(queries, np.float32), int(k), int(precision),
                                            int(rerank_factor), _ptr(indices, np.int32, True),
                                            _ptr(distances, np.float32, True), _stream_ptr(stream)))

    def search_profiled(self, num: int, queries, k: int, indices, distances, precision: int = -1,
                        rerank_factor: int = -1, stream=None):
        ms = (ctypes.c_float * 4)()
        _check(_lib.curplsh_index_search_profiled(self._h, int(num), _ptr(queries, np.float32), int(k),
                                                  int(precision), int(rerank_factor),
                                                  _ptr(indices, np.int32, True), _ptr(distances, np.float32, True),
                                                  _stream_ptr(stream), ms))
        return {"prep_ms": ms[0], "fused_ms": ms[1], "merge_ms": ms[2], "total_ms": ms[3]}

    def search_noalloc(self, num: int, queries, k: int, indices, distances, stream=None) -> None:
        """Search without allocating any memory (for callers that cannot allocate
        device memory while serving).  queries / indices / distances must be CUDA
        tensors on the index's device; runs out of the library's fixed 64 MiB
        scratch and returns once the results are written."""
        _check(_lib.curplsh_index_search_noalloc(self._h, int(num), _ptr(queries, np.float32), int(k),
                                                 _ptr(indices, np.int32, True), _ptr(distances, np.float32, True),
                                                 _stream_ptr(stream)))

    def reset(self) -> None:
        _check(_lib.curplsh_index_reset(self._h))
        self._keep = None

    def getDimension(self) -> int:
        v = ctypes.c_int()
        _check(_lib.curplsh_index_get_dimension(self._h, ctypes.byref(v)))
        return v.value

    def getNumData(self) -> int:
        v = ctypes.c_int64()
        _check(_lib.curplsh_index_get_num_data(self._h, ctypes.byref(v)))
        return v.value

    def getDevice(self) -> int:
        v = ctypes.c_int()
        _check(_lib.curplsh_index_get_device(self._h, ctypes.byref(v)))
        return v.value

    def getResources(self) -> DeviceResources:
        return self._res

    def estimate_plan(self, num_queries: int, k: int, precision: int = -1, rerank_factor: int = -1):
        """(sample_rows, step, rank) of the sampled bound estimate a search of this
        shape would use (rank among the sample_rows / 128 block minima);
        sample_rows == 0 when it uses none."""
        a, b, c = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
        _check(_lib.curplsh_index_estimate_plan(self._h, int(num_queries), int(k), int(precision),
                                                int(rerank_factor), ctypes.byref(a), ctypes.byref(b),
                                                ctypes.byref(c)))
        return a.value, b.value, c.value

    def fallback_count(self) -> int:
        """Queries searched again after their estimated bound failed (since creation)."""
        v = ctypes.c_int64()
        _check(_lib.curplsh_index_get_fallback_count(self._h, ctypes.byref(v)))
        return v.value

    def coarse_fallback_count(self) -> int:
        """Queries searched again in the exact form after their coarse margin failed
        (since creation)."""
        v = ctypes.c_int64()
        _check(_lib.curplsh_index_get_coarse_fallback_count(self._h, ctypes.byref(v)))
        return v.value

    # -- convenience forms
    def add_array(self, data) -> None:
        self.add(int(data.shape[0]), data)

    def search_array(self, queries, k: int, precision: int = -1, rerank_factor: int = -1):
        """Returns (distances [nq,k] float32, indices [nq,k] int32) in the queries' memory space."""
        nq = int(queries.shape[0])
        if hasattr(queries, "is_cuda"):
            import torch
            dist = torch.empty((nq, k), dtype=torch.float32, device=queries.device)
            idx = torch.empty((nq, k), dtype=torch.int32, device=queries.device)
        else:
            dist = np.empty((nq, k), dtype=np.float32)
            idx = np.empty((nq, k), dtype=np.int32)
        if precision < 0 and rerank_factor < 0:
            self.search(nq, queries, k, idx, dist)
        else:
            self.search_ex(nq, queries, k, idx, dist, precision, rerank_factor)
            if hasattr(queries, "is_cuda") and queries.is_cuda:
                import torch
                torch.cuda.synchronize(queries.device)
        return dist, idx


def compute_l2_norm(vectors, norms, squared: bool = True, stream=None) -> None:
    """computeL2Norm (include/internal/norm.h:7-8) over device tensors."""
    _check(_lib.curplsh_compute_l2_norm(_ptr(vectors, np.float32), int(vectors.shape[0]), int(vectors.shape[1]),
                                        _ptr(norms, np.float32, True), int(bool(squared)), _stream_ptr(stream)))


def search_l2_distance(resources: DeviceResources, bases, base_norms, queries, k: int, indices, distances,
                       exact_distances: bool) -> None:
    """searchL2Distance (include/internal/search.h:7-11) over device tensors."""
    _check(_lib.curplsh_search_l2_distance(resources._h, _ptr(bases, np.float32), int(bases.shape[0]),
                                           _ptr(base_norms, np.float32) if base_norms is not None else None,
                                           _ptr(queries, np.float32), int(queries.shape[0]), int(queries.shape[1]),
                                           int(k), _ptr(indices, np.int32, True), _ptr(distances, np.float32, True),
                                           int(bool(exact_distances))))


class SearchBatch:
    """A fixed list of searches over one or more indexes, replayed as one CUDA graph.

    ``items`` is a sequence of ``(index, queries, k, indices, distances)`` with
    CUDA tensors on the indexes' device: queries [nq, dim] float32, indices
    [nq, k] int32 and distances [nq, k] float32.  The tensors are captured by
    address: overwrite ``queries`` in place and call :meth:`run` again.  Every
    item's results equal ``index.search_ex`` of that item alone with the same
    precision and rerank factor.  No counterpart in the reference.
    """

    def __init__(self, items, precision: int = -1, rerank_factor: int = -1):
        arr = (_BatchItem * len(items))()
        self._keep = []
        for i, (index, queries, k, indices, distances) in enumerate(items):
            nq = int(queries.shape[0])
            arr[i].index = index._h
            arr[i].num = nq
            arr[i].queries = _ptr(queries, np.float32).value if nq else None
            arr[i].k = int(k)
            arr[i].indices = _ptr(indices, np.int32, True).value if nq else None
            arr[i].distances = _ptr(distances, np.float32, True).value if nq else None
            self._keep.append((index, queries, indices, distances))
        h = ctypes.c_void_p()
        _check(_lib.curplsh_batch_create(arr, len(items), int(precision), int(rerank_factor), ctypes.byref(h)))
        self._h = h

    def run(self, stream=None, wait: bool = True) -> None:
        _check(_lib.curplsh_batch_run(self._h, _stream_ptr(stream), int(bool(wait))))

    def info(self):
        """(kernel launches per run, device working-memory bytes)."""
        n = ctypes.c_int(0)
        b = ctypes.c_int64(0)
        _check(_lib.curplsh_batch_get_info(self._h, ctypes.byref(n), ctypes.byref(b)))
        return n.value, b.value

    def close(self):
        if getattr(self, "_h", None):
            _lib.curplsh_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tuning_set(precision: int, dim: int, k: int, num_queries: int, split_q4: int, pool_headroom: int) -> None:
    """Sets the fused-pass parameters of one (precision, dim, k, Q) bucket (no reference counterpart)."""
    _check(_lib.curplsh_tuning_set(int(precision), int(dim), int(k), int(num_queries), int(split_q4),
                                   int(pool_headroom)))


def tuning_get(precision: int, dim: int, k: int, num_queries: int):
    """(split_q4, pool_headroom) of the bucket holding this shape."""
    a = ctypes.c_int(0)
    b = ctypes.c_int(0)
    _check(_lib.curplsh_tuning_get(int(precision), int(dim), int(k), int(num_queries), ctypes.byref(a),
                                   ctypes.byref(b)))
    return a.value, b.value


def tuning_clear() -> None:
    _check(_lib.curplsh_tuning_clear())


def set_bound_estimate(enabled: bool) -> None:
    """Process-wide switch of the sampled bound estimate (speed only; results are identical)."""
    _check(_lib.curplsh_set_bound_estimate(1 if enabled else 0))


def estimate_plan_shape(num_rows: int, num_queries: int, kprime: int, num_sms: int = 148):
    """(sample_rows, step, rank) of the sampled bound estimate for a bare search shape
    (no index or device needed); sample_rows == 0 when that shape uses none."""
    a, b, c = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
    _check(_lib.curplsh_estimate_plan_shape(int(num_rows), int(num_queries), int(kprime), int(num_sms),
                                            ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
    return a.value, b.value, c.value


def get_bound_estimate() -> bool:
    v = ctypes.c_int(0)
    _check(_lib.curplsh_get_bound_estimate(ctypes.byref(v)))
    return bool(v.value)


def set_coarse_check(enabled: bool) -> None:
    """Process-wide switch of the BF16/FP8 coarse-margin check: a query whose
    candidate margin does not cover the coarse error seen among its candidates
    is searched again in the FP32-exact form (on by default)."""
    _check(_lib.curplsh_set_coarse_check(1 if enabled else 0))


def get_coarse_check() -> bool:
    v = ctypes.c_int(0)
    _check(_lib.curplsh_get_coarse_check(ctypes.byref(v)))
    return bool(v.value)


def set_cta_pairs(mode) -> None:
    """Process-wide CTA pairs mode: fused passes over >= 4 query blocks run as
    clusters of two CTAs sharing one 256-row tensor-core MMA.  True: every such
    pass; False: none; "auto" (the default): BF16 passes with d >= 320 and
    FP32-exact passes with d >= 192.  Results do not depend on it."""
    v = 2 if mode == "auto" else (1 if mode else 0)
    _check(_lib.curplsh_set_cta_pairs(v))


def get_cta_pairs():
    """True, False or "auto" (see set_cta_pairs)."""
    v = ctypes.c_int(0)
    _check(_lib.curplsh_get_cta_pairs(ctypes.byref(v)))
    return "auto" if v.value == 2 else bool(v.value)


def set_dual_blocks(enabled: bool) -> None:
    """Process-wide switch of dual query blocks (on by default): FP8 fused passes
    over >= 4 query blocks keep two blocks per CTA against 128-row database tiles
    (results do not depend on it)."""
    _check(_lib.curplsh_set_dual_blocks(1 if enabled else 0))


def get_dual_blocks() -> bool:
    v = ctypes.c_int(0)
    _check(_lib.curplsh_get_dual_blocks(ctypes.byref(v)))
    return bool(v.value)


class Server:
    """Serving loop with continuous batching over one resident index (no
    counterpart in the reference).  ``submit`` queues a request and returns a
    ticket at once; ``wait`` blocks until its results are written and returns
    the request's latency in seconds.  Arrays may be host (numpy / CPU torch)
    or CUDA tensors; they must stay alive and unmodified until ``wait``."""

    def __init__(self, index: "IndexBF", precision: int = -1, rerank_factor: int = 0, max_inflight: int = 3,
                 max_step_queries: int = 4096, memory_budget: int = 2 << 30):
        cfg = _ServerCfg()
        _lib.curplsh_server_config_init(ctypes.byref(cfg))
        cfg.precision = int(precision)
        cfg.rerank_factor = int(rerank_factor)
        cfg.max_inflight = int(max_inflight)
        cfg.max_step_queries = int(max_step_queries)
        cfg.memory_budget = int(memory_budget)
        h = ctypes.c_void_p()
        _check(_lib.curplsh_server_create(index._h, ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self._index = index
        self._keep = {}

    def submit(self, queries, k: int, indices, distances) -> int:
        t = ctypes.c_int64(0)
        _check(_lib.curplsh_server_submit(self._h, int(queries.shape[0]), _ptr(queries, np.float32), int(k),
                                          _ptr(indices, np.int32, True), _ptr(distances, np.float32, True),
                                          ctypes.byref(t)))
        self._keep[t.value] = (queries, indices, distances)
        return t.value

    def wait(self, ticket: int, timeout: float = -1.0) -> float:
        lat = ctypes.c_double(0.0)
        rc = _lib.curplsh_server_wait(self._h, int(ticket), float(timeout), ctypes.byref(lat))
        if rc != ERR_STATE:  # anything but a time-out ends the ticket
            self._keep.pop(ticket, None)
        _check(rc)
        return lat.value

    def wait_phases(self, ticket: int, timeout: float = -1.0):
        """wait() that also returns the latency's phases (seconds): (latency,
        waiting for a step, step on the device, retiring) on the host clock,
        the step's device work itself timed by CUDA events, and the time from
        issue until that work was seen begun."""
        lat = ctypes.c_double(0.0)
        ph = (ctypes.c_double * 5)()
        rc = _lib.curplsh_server_wait_phases(self._h, int(ticket), float(timeout), ctypes.byref(lat), ph)
        if rc != ERR_STATE:
            self._keep.pop(ticket, None)
        _check(rc)
        return lat.value, ph[0], ph[1], ph[2], ph[3], ph[4]

    def stats(self) -> dict:
        st = _ServerStats()
        _check(_lib.curplsh_server_get_stats(self._h, ctypes.byref(st)))
        return {name: getattr(st, name) for name, _ in _ServerStats._fields_ if name != "pad0"}

    def close(self):
        if getattr(self, "_h", None):
            _lib.curplsh_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def merge_shard_results(distances, indices, shard_bases, out_indices, out_distances, stream=None) -> None:
    """Global top-k from per-shard results (CUDA tensors): distances [G, Q, k] float32, indices
    [G, Q, k] int32 (shard-local rows), shard_bases [G] int64 (first global row of each shard)."""
    import torch
    if shard_bases.dtype != torch.int64 or not shard_bases.is_contiguous():
        raise TypeError("shard_bases must be a contiguous int64 tensor")
    G, Q, k = (int(x) for x in distances.shape)
    _check(_lib.curplsh_merge_shard_results(Q, k, G, _ptr(distances, np.float32), _ptr(indices, np.int32),
                                            ctypes.c_void_p(shard_bases.data_ptr()),
                                            _ptr(out_indices, np.int32, True), _ptr(out_distances, np.float32, True),
                                            _stream_ptr(stream)))
