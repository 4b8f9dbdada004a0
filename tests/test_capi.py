"""C ABI checks that need no GPU: the library loads, exports every symbol that
include/*.h declares, and the host-side argument validation works."""
import ctypes
import os
import re

import numpy as np
import pytest

import curplsh_b200 as cb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if not f.endswith(".h"):
            continue
        src = open(os.path.join(inc, f)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(curplsh_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return names


def test_library_is_in_tree_and_loads():
    assert os.path.exists(cb.lib_path())
    assert os.path.dirname(cb.lib_path()) == os.path.join(ROOT, "curplsh_b200")
    assert "sm_100a" in cb.version()


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(cb.lib_path())
    decl = declared_symbols()
    assert len(decl) >= 25
    missing = [s for s in sorted(decl) if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_declarations():
    assert set(cb.EXPORTED_SYMBOLS) <= declared_symbols()


def test_config_defaults():
    c = cb._Cfg()
    cb._lib.curplsh_bf_config_init(ctypes.byref(c))
    assert (c.device, c.memory_space, c.precision, c.rerank_factor, c.borrow_device_data) == (0, 0, 0, 0, 0)
    assert c.store_transposed == 0 and c.compute_exact_distances == 0


def test_resources_create_destroy_without_gpu():
    r = cb.DeviceResources()
    r.close()
    r.close()  # idempotent


def test_null_arguments_rejected():
    lib = cb._lib
    assert lib.curplsh_index_add(None, 10, None) == cb.ERR_INVALID_ARG
    assert "null" in cb._lib.curplsh_last_error().decode()
    assert lib.curplsh_index_search(None, 1, None, 1, None, None) == cb.ERR_INVALID_ARG
    assert lib.curplsh_resources_initialize_for_device(None, 0) == cb.ERR_INVALID_ARG
    assert lib.curplsh_compute_l2_norm(None, 5, 0, None, 1, None) == cb.ERR_INVALID_ARG
    assert lib.curplsh_compute_l2_norm(None, 0, 4, None, 1, None) == cb.OK  # empty is a no-op
    v = ctypes.c_int()
    assert lib.curplsh_index_get_dimension(None, ctypes.byref(v)) == cb.ERR_INVALID_ARG


def test_index_creation_needs_a_device():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present; covered by the gpu tests")
    except ImportError:
        pass
    r = cb.DeviceResources()
    with pytest.raises(cb.CurplshError) as e:
        cb.IndexBF(r, 16)
    assert e.value.code in (cb.ERR_CUDA, cb.ERR_INVALID_ARG, cb.ERR_UNSUPPORTED)


def test_array_pointer_validation():
    with pytest.raises(TypeError):
        cb._ptr(np.zeros((2, 2), np.float64), np.float32)
    with pytest.raises(TypeError):
        cb._ptr(np.zeros((4, 4), np.float32)[:, ::2], np.float32)
    assert cb._ptr(np.zeros((2, 2), np.float32), np.float32).value


def test_tuning_table_roundtrip():
    """The tuning table needs no GPU: set, bucketed get, defaults, clear, and argument checks."""
    import curplsh_b200 as cb
    cb.tuning_clear()
    assert cb.tuning_get(1, 128, 100, 10000) == (4, 256)
    cb.tuning_set(1, 128, 100, 10000, 2, 512)
    # same bucket: k in (64, 128], nq in [8192, 16384)
    assert cb.tuning_get(1, 128, 65, 8192) == (2, 512)
    assert cb.tuning_get(1, 128, 128, 16383) == (2, 512)
    # other buckets keep the defaults
    assert cb.tuning_get(1, 128, 100, 16384) == (4, 256)
    assert cb.tuning_get(0, 128, 100, 10000) == (4, 256)
    assert cb.tuning_get(1, 64, 100, 10000) == (4, 256)
    with pytest.raises(cb.CurplshError):
        cb.tuning_set(1, 128, 100, 10000, 0, 512)
    with pytest.raises(cb.CurplshError):
        cb.tuning_set(1, 128, 100, 10000, 4, 64)
    with pytest.raises(cb.CurplshError):
        cb.tuning_set(3, 128, 100, 10000, 4, 256)
    cb.tuning_clear()
    assert cb.tuning_get(1, 128, 100, 10000) == (4, 256)


def test_autotune_bucket_matches_library():
    from curplsh_b200 import autotune
    assert autotune.bucket(1, 128, 100, 10000) == "1,128,7,13"
    assert autotune.bucket(0, 64, 1, 1) == "0,64,0,0"
    assert autotune.bucket(2, 96, 1024, 4096) == "2,96,10,12"
