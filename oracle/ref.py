"""The reference's own search path (cuRPLSH computeL2Norm + searchL2Distance,
compiled from its sources into oracle/_ref/libcurplsh_ref.so by
``make -C oracle ref``) -- TEST AND BASELINE INFRASTRUCTURE ONLY.

Used to produce the golden outputs the parity tests compare against
(tests/golden/gen_ref_fixtures.py) and, in a subprocess of bench.py, to time
the reference on the same GPU.  Never imported by the curplsh_b200 product.

The reference code runs in bounds only for d = 128, row counts that are
multiples of 8 and 2 <= k <= 1024 (see ref_driver.cu).  `search` pads what
it can without changing any distance: zero columns up to d = 128 (queries
and rows alike), zero query rows up to a multiple of 8 (their results are
dropped), and host-computed FP32 row norms when N is not a multiple of 8.

    python -m oracle.ref --workload mixture_int_1m --queries 256 --reps 3
prints one JSON line with the reference's timings on cuda:0.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")
LIB_PATH = os.path.join(REF_DIR, "libcurplsh_ref.so")
REF_SOURCES = "/root/reference"
_lib = None


def build(force: bool = False) -> str | None:
    """Compile the reference's search path when its sources are present (this
    container); elsewhere the prebuilt library, if any, is used."""
    if not os.path.isdir(os.path.join(REF_SOURCES, "src", "internal")):
        return LIB_PATH if os.path.exists(LIB_PATH) else None
    cmd = ["make", "-s", "-C", _HERE, "-j8", "ref", f"REF={REF_SOURCES}"]
    if force:
        subprocess.check_call(["make", "-s", "-C", _HERE, "clean"])
        subprocess.check_call(["make", "-s", "-C", _HERE, "libknn_oracle.so"])
    subprocess.check_call(cmd)
    return LIB_PATH


def available() -> bool:
    return os.path.exists(LIB_PATH)


def _load():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"{LIB_PATH} is not built (make -C oracle ref, with the reference sources present)")
        lib = ctypes.CDLL(LIB_PATH)
        lib.curplsh_ref_last_error.restype = ctypes.c_char_p
        lib.curplsh_ref_open.argtypes = [ctypes.c_int]
        lib.curplsh_ref_add.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p,
                                        ctypes.POINTER(ctypes.c_void_p)]
        lib.curplsh_ref_free.argtypes = [ctypes.c_void_p]
        lib.curplsh_ref_search.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int,
                                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
        _lib = lib
    return _lib


def _check(rc):
    if rc != 0:
        raise RuntimeError("reference: " + _load().curplsh_ref_last_error().decode())


def _pad_cols(x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float32)
    d = x.shape[1]
    if d == 128:
        return x
    if d > 128:
        raise ValueError("the reference's norm kernel runs in bounds only for d = 128; d > 128 is not supported here")
    out = np.zeros((x.shape[0], 128), dtype=np.float32)
    out[:, :d] = x
    return out


class Database:
    """IndexBF::add of the reference on cuda:`device` (rows stay resident)."""

    def __init__(self, rows: np.ndarray, device: int = 0):
        lib = _load()
        _check(lib.curplsh_ref_open(int(device)))
        x = _pad_cols(rows)
        self.n = x.shape[0]
        norms = None
        if self.n % 8:
            norms = np.einsum("ij,ij->i", x, x).astype(np.float32)  # FP32 norms, as computeL2Norm gives
        h = ctypes.c_void_p()
        _check(lib.curplsh_ref_add(x.ctypes.data, self.n, 128,
                                   norms.ctypes.data if norms is not None else None, ctypes.byref(h)))
        self._h = h

    def search(self, queries: np.ndarray, k: int, reps: int = 1):
        """IndexBF::search with host queries.  Returns (distances [nq,k] f32,
        indices [nq,k] i32, ms_e2e, ms_resident) -- mean times over `reps`."""
        q = _pad_cols(queries)
        nq = q.shape[0]
        nq8 = (nq + 7) // 8 * 8
        if nq8 != nq:
            q = np.concatenate([q, np.zeros((nq8 - nq, 128), np.float32)])
        q = np.ascontiguousarray(q)
        idx = np.empty((nq8, k), np.int32)
        dist = np.empty((nq8, k), np.float32)
        e2e = ctypes.c_double()
        res = ctypes.c_double()
        _check(_load().curplsh_ref_search(self._h, q.ctypes.data, nq8, int(k), idx.ctypes.data, dist.ctypes.data,
                                          int(reps), ctypes.byref(e2e), ctypes.byref(res)))
        return dist[:nq], idx[:nq], e2e.value, res.value

    def close(self):
        if self._h:
            _load().curplsh_ref_free(self._h)
            self._h = None


def _load_synth():
    import importlib.util
    path = os.path.join(os.path.dirname(_HERE), "curplsh_b200", "synth.py")
    spec = importlib.util.spec_from_file_location("curplsh_synth", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main(argv=None) -> int:
    """Times the reference on one synthetic workload (numpy-generated inputs)."""
    import argparse
    import time
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", required=True)
    ap.add_argument("--queries", type=int, default=0, help="first Q queries of the workload (0: all)")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    a = ap.parse_args(argv)
    synth = _load_synth()
    t0 = time.perf_counter()
    N, Q, d, k = synth.CONFIGS[a.workload]
    base, queries, k = synth.make(a.workload, q=a.queries or None)
    gen_s = time.perf_counter() - t0
    db = Database(base)
    for _ in range(a.warmup):
        db.search(queries, k)
    dist, idx, e2e, resident = db.search(queries, k, reps=a.reps)
    db.close()
    nq = queries.shape[0]
    print(json.dumps({"workload": a.workload, "N": int(base.shape[0]), "Q": nq, "d": d, "k": k,
                      "queries_per_s_resident": nq / (resident / 1e3), "queries_per_s_e2e": nq / (e2e / 1e3),
                      "ms_resident": resident, "ms_e2e": e2e, "reps": a.reps, "data_gen_s": gen_s,
                      "idx_checksum": int(idx.astype(np.int64).sum()), "padded_d": d != 128}), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
