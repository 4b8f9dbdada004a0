"""Record the reference's own search outputs as golden fixtures.

Runs cuRPLSH's computeL2Norm + searchL2Distance(..., computeExactDistances=true)
-- compiled from its sources into oracle/_ref/libcurplsh_ref.so, driven as
IndexBF::add/search do (oracle/ref_driver.cu) -- on cuda:0 for each case below
and saves (distances, indices) with a SHA-256 of the inputs, which the tests
regenerate with curplsh_b200/synth.py (numpy backend) and compare against.

    python tests/golden/gen_ref_fixtures.py [--out DIR]     # needs a GPU

Cases (all inputs seeded, see synth.py):
  ref_c0        uniform [0,1) N=10,000, Q=100, d=128, k=10 (the whole workload)
  ref_c1_sub    integer Gaussian mixture N=1,000,000, d=128, k=100, first 256 queries
  ref_c2_sub    unit-sphere mixture N=10,000,000, d=96 (zero-padded to 128 for the
                reference), k=10, first 256 queries
  ref_k1024     N(0,1) rounded to BF16, N=20,000, Q=64, d=128, k=1024 (the largest k)
  ref_k2        uniform N=3,000, Q=40, d=128, k=2 (the smallest k the reference runs)
  ref_ragged    uniform N=1,003 (not a multiple of 8: host FP32 norms), Q=19, d=128, k=10
"""
from __future__ import annotations

import argparse
import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def load_synth():
    import importlib.util
    spec = importlib.util.spec_from_file_location("curplsh_synth", os.path.join(ROOT, "curplsh_b200", "synth.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.float32).tobytes())
    return h.hexdigest()


def cases(synth):
    """name -> (description dict, generator returning (base, queries, k))."""
    return {
        "ref_c0": ({"gen": "make", "workload": "uniform_small", "q": 100},
                   lambda: synth.make("uniform_small")),
        "ref_c1_sub": ({"gen": "make", "workload": "mixture_int_1m", "q": 256},
                       lambda: synth.make("mixture_int_1m", q=256)),
        "ref_c2_sub": ({"gen": "make", "workload": "sphere_10m", "q": 256},
                       lambda: synth.make("sphere_10m", q=256)),
        "ref_k1024": ({"gen": "normal_bf16", "n": 20000, "q": 64, "d": 128, "k": 1024, "seed": 61},
                      lambda: (synth.normal_bf16(20000, 128, 61), synth.normal_bf16(64, 128, 62), 1024)),
        "ref_k2": ({"gen": "uniform", "n": 3000, "q": 40, "d": 128, "k": 2, "seed": 71},
                   lambda: (*synth.uniform(3000, 40, 128, seed=71), 2)),
        "ref_ragged": ({"gen": "uniform", "n": 1003, "q": 19, "d": 128, "k": 10, "seed": 81},
                       lambda: (*synth.uniform(1003, 19, 128, seed=81), 10)),
    }


def regenerate(synth, meta: dict):
    """Inputs of a fixture from its stored description."""
    g = str(meta["gen"])
    if g == "make":
        return synth.make(str(meta["workload"]), q=int(meta["q"]))
    if g == "normal_bf16":
        s = int(meta["seed"])
        return (synth.normal_bf16(int(meta["n"]), int(meta["d"]), s),
                synth.normal_bf16(int(meta["q"]), int(meta["d"]), s + 1), int(meta["k"]))
    if g == "uniform":
        b, q = synth.uniform(int(meta["n"]), int(meta["q"]), int(meta["d"]), seed=int(meta["seed"]))
        return b, q, int(meta["k"])
    raise KeyError(g)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--only", default="", help="comma-separated case names")
    a = ap.parse_args()
    from oracle import ref
    synth = load_synth()
    os.makedirs(a.out, exist_ok=True)
    only = set(x for x in a.only.split(",") if x)
    for name, (meta, gen) in cases(synth).items():
        if only and name not in only:
            continue
        t0 = time.time()
        base, queries, k = gen()
        t1 = time.time()
        db = ref.Database(base)
        dist, idx, e2e, resident = db.search(queries, k)
        db.close()
        np.savez_compressed(os.path.join(a.out, name + ".npz"), dist=dist, idx=idx, k=k,
                            input_sha256=digest(base, queries), **{"meta_" + key: v for key, v in meta.items()})
        print(f"{name}: N={base.shape[0]} Q={queries.shape[0]} d={base.shape[1]} k={k} gen {t1 - t0:.1f}s "
              f"reference search {resident:.1f} ms", flush=True)


if __name__ == "__main__":
    main()
