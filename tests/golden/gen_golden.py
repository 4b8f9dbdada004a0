"""Generate the golden fixtures under tests/golden/.

Run from the repository root:  python tests/golden/gen_golden.py

ref_smoke_patterns.npz -- known answers of the reference's own smoke programs,
derived analytically (NOT from the oracle), so they pin the oracle:

* test/test_search.cpp:12-36 -- numBases=1000, numQueries=100, dim=128, k=10,
  every query is all ones, base row i is min(i, 10) in every coordinate.  The
  squared distance of row i is 128 * (min(i,10) - 1)^2.  The program itself
  calls searchL2Distance(..., computeExactDistances=false), which omits
  ||q||^2 = 128, i.e. 128 * (m^2 - 2m); IndexBF::search passes true
  (src/index_bf.cpp:68-69).  Rows 0 and 2 tie at the second position; the
  reference leaves that order unspecified, the lower-index rule gives 0 then 2.
* test/test_norm.cpp:15-22 -- all-ones [num x dim] input; every squared norm
  equals dim.  (num, dim) come from argv there; a spread of shapes is stored.

random_small.npz -- a seeded uniform [0,1) case (N=2000, Q=37, d=128, k=10)
with the oracle's FP64 answer, used as a regression fixture for the GPU path.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def search_pattern():
    n, nq, d, k = 1000, 100, 128, 10
    m = np.minimum(np.arange(n), 10).astype(np.float64)
    exact = d * (m - 1.0) ** 2            # ||q - x||^2
    relative = d * (m * m - 2.0 * m)      # ||x||^2 - 2 q.x
    order = np.lexsort((np.arange(n), exact))[:k]
    return dict(
        search_n=np.int64(n), search_nq=np.int64(nq), search_d=np.int64(d), search_k=np.int64(k),
        search_idx=np.tile(order.astype(np.int64), (nq, 1)),
        search_dist_exact=np.tile(exact[order], (nq, 1)),
        search_dist_relative=np.tile(relative[order], (nq, 1)),
    )


def norm_pattern():
    shapes = np.array([[1, 1], [7, 32], [100, 96], [33, 128], [64, 256], [5, 513], [3, 1024]], dtype=np.int64)
    return dict(norm_shapes=shapes)


def random_small():
    import oracle

    rng = np.random.default_rng(20240611)
    n, nq, d, k = 2000, 37, 128, 10
    base = rng.random((n, d), dtype=np.float32)
    queries = rng.random((nq, d), dtype=np.float32)
    dist, idx = oracle.knn(base, queries, k + 1)
    return dict(seed=np.int64(20240611), n=np.int64(n), nq=np.int64(nq), d=np.int64(d), k=np.int64(k),
                base=base, queries=queries, idx=idx, dist=dist)


def main():
    np.savez_compressed(os.path.join(HERE, "ref_smoke_patterns.npz"), **search_pattern(), **norm_pattern())
    np.savez_compressed(os.path.join(HERE, "random_small.npz"), **random_small())
    print("wrote", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))


if __name__ == "__main__":
    main()
