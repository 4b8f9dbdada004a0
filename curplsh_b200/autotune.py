"""Autotuner of the fused pass's launch parameters (no counterpart in the
reference, whose tile sizes are fixed: src/internal/search.cu:12-77).

Per (precision, dim, k bucket, query-count bucket) it picks, by timing on the
device with CUDA events, the two parameters that change speed and never
results (include/curplsh_b200.h, "launch tuning"):

* ``split_q4`` -- the longest run of database tiles one candidate pool covers,
  in quarters of the search's own CTA range (split-N);
* ``pool_headroom`` -- the candidate-pool slack (k-select width).

Coordinate search: the split first (default headroom), then the headroom with
the best split.  Every candidate's output is compared with the default's and
must be identical.  Results are cached in a JSON file keyed by GPU name,
driver version and library version, and loaded back into the library's table
with :func:`load`.
"""
from __future__ import annotations

import json
import os

import curplsh_b200 as cb

SPLITS = (1, 2, 3, 4)  # 4 = whole CTA ranges; a unit is never longer than its range
HEADROOMS = (128, 256, 512, 1024)
DEFAULT = (4, 256)


def default_cache_path() -> str:
    return os.environ.get("CURPLSH_B200_TUNE_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "curplsh_b200", "tuning.json")


def device_key(device: int = 0) -> str:
    """GPU name + driver version + library version."""
    import torch
    name = torch.cuda.get_device_name(device)
    driver = "unknown"
    try:
        import pynvml
        pynvml.nvmlInit()
        driver = pynvml.nvmlSystemGetDriverVersion()
        driver = driver.decode() if isinstance(driver, bytes) else driver
    except Exception:
        pass
    return f"{name}|driver {driver}|{cb.version()}"


def bucket(precision: int, dim: int, k: int, nq: int) -> str:
    kb = max(0, (int(k) - 1).bit_length())
    qb = max(1, int(nq)).bit_length() - 1
    return f"{precision},{dim},{kb},{qb}"


def _time_search(index, queries, k, precision, idx, dist, stream, reps):
    import torch
    nq = int(queries.shape[0])
    index.search_ex(nq, queries, k, idx, dist, precision, stream=stream)  # warm-up (and lazy set-up)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    stream.synchronize()
    e0.record(stream)
    for _ in range(reps):
        index.search_ex(nq, queries, k, idx, dist, precision, stream=stream)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def tune(index, queries, k: int, precision: int = -1, reps: int = 3, stream=None) -> dict:
    """Tunes the bucket of (index dim, k, len(queries)) with `queries` (a CUDA
    float32 tensor on the index's device), installs the winner in the library
    and returns {"bucket", "split_q4", "pool_headroom", "ms", "default_ms",
    "candidates"}."""
    import torch
    dev = queries.device
    stream = stream or torch.cuda.Stream(device=dev)
    form = index.config.precision if precision < 0 else precision
    dim = index.getDimension()
    nq = int(queries.shape[0])
    idx = torch.empty((nq, k), dtype=torch.int32, device=dev)
    dist = torch.empty((nq, k), dtype=torch.float32, device=dev)
    ref_i = torch.empty_like(idx)
    ref_d = torch.empty_like(dist)

    def run(split, head):
        cb.tuning_set(form, dim, k, nq, split, head)
        ms = _time_search(index, queries, k, form, idx, dist, stream, reps)
        if not (torch.equal(idx, ref_i) and torch.equal(dist, ref_d)):
            raise RuntimeError(f"tuning candidate split_q4={split} headroom={head} changed the results")
        return ms

    cb.tuning_set(form, dim, k, nq, *DEFAULT)
    index.search_ex(nq, queries, k, ref_i, ref_d, form, stream=stream)
    stream.synchronize()
    cands = {}
    for s in SPLITS:
        cands[(s, DEFAULT[1])] = run(s, DEFAULT[1])
    best_s = min((v, key) for key, v in cands.items())[1][0]
    for h in HEADROOMS:
        if (best_s, h) not in cands:
            cands[(best_s, h)] = run(best_s, h)
    best_ms, best = min((v, key) for key, v in cands.items())
    cb.tuning_set(form, dim, k, nq, *best)
    return {"bucket": bucket(form, dim, k, nq), "split_q4": best[0], "pool_headroom": best[1], "ms": best_ms,
            "default_ms": cands[DEFAULT],
            "candidates": {f"{a},{b}": v for (a, b), v in sorted(cands.items())}}


def tune_batch(items, precision: int = -1, reps: int = 3, stream=None) -> list:
    """Tunes every bucket a SearchBatch over `items` ((index, queries, k,
    indices, distances) tuples) will look up: the batch concatenates the
    queries of items with the same index and k, so each (index, k) group is
    tuned with its concatenated queries."""
    import torch
    groups = {}
    for ix, q, k, _, _ in items:
        if int(q.shape[0]) == 0:
            continue
        groups.setdefault((id(ix), int(k)), (ix, []))[1].append(q)
    out = []
    for (_, k), (ix, qs) in groups.items():
        out.append(tune(ix, torch.cat(qs), k, precision, reps, stream))
    return out


def save(records, path: str | None = None, device: int = 0) -> str:
    """Merges tune() records into the JSON cache under this GPU's key."""
    path = path or default_cache_path()
    data = {}
    if os.path.exists(path):
        with open(path) as f:
            data = json.load(f)
    entry = data.setdefault(device_key(device), {})
    for r in records:
        entry[r["bucket"]] = {"split_q4": r["split_q4"], "pool_headroom": r["pool_headroom"], "ms": r["ms"]}
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    return path


def load(path: str | None = None, device: int = 0) -> int:
    """Installs the cached parameters of this GPU into the library; returns how many."""
    path = path or default_cache_path()
    if not os.path.exists(path):
        return 0
    with open(path) as f:
        data = json.load(f)
    n = 0
    for key, v in data.get(device_key(device), {}).items():
        form, dim, kb, qb = (int(x) for x in key.split(","))
        cb.tuning_set(form, dim, 1 << kb, 1 << qb, int(v["split_q4"]), int(v["pool_headroom"]))
        n += 1
    return n
