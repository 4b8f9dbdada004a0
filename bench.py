"""Benchmark: exact L2 kNN search throughput on one B200 (or N replicas).

Headline workload (one "step" = one IndexBF search of the whole query batch):
the integer Gaussian mixture -- N = 1,000,000 database rows, Q = 10,000
queries, d = 128, k = 100, integer-valued FP32 data from 1,000 centroids
(seeded SplitMix64 / Box-Muller inputs, curplsh_b200/synth.py).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload mixture_int_1m|uniform_small|sphere_10m|batched_uneven|serving]
                    [--configs uniform_small,sphere_10m,batched_uneven,serving,reference_gpu | none]

Prints ONE JSON line (rank 0).  `value` is queries/s of the headline form
(BF16 coarse + exact FP32 rerank) with queries resident in HBM, kernels timed
with CUDA events on the launching stream; `e2e` is the same metric through
the C ABI call a user makes (IndexBF.search with pinned host queries and
results), timed on the host clock around the call.  Every form's recall@k is
checked against the FP64 oracle on a query subsample; `cpu_baseline` times
that oracle on the host cores.  On one GPU the same line carries a record per
other workload (`configs`): the uniform 10k-row case, the 10M-row unit-sphere
case (FP8 + rerank vs FP32-exact), the uneven batch over 8 databases in one
graph replay, the serving loop (p50/p99 latency), and the reference's own
search path (cuRPLSH searchL2Distance, built from its sources) timed on the
same GPU in a subprocess.

Multi-GPU (torchrun): each rank searches its own query batch against a
replicated database (weak scaling, no collective on the data path); timing is
the max over ranks; the per-workload records are skipped.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "mixture_int_1m"
FORMS = {0: "fp32_exact", 1: "bf16_rerank", 2: "fp8_rerank"}
RECALL_SAMPLE = 128       # queries checked against the oracle per form
METRIC = "queries/s at recall@k=1.0"
# single-search workloads: headline form, forms timed, data description
WORKLOADS = {
    "mixture_int_1m": {"headline": 1, "forms": "0,1,2",
                       "data": "synthetic (seeded Gaussian mixture, 1000 centroids, sigma 12, integer-valued FP32)",
                       "l2": "database (0.5 GB FP32 + 0.5 GB BF16 copies) larger than L2"},
    "uniform_small": {"headline": 1, "forms": "0,1",
                      "data": "synthetic (seeded i.i.d. uniform [0,1) FP32)",
                      "l2": "database (5 MB) fits in L2: latency-bound"},
    "sphere_10m": {"headline": 2, "forms": "0,2",
                   "data": "synthetic (seeded Gaussian mixture on the unit sphere, 4096 centroids, sigma 0.05)",
                   "l2": "database (3.8 GB FP32, 1.0 GB FP8 copy) larger than L2"},
}
SUB_CONFIGS = ("uniform_small", "sphere_10m", "batched_uneven", "serving", "reference_gpu")


def load_synth():
    """curplsh_b200/synth.py by file path (importing the package would load the library)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("curplsh_synth", os.path.join(ROOT, "curplsh_b200", "synth.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), d.get("bf16_tflops_sustained"), "measured"
    return 6650.0, 1590.0, 1400.0, "fallback"


def measure_fp8_peak(dev):
    """Dense FP8-E4M3 GEMM throughput of the library GEMM on this GPU (torch._scaled_mm,
    8192^3, BF16 output), timed like the BF16 peak: warm-up, then CUDA events."""
    import torch
    try:
        n = 8192
        a = torch.randn((n, n), device=dev).to(torch.float8_e4m3fn)
        b = torch.randn((n, n), device=dev).to(torch.float8_e4m3fn).t()
        one = torch.ones((), device=dev)
        for _ in range(3):
            torch._scaled_mm(a, b, scale_a=one, scale_b=one, out_dtype=torch.bfloat16)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 20
        e0.record()
        for _ in range(reps):
            torch._scaled_mm(a, b, scale_a=one, scale_b=one, out_dtype=torch.bfloat16)
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1) / reps
        del a, b
        return 2.0 * n ** 3 / (ms / 1e3) / 1e12, "measured fp8 burst (torch._scaled_mm, 8192^3)"
    except Exception as e:  # noqa: BLE001
        return None, f"fp8 GEMM unavailable ({type(e).__name__})"


def load_traffic(workload, form_name):
    """DRAM bytes per fused launch from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "fused_knn_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    return d.get(workload, {}).get(form_name)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""

    def __init__(self, index=0, interval_ms=50, settle_s=0.25):
        self.index = index
        self.interval_ms = interval_ms
        self.settle_s = settle_s  # nvidia-smi's start-up (device queries) ends before the timed work
        self.proc = None
        self.lines = []

    def __enter__(self):
        cmd = ["nvidia-smi", "-i", str(self.index),
               "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
               "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
               "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
               "--format=csv,noheader,nounits", "-lms", str(self.interval_ms)]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        time.sleep(self.settle_s)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def form_peak(form, bf16_burst, fp8_peak):
    """(TF/s, basis) the fused pass of a form is compared with."""
    if form == 0:
        return bf16_burst / 3.0, "bf16 burst / 3 (three BF16 products)"
    if form == 2:
        if fp8_peak[0]:
            return fp8_peak[0], fp8_peak[1]
        return 2.0 * bf16_burst, "nominal 2 x bf16 burst (" + fp8_peak[1] + ")"
    return bf16_burst, "bf16 burst"


# --------------------------------------------------------------------- reference arm
def run_reference(args, world, rank):
    """--impl reference: the reference ships no CPU search of its own; its search
    semantics (src/internal/search.cu:79-216) are restated by the FP64 host
    oracle, timed here on all host cores over a bounded query sample per step.
    Inputs come from synth.py loaded by path: the curplsh_b200 library is not
    loaded by this arm."""
    if rank != 0:
        return 0
    import oracle
    synth = load_synth()
    wl = args.workload if args.workload in WORKLOADS else WORKLOAD
    n_db, n_q, dim, _ = synth.CONFIGS[wl]
    sample = 128
    need = sample * (args.warmup + args.steps)
    base_h, q_h, k = synth.make(wl, q=min(n_q, need))  # numpy backend: the first rows of the full draw
    for w in range(args.warmup):
        oracle.knn(base_h, q_h[(w * sample) % q_h.shape[0]:][:sample], k)
    times = []
    for s in range(args.steps):
        off = ((args.warmup + s) * sample) % max(1, q_h.shape[0] - sample)
        t0 = time.perf_counter()
        oracle.knn(base_h, q_h[off:off + sample], k)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    qps = sample * args.steps / total
    cores = oracle.num_threads()
    line = {
        "impl": "reference", "metric": METRIC, "value": qps, "unit": "queries/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": WORKLOADS[wl]["data"],
        "config": {"workload": wl, "N": n_db, "Q": n_q, "d": dim, "k": k, "q_per_step_sample": sample,
                   "seed": synth.SEEDS[wl]},
        "cpu_baseline": {"value": qps, "unit": "queries/s", "cores": cores, "kind": "port",
                         "sample": f"{sample} queries per step against all {n_db} rows"},
        "e2e": {"value": qps, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference ships no CPU search; this arm times the FP64 restatement of its searchL2Distance "
                "semantics (oracle/knn_oracle.c) on the host cores. The reference's own GPU path is timed on the "
                "same GPU in the main arm's configs.reference_gpu record",
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------- one workload, several forms
def run_single(cb, synth, wl, args, world, rank, local, res, peaks, fp8_peak, with_clocks, forms=None):
    """Times every form of one single-search workload; returns its record."""
    import numpy as np
    import torch

    import oracle
    dev = f"cuda:{local}"
    info = WORKLOADS[wl]
    n_db, _, dim, _ = synth.CONFIGS[wl]
    if args.rows:  # a smaller case of the same workload (profiling captures)
        n_db = args.rows
    # every rank holds the same database and searches a full query batch (replicas)
    base, queries, k = synth.make(wl, backend="torch", device=dev, n=args.rows or None, q=args.queries or None)
    torch.cuda.synchronize()  # generated on torch's stream; the library orders its work on its own streams
    stream = torch.cuda.Stream(device=dev)
    Q = queries.shape[0]
    oi = torch.empty((Q, k), dtype=torch.int32, device=dev)
    od = torch.empty((Q, k), dtype=torch.float32, device=dev)

    # ---- recall of every form on a query subsample (rank 0), and the CPU baseline
    n_sub = min(RECALL_SAMPLE, Q)
    sub = torch.arange(0, Q, max(1, Q // n_sub), device=dev)[:n_sub]
    form_results = {}
    cpu = None
    base_h = qs_h = rd = None
    if rank == 0 and not args.no_recall:
        base_h = base.cpu().numpy()
        qs_h = queries[sub].cpu().numpy()
        t0 = time.perf_counter()
        rd, ri = oracle.knn(base_h, qs_h, k + 1)
        dt = time.perf_counter() - t0
        cpu = {"value": n_sub / dt, "unit": "queries/s", "cores": oracle.num_threads(), "kind": "port",
               "sample": f"{n_sub} queries against all {n_db} rows (FP64 oracle, OpenMP)"}
    forms = forms or [int(f) for f in (args.forms or info["forms"]).split(",") if f != ""]
    headline = info["headline"] if info["headline"] in forms else forms[0]
    indexes = {}
    for form in forms:
        ix = cb.IndexBF(res, dim, cb.IndexBFConfig(device=local, precision=form))
        ix.add(n_db, base)
        indexes[form] = ix
        fb0, cf0 = ix.fallback_count(), ix.coarse_fallback_count()
        ix.search_ex(Q, queries, k, oi, od, stream=stream)
        stream.synchronize()
        if rank == 0 and not args.no_recall:
            gi = oi[sub].cpu().numpy()
            gd = od[sub].cpu().numpy().astype(np.float64)
            rec, _ = oracle.recall_at_k(base_h, qs_h, gi, rd[:, :k])
            err = float(np.max(np.abs(gd - rd[:, :k]) / np.maximum(np.abs(rd[:, :k]), 1e-30)))
            form_results[FORMS[form]] = {"recall_at_k": rec, "max_rel_dist_err": err,
                                         "estimate_failed_queries": ix.fallback_count() - fb0,
                                         "coarse_check_failed_queries": ix.coarse_fallback_count() - cf0}

    # ---- timed region: device-resident queries, CUDA events on our stream
    flops = 2.0 * Q * n_db * dim
    timing, estimates, clocks = {}, {}, None

    def timed_searches(ix, steps):
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            ix.search_ex(Q, queries, k, oi, od, stream=stream)
        ev1.record(stream)
        ev1.synchronize()
        return ev0.elapsed_time(ev1) / steps

    for form in forms:
        ix = indexes[form]
        for _ in range(args.warmup):
            ix.search_ex(Q, queries, k, oi, od, stream=stream)
        stream.synchronize()
        barrier(world)
        sampler = ClockSampler(local) if (with_clocks and form == headline) else None
        if sampler:
            sampler.__enter__()
        fb0 = ix.fallback_count() + ix.coarse_fallback_count()
        ms = timed_searches(ix, args.steps)
        fb = ix.fallback_count() + ix.coarse_fallback_count() - fb0
        if sampler:
            sampler.__exit__(None, None, None)
            clocks = sampler.summary()
        ms = max_over_ranks(ms, world)
        passes = ix.search_profiled(Q, queries, k, oi, od, stream=stream)
        fused_ms = max_over_ranks(passes["fused_ms"], world)
        timing[form] = (ms, fused_ms, passes)
        rows, step, rank_r = ix.estimate_plan(Q, k, form)
        est = {"sample_rows": rows, "step": step, "rank": rank_r}
        if rows and not args.quick:
            cb.set_bound_estimate(False)
            for _ in range(2):
                ix.search_ex(Q, queries, k, oi, od, stream=stream)
            est["ms_per_search_without"] = max_over_ranks(timed_searches(ix, max(1, args.steps // 2)), world)
            cb.set_bound_estimate(True)
        estimates[form] = (est, fb)

    # ---- end to end through the C ABI: pinned host queries in, host results out,
    # host clock around the call (IndexBF::search with host pointers)
    qh = torch.empty((Q, dim), dtype=torch.float32, pin_memory=True)
    qh.copy_(queries.cpu())
    ih = torch.empty((Q, k), dtype=torch.int32, pin_memory=True)
    dh = torch.empty((Q, k), dtype=torch.float32, pin_memory=True)
    ix = indexes[headline]
    for _ in range(args.warmup):
        ix.search(Q, qh, k, ih, dh)
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ix.search(Q, qh, k, ih, dh)
    e2e = max_over_ranks((time.perf_counter() - t0) / args.steps * 1e3, world)

    hbm, bf16_burst, bf16_sust, peak_kind = peaks
    forms_out = {}
    for form in forms:
        name = FORMS[form]
        f_ms, f_fused, f_passes = timing[form]
        p_form, basis = form_peak(form, bf16_burst, fp8_peak)
        est, fb = estimates[form]
        forms_out[name] = {
            "queries_per_s": Q * world / (f_ms / 1e3), "ms_per_search": f_ms, "fused_ms": f_fused,
            "fused_tflops": flops / (f_fused / 1e3) / 1e12,
            "roofline_frac": flops / (f_fused / 1e3) / 1e12 / p_form, "peak_basis_tflops": p_form,
            "peak_basis": basis, "bound_estimate": est, "queries_searched_again_timed": fb,
            "passes_ms": f_passes, **form_results.get(name, {}),
        }
    ms, fused_ms, passes = timing[headline]
    p_head, basis_head = form_peak(headline, bf16_burst, fp8_peak)
    achieved = flops / (fused_ms / 1e3) / 1e12
    rec = form_results.get(FORMS[headline], {}).get("recall_at_k")
    sample_rows = estimates[headline][0]["sample_rows"]
    launches = {"prep_rows_kernel": 1, "fused_knn_kernel": 2 if sample_rows else 1,
                "estimate_select_kernel": 1 if sample_rows else 0, "merge_rerank_kernel": 1}
    out = {
        "workload": wl, "value": Q * world / (ms / 1e3), "ms_per_step": ms,
        "dtype": FORMS[headline].split("_")[0], "data": info["data"],
        "config": {"workload": wl, "N": n_db, "Q": Q, "d": dim, "k": k, "form": FORMS[headline],
                   "kprime": {"bf16_rerank": "2k (coarse-margin check on)", "fp8_rerank": "max(4k, 480)", "fp32_exact": "k + 16", "rounding": "up to a multiple of 32"}, "l2": info["l2"], "seed": synth.SEEDS[wl],
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "recall_at_k": rec, "recall_ok": rec is not None and rec >= 1.0,
        "forms": forms_out,
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": p_head, "unit": "TFLOP/s",
                     "frac": achieved / p_head, "traffic": load_traffic(wl, FORMS[headline]),
                     "kernel": f"fused_knn_kernel<{FORMS[headline]}>",
                     "peak_kind": (peak_kind + " " + basis_head) if headline != 2 else basis_head,
                     "algorithmic": "2*Q*N*d flops per launch"},
        "cpu_baseline": cpu,
        "e2e": {"value": Q * world / (e2e / 1e3), "unit": "queries/s", "ms_per_step": e2e,
                "timing": "host clock around IndexBF.search (C ABI), pinned host buffers",
                "h2d_bytes_per_step": Q * dim * 4, "d2h_bytes_per_step": Q * k * 8},
        "gpu_launches": sum(launches.values()) * args.steps, "launches_per_step": launches,
        "clocks": clocks,
    }
    for ix in indexes.values():
        ix.close()
    del base, queries
    torch.cuda.empty_cache()
    return out


# --------------------------------------------------------------------- uneven batch (one graph)
def run_batched(cb, synth, args, world, rank, local, res, peaks):
    """64 query batches of log-uniform size 1-4096 over 8 resident databases
    (N log-uniform 10k-2M, d in {64,128,256,512}, k in {1,10,100,1024}, N(0,1)
    data rounded to BF16), one step = one replay of the captured batch graph.
    Compared with the same items searched one by one."""
    import numpy as np
    import torch

    import oracle
    dev = f"cuda:{local}"
    dbs_spec, batches = synth.batched_uneven_spec(seed=synth.SEEDS["batched_uneven"])
    stream = torch.cuda.Stream(device=dev)
    precision = args.batch_form
    dbs = []
    for i, (n, d) in enumerate(dbs_spec):
        x = synth.normal_bf16(n, d, seed=100 + i, backend="torch", device=dev)
        ix = cb.IndexBF(res, d, cb.IndexBFConfig(device=local, precision=precision))
        ix.add(n, x)
        dbs.append((ix, x))
    items = []
    for j, (db, nq, k) in enumerate(batches):
        ix, x = dbs[db]
        q = synth.normal_bf16(nq, x.shape[1], seed=1000 + j + 7919 * rank, backend="torch", device=dev)
        items.append((ix, q, k, torch.empty((nq, k), dtype=torch.int32, device=dev),
                      torch.empty((nq, k), dtype=torch.float32, device=dev)))
    torch.cuda.synchronize()
    total_q = sum(it[1].shape[0] for it in items)
    tuned = None
    if args.tune:
        from curplsh_b200 import autotune
        cb.tuning_clear()
        recs = autotune.tune_batch(items, precision=precision, reps=2, stream=stream)
        tuned = {"buckets": len(recs),
                 "changed": sum(1 for r in recs if (r["split_q4"], r["pool_headroom"]) != autotune.DEFAULT)}
    batch = cb.SearchBatch(items, precision=precision)
    kernels, ws_bytes = batch.info()
    batch.run(stream=stream)
    mismatches = 0
    recall_min, err_max = 1.0, 0.0
    for j, (ix, q, k, oi, od) in enumerate(items):
        ai = torch.empty_like(oi)
        ad = torch.empty_like(od)
        ix.search_ex(q.shape[0], q, k, ai, ad, precision, stream=stream)
        stream.synchronize()
        if not (torch.equal(ai, oi) and torch.equal(ad, od)):
            mismatches += 1
        if rank == 0 and not args.no_recall and j % 8 == 0:
            x = dbs[batches[j][0]][1]
            qs = q[:4].cpu().numpy()
            rd, ri = oracle.knn(x.cpu().numpy(), qs, k)
            rec, _ = oracle.recall_at_k(x.cpu().numpy(), qs, oi[:4].cpu().numpy(), rd)
            gd = od[:4].cpu().numpy().astype(np.float64)
            ok = ri >= 0
            err = float(np.max(np.abs(gd[ok] - rd[ok]) / np.maximum(np.abs(rd[ok]), 1e-30))) if ok.any() else 0.0
            recall_min = min(recall_min, rec)
            err_max = max(err_max, err)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        stream.synchronize()
        barrier(world)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return max_over_ranks(e0.elapsed_time(e1) / args.steps, world)

    ms_graph = timed(lambda: batch.run(stream=stream, wait=False))
    # the other form's graph over the same items: its replay time, and its
    # results must equal this form's (both rerank exactly)
    other = 1 - precision if precision in (0, 1) else 1
    alt_batch = cb.SearchBatch(items, precision=other)
    ref_out = [(it[3].clone(), it[4].clone()) for it in items]
    alt_batch.run(stream=stream)
    alt_same = all(torch.equal(a, it[3]) and torch.equal(b, it[4]) for (a, b), it in zip(ref_out, items))
    ms_alt = timed(lambda: alt_batch.run(stream=stream, wait=False))
    alt_batch.close()
    del ref_out

    def one_by_one():
        for ix, q, k, oi, od in items:
            ix.search_ex(q.shape[0], q, k, oi, od, precision, stream=stream)
    ms_loop = timed(one_by_one)
    qh = [torch.empty(tuple(it[1].shape), dtype=torch.float32, pin_memory=True).copy_(it[1].cpu()) for it in items]
    ih = [torch.empty(tuple(it[3].shape), dtype=torch.int32, pin_memory=True) for it in items]
    dh = [torch.empty(tuple(it[4].shape), dtype=torch.float32, pin_memory=True) for it in items]

    def e2e_step():
        with torch.cuda.stream(stream):
            for it, h in zip(items, qh):
                it[1].copy_(h, non_blocking=True)
            batch.run(stream=stream, wait=False)
            for it, a, b in zip(items, ih, dh):
                a.copy_(it[3], non_blocking=True)
                b.copy_(it[4], non_blocking=True)
        stream.synchronize()
    for _ in range(args.warmup):
        e2e_step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    ms_e2e = max_over_ranks((time.perf_counter() - t0) / args.steps * 1e3, world)
    # Roofline: per database, the tensor time of all its queries or one stream of
    # its BF16 rows, whichever is longer (small batches are HBM-bound).
    hbm, bf16_burst, _, peak_kind = peaks
    p_form = form_peak(precision, bf16_burst, (None, "nominal"))[0]
    t_roof = 0.0
    per_db_q = {}
    for (db, nq, k) in batches:
        per_db_q[db] = per_db_q.get(db, 0) + nq
    for db, nq in per_db_q.items():
        n, d = dbs_spec[db]
        flops_db = 2.0 * nq * n * d
        bytes_db = n * (d + 6) * 2.0 + 4.0 * n + 4.0 * nq * d
        t_roof += max(flops_db / (p_form * 1e12), bytes_db / (hbm * 1e9))
    out = {
        "workload": "batched_uneven", "value": total_q * world / (ms_graph / 1e3), "ms_per_step": ms_graph,
        "dtype": FORMS[precision].split("_")[0], "data": "synthetic (seeded N(0,1) rounded to BF16, stored FP32)",
        "config": {"workload": "batched_uneven", "databases": [{"N": n, "d": d} for n, d in dbs_spec],
                   "batches": len(batches), "queries_per_step": total_q,
                   "k_values": sorted({b[2] for b in batches}), "form": FORMS[precision],
                   "seed": synth.SEEDS["batched_uneven"], "l2": "databases (3.1 GB) larger than L2"},
        "one_by_one": {"queries_per_s": total_q * world / (ms_loop / 1e3), "ms_per_step": ms_loop},
        "other_form": {"form": FORMS[other], "ms_per_step": ms_alt, "queries_per_s": total_q * world / (ms_alt / 1e3),
                       "identical_results": alt_same},
        "batch_speedup": ms_loop / ms_graph,
        "identical_to_alone": mismatches == 0, "items_differing": mismatches,
        "recall_at_k_min_sampled": recall_min, "max_rel_dist_err_sampled": err_max,
        "roofline": {"bound": "per database: max(tensor, hbm)", "achieved_ms_roof": t_roof * 1e3,
                     "measured_ms": ms_graph, "frac": t_roof * 1e3 / ms_graph, "unit": "time ratio",
                     "peak": {"tensor_tflops": p_form, "hbm_gbs": hbm}, "peak_kind": peak_kind,
                     "algorithmic": "sum over databases of max(2*Q*N*d / P_bf16, N*(d+6)*2+4N+4Qd bytes / BW)"},
        "e2e": {"value": total_q * world / (ms_e2e / 1e3), "unit": "queries/s", "ms_per_step": ms_e2e,
                "timing": "host clock around copies in + graph replay + copies out",
                "h2d_bytes_per_step": sum(it[1].numel() * 4 for it in items),
                "d2h_bytes_per_step": sum(it[3].numel() * 8 for it in items)},
        "gpu_launches_per_step": kernels, "workspace_bytes": ws_bytes, "autotune": tuned,
    }
    batch.close()
    for ix, _ in dbs:
        ix.close()
    del dbs, items
    torch.cuda.empty_cache()
    return out


# --------------------------------------------------------------------- serving loop
def run_serving(cb, synth, args, world, rank, local, res):
    """One resident database (N = 5,000,000, d = 256, BF16-valued Gaussian
    mixture of 2,048 centroids), requests of 1-256 queries (log-uniform)
    arriving as a Poisson process, k = 50, queries and results in pinned host
    memory.  For the BF16 + rerank form and the plain FP32-exact form:
    saturated throughput (every request queued at once) and, per offered rate,
    p50 / p99 latency (submit to results in host memory)."""
    import numpy as np
    import torch

    import gc

    import oracle
    dev = f"cuda:{local}"
    # free what earlier workloads left to the garbage collector now, and run
    # no collection during the measurements: freeing a pinned host buffer
    # (cudaFreeHost) takes the driver for milliseconds, and a collection inside
    # a timed load shows up as one slow request or a slower saturated run
    gc.collect()
    torch.cuda.empty_cache()
    gc.disable()
    try:
        return _serving_measure(cb, synth, args, rank, local, res, oracle, dev)
    finally:
        gc.enable()


def _serving_measure(cb, synth, args, rank, local, res, oracle, dev):
    import numpy as np
    import torch
    n, d, k = args.serve_n, 256, 50
    base, qpool = synth.mixture_bf16(n, 20000, d, seed=synth.SEEDS["serving"], backend="torch", device=dev)
    torch.cuda.synchronize()
    ix = cb.IndexBF(res, d, cb.IndexBFConfig(device=local, precision=1))
    ix.add(n, base)
    qpool_h = qpool.cpu().pin_memory()
    rng = np.random.default_rng(17 + rank)

    def request_sizes(count):
        return [int(round(np.exp(rng.uniform(0.0, np.log(256))))) for _ in range(count)]

    def make_outputs(sizes):
        return [(torch.empty((m, k), dtype=torch.int32).pin_memory(), torch.empty((m, k)).pin_memory())
                for m in sizes]

    def run_load(srv, sizes, arrivals):
        outs = make_outputs(sizes)
        offs = np.cumsum([0] + sizes[:-1]) % (qpool_h.shape[0] - 256)
        qs = [qpool_h[o:o + m] for o, m in zip(offs, sizes)]
        tickets = [None] * len(sizes)
        lat = [None] * len(sizes)
        phases = [None] * len(sizes)
        done = threading.Event()

        def waiter():
            for i in range(len(sizes)):
                while tickets[i] is None:
                    time.sleep(20e-6)
                r = srv.wait_phases(tickets[i], timeout=600.0)
                lat[i] = r[0]
                phases[i] = r[1:]
            done.set()

        th = threading.Thread(target=waiter)
        th.start()
        t0 = time.perf_counter()
        for i, m in enumerate(sizes):
            due = t0 + arrivals[i]
            while True:
                now = time.perf_counter()
                if now >= due:
                    break
                time.sleep(min(due - now, 500e-6))
            tickets[i] = srv.submit(qs[i], k, outs[i][0], outs[i][1])
        done.wait()
        wall = time.perf_counter() - t0
        th.join()
        return np.array(lat), wall, (qs, outs, phases)

    forms_out = {}
    recall = None
    qsample = gsample = None
    for form in (1, 0):
        srv = cb.Server(ix, precision=form, max_inflight=3, max_step_queries=4096, memory_budget=4 << 30)
        sizes = request_sizes(64)
        run_load(srv, sizes, [0.0] * len(sizes))
        sizes = request_sizes(16)
        run_load(srv, sizes, [i * 2e-3 for i in range(len(sizes))])
        # saturated throughput: the median of three runs of 600 requests queued
        # at once (a run lasts ~0.1 s, and a single host-side stall of tens of
        # ms, as seen at the lowest offered rate, would halve one run)
        sat_runs = []
        for rep in range(3):
            sizes = request_sizes(600)
            lat, wall, loaded = run_load(srv, sizes, [0.0] * len(sizes))
            sat_runs.append(sum(sizes) / wall)
            if rep == 0:
                qs, outs, _ = loaded
        sat = statistics.median(sat_runs)
        if form == 1:
            qsample = np.concatenate([qs[i][:1].numpy() for i in range(8)])
            gsample = np.concatenate([outs[i][0][:1].numpy() for i in range(8)])
        per_rate = {}
        for rate in args.serve_rates:
            mean_req = rate / 46.0  # mean of the log-uniform 1..256 request size is ~46 queries
            count = int(min(3000, max(200, mean_req * args.serve_seconds)))
            sizes = request_sizes(count)
            gaps = rng.exponential(1.0 / mean_req, size=count)
            arrivals = np.cumsum(gaps) - gaps[0]
            # half a second of the same load first, not measured: the rate is
            # measured in its steady state, not in the transition from the
            # previous (heavier) load
            wcount = int(max(20, mean_req * 0.5))
            wgaps = rng.exponential(1.0 / mean_req, size=wcount)
            run_load(srv, request_sizes(wcount), list(np.cumsum(wgaps) - wgaps[0]))
            # a slower sampler with a longer settle: each nvidia-smi query takes
            # driver locks that a latency measurement would otherwise see
            sampler = ClockSampler(local, interval_ms=200, settle_s=1.0)
            sampler.__enter__()
            lat, wall, (_, _, ph) = run_load(srv, sizes, list(arrivals))
            sampler.__exit__(None, None, None)
            sm = [float(x.split(",")[0]) for x in sampler.lines if x and x.split(",")[0].strip().replace(".", "").isdigit()]
            slow = np.argsort(-lat)[:3]
            ph = np.array(ph) * 1e3
            per_rate[str(rate)] = {"p50_ms": float(np.percentile(lat, 50) * 1e3),
                                   "p99_ms": float(np.percentile(lat, 99) * 1e3),
                                   "max_ms": float(lat.max() * 1e3),
                                   "phases_p99_ms": {"queued": float(np.percentile(ph[:, 0], 99)),
                                                     "device": float(np.percentile(ph[:, 1], 99)),
                                                     "retire": float(np.percentile(ph[:, 2], 99)),
                                                     "gpu_exec": float(np.percentile(ph[:, 3], 99)),
                                                     "start_lag": float(np.percentile(ph[:, 4], 99))},
                                   "slowest": [[int(i), sizes[i], round(float(lat[i] * 1e3), 3),
                                                [round(float(x), 3) for x in ph[i]]] for i in slow],
                                   "achieved_queries_per_s": sum(sizes) / wall, "requests": count,
                                   "sm_mhz": {"median": statistics.median(sm) if sm else None,
                                              "min": min(sm) if sm else None, "samples": len(sm)}}
        st = srv.stats()
        srv.close()
        forms_out[FORMS[form]] = {"saturated_queries_per_s": sat, "saturated_runs_queries_per_s": sat_runs,
                                  "rates": per_rate, **st}
    if rank == 0 and not args.no_recall:
        base_h = base.cpu().numpy()
        rd, ri = oracle.knn(base_h, qsample, k)
        recall, _ = oracle.recall_at_k(base_h, qsample, gsample, rd)
    b = forms_out["bf16_rerank"]
    out = {
        "workload": "serving", "metric": "serving p50/p99 latency (ms) and queries/s",
        "value": b["saturated_queries_per_s"], "unit": "queries/s", "dtype": "bf16",
        "data": "synthetic (seeded Gaussian mixture, 2048 centroids, BF16-valued)",
        "config": {"workload": "serving", "N": n, "d": d, "k": k, "request_queries": "log-uniform 1-256",
                   "arrivals": "Poisson", "io": "pinned host queries and results", "seed": synth.SEEDS["serving"],
                   "max_inflight": 3, "memory_budget_bytes": 4 << 30},
        "recall_at_k_sampled": recall, "forms": forms_out,
        "bf16_vs_exact_saturated": b["saturated_queries_per_s"] / forms_out["fp32_exact"]["saturated_queries_per_s"],
    }
    ix.close()
    del base, qpool
    torch.cuda.empty_cache()
    return out


# --------------------------------------------------------------------- the reference on the same GPU
def run_reference_gpu(args):
    """The reference's own search path (cuRPLSH computeL2Norm + searchL2Distance,
    compiled from its sources into oracle/_ref) timed on this GPU, one
    subprocess per workload (the reference exits the process on a CUDA error)."""
    from oracle import ref
    if not ref.available():
        return {"unavailable": "oracle/_ref/libcurplsh_ref.so was not built (the reference sources were absent)"}
    out = {"what": "cuRPLSH searchL2Distance(..., exact distances) driven as IndexBF::add/search, cuBLAS SGEMM + "
                   "block select, inputs from the same seeded generator (numpy)",
           "kind": "reference"}
    plan = [("uniform_small", 0, 5), ("mixture_int_1m", 0, 2), ("sphere_10m", 2048, 1)]
    for wl, q, reps in plan:
        cmd = [sys.executable, "-m", "oracle.ref", "--workload", wl, "--reps", str(reps)]
        if q:
            cmd += ["--queries", str(q)]
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=900, cwd=ROOT)
            lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
            out[wl] = json.loads(lines[-1]) if (r.returncode == 0 and lines) else \
                {"error": f"rc={r.returncode}: {r.stderr.strip()[-300:]}"}
        except subprocess.TimeoutExpired:
            out[wl] = {"error": "timed out"}
    return out


# --------------------------------------------------------------------- main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--forms", default=None, help="precision forms to time (0 exact, 1 bf16, 2 fp8)")
    ap.add_argument("--no-recall", action="store_true", help="skip the oracle recall check (profiling runs)")
    ap.add_argument("--quick", action="store_true", help="skip the without-estimate comparison")
    ap.add_argument("--workload", default=WORKLOAD, choices=list(WORKLOADS) + ["batched_uneven", "serving"])
    ap.add_argument("--configs", default=",".join(SUB_CONFIGS),
                    help="per-workload records added to the headline line on one GPU ('none' for none)")
    ap.add_argument("--rows", type=int, default=0,
                    help="single-search workloads: the first ROWS database rows only (small profiling cases)")
    ap.add_argument("--queries", type=int, default=0, help="single-search workloads: the first QUERIES queries only")
    ap.add_argument("--serve-n", type=int, default=5_000_000, help="serving workload: database rows")
    ap.add_argument("--serve-rates", type=lambda v: [int(x) for x in v.split(",")], default=[1000, 5000, 20000, 50000],
                    help="serving workload: offered query rates (queries/s)")
    ap.add_argument("--serve-seconds", type=float, default=2.0, help="serving workload: seconds per rate")
    ap.add_argument("--batch-form", type=int, default=0,
                    help="precision form of the batched workload (the other of 0 / 1 is timed beside it)")
    ap.add_argument("--tune", action="store_true", help="batched workload: autotune its buckets first")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world, rank, local = dist_init()
    if args.impl == "reference":
        rc = run_reference(args, world, rank)
        barrier(world)
        return rc

    # the reference's own GPU path first, in subprocesses, before this process
    # creates its CUDA context (two contexts on one GPU time-slice)
    wanted = [c for c in args.configs.split(",") if c and c != "none"] if world == 1 else []
    ref_gpu = None
    if "reference_gpu" in wanted and args.workload in WORKLOADS:
        t0 = time.perf_counter()
        try:
            ref_gpu = run_reference_gpu(args)
        except Exception as e:  # noqa: BLE001
            ref_gpu = {"error": f"{type(e).__name__}: {e}"[:400]}
        ref_gpu["bench_s"] = time.perf_counter() - t0

    import torch

    import curplsh_b200 as cb
    synth = load_synth()
    torch.cuda.set_device(local)
    dev = f"cuda:{local}"
    res = cb.DeviceResources(local)
    peaks = load_peaks()
    fp8_peak = measure_fp8_peak(dev)
    hbm, bf16_burst, bf16_sust, peak_kind = peaks
    base_line = {"metric": METRIC, "unit": "queries/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                 "higher_is_better": True, "scaling": "weak", "vs_baseline": None}
    if args.workload in ("batched_uneven", "serving"):
        if args.workload == "batched_uneven":
            rec = run_batched(cb, synth, args, world, rank, local, res, peaks)
        else:
            rec = run_serving(cb, synth, args, world, rank, local, res)
        if rank == 0:
            print(json.dumps({**base_line, **rec}), flush=True)
        res.close()
        barrier(world)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return 0

    head = run_single(cb, synth, args.workload, args, world, rank, local, res, peaks, fp8_peak, with_clocks=True)
    configs = {}
    for c in wanted:
        if c == args.workload:
            continue
        if c == "reference_gpu":
            if ref_gpu is not None:
                configs[c] = ref_gpu
            continue
        t0 = time.perf_counter()
        try:
            if c in WORKLOADS:
                r = run_single(cb, synth, c, args, world, rank, local, res, peaks, fp8_peak, with_clocks=False)
            elif c == "batched_uneven":
                r = run_batched(cb, synth, args, world, rank, local, res, peaks)
            elif c == "serving":
                r = run_serving(cb, synth, args, world, rank, local, res)
            else:
                continue
        except Exception as e:  # noqa: BLE001  (a failed sub-record must not lose the headline)
            r = {"error": f"{type(e).__name__}: {e}"[:400]}
        r["bench_s"] = time.perf_counter() - t0
        configs[c] = r
    if rank == 0:
        line = {**base_line, **{k: v for k, v in head.items() if k != "workload"}}
        line["peaks"] = {"hbm_gbs": hbm, "bf16_tflops_burst": bf16_burst, "bf16_tflops_sustained": bf16_sust,
                         "kind": peak_kind, "fp8_tflops": fp8_peak[0], "fp8_kind": fp8_peak[1]}
        if configs:
            line["configs"] = configs
        print(json.dumps(line), flush=True)
    res.close()
    barrier(world)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
