"""Benchmark: exact L2 kNN search throughput on one B200 (or N replicas).

Workload (one "step" = one IndexBF search of the whole query batch): the
Gaussian-mixture configuration -- N = 1,000,000 database rows, Q = 10,000
queries, d = 128, k = 100, integer-valued FP32 data from 1,000 centroids
(seeded synthetic data, see curplsh_b200/synth.py).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload mixture_int_1m|sphere_10m|batched_uneven|serving]

Other workloads: sphere_10m (N = 10,000,000, Q = 10,000, d = 96, k = 10,
unit-sphere mixture, FP8-E4M3 + rerank headline), batched_uneven (64 query
batches over 8 databases in one graph replay) and serving (continuous batching
of Poisson-arriving requests; p50/p99 latency and throughput).

Prints ONE JSON line (rank 0).  `value` is queries/s of the headline form
(BF16 coarse + exact FP32 rerank) with queries resident in HBM, kernels timed
with CUDA events on the launching stream; `e2e` is the same metric through the
C ABI with pinned host buffers (H2D of the queries and D2H of the results inside
the timed region).  Every form's recall@k is checked against the FP64 oracle on
a query subsample; `cpu_baseline` times that oracle on the host cores.

Multi-GPU (torchrun): each rank searches its own query batch against a
replicated database (weak scaling, no collective on the data path); timing is
the max over ranks.
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
# single-search workloads: headline form, forms timed by default, data description
WORKLOADS = {
    "mixture_int_1m": {"headline": 1, "forms": "0,1,2",
                       "data": "synthetic (seeded Gaussian mixture, 1000 centroids, sigma 12, integer-valued FP32)",
                       "l2": "database (1.0 GB FP32 + 0.5 GB BF16 copies) larger than L2"},
    "sphere_10m": {"headline": 2, "forms": "0,2",
                   "data": "synthetic (seeded Gaussian mixture on the unit sphere, 4096 centroids, sigma 0.05)",
                   "l2": "database (3.8 GB FP32, 1.0 GB FP8 copy) larger than L2"},
}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), d.get("bf16_tflops_sustained"), "measured"
    return 6650.0, 1590.0, 1400.0, "fallback"


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

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        cmd = ["nvidia-smi", "-i", str(self.index),
               "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
               "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
               "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
               "--format=csv,noheader,nounits", "-lms", "50"]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        time.sleep(0.25)
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


def cpu_oracle_rate(base_h, q_h, k, nq_sample):
    import oracle
    t0 = time.perf_counter()
    dist_, idx_ = oracle.knn(base_h, q_h[:nq_sample], k + 1)
    dt = time.perf_counter() - t0
    return nq_sample / dt, dist_, idx_, oracle.num_threads()


def run_reference(args, world, rank):
    """--impl reference: the reference has no CPU path of its own; its search
    semantics (search.cu:79-216) are restated by the FP64 host oracle, timed
    here on all host cores over a bounded query sample per step."""
    if rank != 0:
        return 0
    import numpy as np
    import torch

    import oracle
    from curplsh_b200 import synth
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    wl = args.workload if args.workload in WORKLOADS else WORKLOAD
    n_db, n_q, dim, _ = synth.CONFIGS[wl]
    base, queries, k = synth.make(wl, backend="torch", device=dev)
    base_h = base.cpu().numpy()
    q_h = queries.cpu().numpy()
    sample = 128
    for w in range(args.warmup):
        oracle.knn(base_h, q_h[w * sample:(w + 1) * sample], k)
    times = []
    for s in range(args.steps):
        off = ((args.warmup + s) * sample) % (q_h.shape[0] - sample)
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
        "config": {"workload": wl, "N": n_db, "Q": n_q, "d": dim, "k": k, "q_per_step_sample": sample},
        "cpu_baseline": {"value": qps, "unit": "queries/s", "cores": cores, "kind": "port",
                         "sample": f"{sample} queries per step against all {n_db} rows"},
        "e2e": {"value": qps, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference ships no CPU search; this arm times the FP64 restatement of its searchL2Distance "
                "semantics (oracle/knn_oracle.c) on the host cores",
    }
    print(json.dumps(line), flush=True)
    return 0


def run_batched(args, world, rank, local):
    """--workload batched_uneven: 64 query batches of log-uniform size 1-4096
    over 8 resident databases (N log-uniform 10k-2M, d in {64,128,256,512},
    k in {1,10,100,1024}, N(0,1) data rounded to BF16), one step = one replay
    of the captured batch graph.  Compared with the same items searched one by
    one (search_ex in a loop on one stream)."""
    import numpy as np
    import torch

    import curplsh_b200 as cb
    import oracle
    from curplsh_b200 import synth

    torch.cuda.set_device(local)
    dev = f"cuda:{local}"
    dbs_spec, batches = synth.batched_uneven_spec()
    res = cb.DeviceResources(local)
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
    torch.cuda.synchronize()  # the inputs were generated on torch's stream; the library uses its own
    total_q = sum(it[1].shape[0] for it in items)
    flops = sum(2.0 * it[1].shape[0] * dbs[b[0]][1].shape[0] * it[1].shape[1] for it, b in zip(items, batches))
    tuned = None
    if args.tune:
        # one-time autotuning of every bucket the batch looks up (outside the timed region)
        from curplsh_b200 import autotune
        cb.tuning_clear()
        untuned = cb.SearchBatch(items, precision=precision)
        for _ in range(args.warmup):
            untuned.run(stream=stream, wait=False)
        stream.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            untuned.run(stream=stream, wait=False)
        e1.record(stream)
        e1.synchronize()
        untuned.close()
        t0 = time.perf_counter()
        recs = autotune.tune_batch(items, precision=precision, reps=2, stream=stream)
        tuned = {"buckets": len(recs), "tuning_s": time.perf_counter() - t0,
                 "untuned_ms_per_step": e0.elapsed_time(e1) / args.steps,
                 "changed": sum(1 for r in recs if (r["split_q4"], r["pool_headroom"]) != autotune.DEFAULT),
                 "picks": {r["bucket"]: [r["split_q4"], r["pool_headroom"], round(r["ms"], 3), round(r["default_ms"], 3)]
                           for r in recs}}
    batch = cb.SearchBatch(items, precision=precision)
    kernels, ws_bytes = batch.info()
    # correctness: every item equals its search alone; a query sample against the oracle
    batch.run(stream=stream)
    mismatches = 0
    recall_min, err_max = 1.0, 0.0
    recall_failures = []
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
            if rec < 1.0:
                recall_failures.append({"item": j, "nq": int(q.shape[0]), "k": k, "recall": rec, "max_rel_err": err,
                                        "got": oi[:1, :3].cpu().tolist(), "ref": ri[:1, :3].tolist()})

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

    sampler = ClockSampler(local)
    sampler.__enter__()
    ms_graph = timed(lambda: batch.run(stream=stream, wait=False))
    sampler.__exit__(None, None, None)

    def one_by_one():
        for ix, q, k, oi, od in items:
            ix.search_ex(q.shape[0], q, k, oi, od, precision, stream=stream)
    ms_loop = timed(one_by_one)
    # end to end: pinned host queries in, host results out, around the graph replay
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
    ms_e2e = timed(e2e_step)
    if rank == 0:
        hbm, bf16_burst, bf16_sust, peak_kind = load_peaks()
        p_form = bf16_burst / 3.0 if precision == 0 else (2 * bf16_burst if precision == 2 else bf16_burst)
        achieved = flops / (ms_graph / 1e3) / 1e12
        line = {
            "metric": METRIC, "value": total_q * world / (ms_graph / 1e3), "unit": "queries/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_graph, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": FORMS[precision].split("_")[0],
            "data": "synthetic (seeded N(0,1) rounded to BF16, stored FP32)",
            "config": {"workload": "batched_uneven", "databases": [{"N": n, "d": d} for n, d in dbs_spec],
                       "batches": len(batches), "queries_per_step": total_q,
                       "k_values": sorted({b[2] for b in batches}), "form": FORMS[precision],
                       "l2": "databases (3.1 GB) larger than L2"},
            "one_by_one": {"queries_per_s": total_q * world / (ms_loop / 1e3), "ms_per_step": ms_loop},
            "batch_speedup": ms_loop / ms_graph,
            "identical_to_alone": mismatches == 0, "items_differing": mismatches,
            "recall_at_k_min_sampled": recall_min, "max_rel_dist_err_sampled": err_max,
            "recall_failures": recall_failures,
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": p_form, "unit": "TFLOP/s",
                         "frac": achieved / p_form, "traffic": None, "kernel": "whole graph (prep + fused + merge)",
                         "peak_kind": peak_kind + " bf16 burst", "algorithmic": "sum 2*nq*N*d"},
            "cpu_baseline": None,
            "e2e": {"value": total_q * world / (ms_e2e / 1e3), "unit": "queries/s", "ms_per_step": ms_e2e,
                    "h2d_bytes_per_step": sum(it[1].numel() * 4 for it in items),
                    "d2h_bytes_per_step": sum(it[3].numel() * 8 for it in items)},
            "gpu_launches": kernels * args.steps, "launches_per_step": {"graph": 1, "kernels_in_graph": kernels},
            "workspace_bytes": ws_bytes, "autotune": tuned,
            "clocks": sampler.summary(),
        }
        print(json.dumps(line), flush=True)
    batch.close()
    for ix, _ in dbs:
        ix.close()
    res.close()
    barrier(world)
    return 0


def run_serving(args, world, rank, local):
    """--workload serving: one resident database (N = 5,000,000, d = 256,
    BF16-valued Gaussian mixture of 2,048 centroids), requests of 1-256
    queries (log-uniform) arriving as a Poisson process, k = 50, queries and
    results in pinned host memory.  For the BF16 + rerank form and the plain
    FP32-exact form: saturated throughput (every request queued at once) and,
    per offered rate, p50 / p99 latency (submit to results in host memory)
    and achieved throughput."""
    import numpy as np
    import torch

    import curplsh_b200 as cb
    import oracle
    from curplsh_b200 import synth

    torch.cuda.set_device(local)
    dev = f"cuda:{local}"
    n, d, k = args.serve_n, 256, 50
    base, qpool = synth.mixture_bf16(n, 20000, d, backend="torch", device=dev)
    torch.cuda.synchronize()
    res = cb.DeviceResources(local)
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
        """Submits request i at arrivals[i] seconds; returns (latencies, wall seconds, results)."""
        outs = make_outputs(sizes)
        offs = np.cumsum([0] + sizes[:-1]) % (qpool_h.shape[0] - 256)
        qs = [qpool_h[o:o + m] for o, m in zip(offs, sizes)]
        tickets = [None] * len(sizes)
        lat = [None] * len(sizes)
        done = threading.Event()

        def waiter():
            for i in range(len(sizes)):
                while tickets[i] is None:
                    time.sleep(20e-6)
                lat[i] = srv.wait(tickets[i], timeout=600.0)
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
        return np.array(lat), wall, (qs, outs)

    forms_out = {}
    recall = None
    for form in (1, 0):
        srv = cb.Server(ix, precision=form, max_inflight=3, max_step_queries=4096, memory_budget=4 << 30)
        # warm-up: a burst, then a few requests spaced out (first-call costs of the paced path)
        sizes = request_sizes(64)
        run_load(srv, sizes, [0.0] * len(sizes))
        sizes = request_sizes(16)
        run_load(srv, sizes, [i * 2e-3 for i in range(len(sizes))])
        # saturated throughput: every request queued at once
        sizes = request_sizes(600)
        lat, wall, (qs, outs) = run_load(srv, sizes, [0.0] * len(sizes))
        sat = sum(sizes) / wall
        if form == 1:
            # a sample of served results, checked against the FP64 oracle after all timing
            qsample = np.concatenate([qs[i][:1].numpy() for i in range(8)])
            gsample = np.concatenate([outs[i][0][:1].numpy() for i in range(8)])
        per_rate = {}
        for rate in args.serve_rates:
            mean_req = rate / 46.0  # mean of the log-uniform 1..256 request size is ~46 queries
            count = int(min(3000, max(200, mean_req * args.serve_seconds)))
            sizes = request_sizes(count)
            gaps = rng.exponential(1.0 / mean_req, size=count)
            arrivals = np.cumsum(gaps) - gaps[0]
            lat, wall, _ = run_load(srv, sizes, list(arrivals))
            slow = np.argsort(-lat)[:3]
            per_rate[str(rate)] = {"p50_ms": float(np.percentile(lat, 50) * 1e3),
                                   "p99_ms": float(np.percentile(lat, 99) * 1e3),
                                   "max_ms": float(lat.max() * 1e3),
                                   "slowest": [[int(i), sizes[i], float(lat[i] * 1e3)] for i in slow],
                                   "achieved_queries_per_s": sum(sizes) / wall, "requests": count}
        st = srv.stats()
        srv.close()
        forms_out[FORMS[form]] = {"saturated_queries_per_s": sat, "rates": per_rate,
                                  "steps": st["steps"], "max_inflight_seen": st["max_inflight_seen"],
                                  "peak_bytes_in_use": st["peak_bytes_in_use"],
                                  "kernel_launches": st["kernel_launches"]}
    if rank == 0 and not args.no_recall:
        base_h = base.cpu().numpy()
        rd, ri = oracle.knn(base_h, qsample, k)
        recall, _ = oracle.recall_at_k(base_h, qsample, gsample, rd)
    if rank == 0:
        b = forms_out["bf16_rerank"]
        line = {
            "metric": "serving p50/p99 latency (ms) and queries/s", "value": b["saturated_queries_per_s"],
            "unit": "queries/s", "n_gpus": world, "steps": None, "warmup": 1, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16",
            "data": "synthetic (seeded Gaussian mixture, 2048 centroids, BF16-valued)",
            "config": {"workload": "serving", "N": n, "d": d, "k": k, "request_queries": "log-uniform 1-256",
                       "arrivals": "Poisson", "io": "pinned host queries and results",
                       "max_inflight": 3, "memory_budget_bytes": 4 << 30},
            "recall_at_k_sampled": recall, "forms": forms_out,
            "bf16_vs_exact_saturated": b["saturated_queries_per_s"] / forms_out["fp32_exact"]["saturated_queries_per_s"],
        }
        print(json.dumps(line), flush=True)
    ix.close()
    res.close()
    barrier(world)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--forms", default=None, help="precision forms to time (0 exact, 1 bf16, 2 fp8)")
    ap.add_argument("--no-recall", action="store_true", help="skip the oracle recall check (profiling runs)")
    ap.add_argument("--workload", default=WORKLOAD, choices=list(WORKLOADS) + ["batched_uneven", "serving"])
    ap.add_argument("--serve-n", type=int, default=5_000_000, help="serving workload: database rows")
    ap.add_argument("--serve-rates", type=lambda v: [int(x) for x in v.split(",")], default=[1000, 5000, 20000, 50000],
                    help="serving workload: offered query rates (queries/s)")
    ap.add_argument("--serve-seconds", type=float, default=3.0, help="serving workload: seconds per rate")
    ap.add_argument("--batch-form", type=int, default=1, help="precision form of the batched workload")
    ap.add_argument("--tune", action="store_true", help="batched workload: autotune its buckets first")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world, rank, local = dist_init()
    if args.impl == "reference":
        rc = run_reference(args, world, rank)
        barrier(world)
        return rc
    if args.workload in ("batched_uneven", "serving"):
        rc = (run_batched if args.workload == "batched_uneven" else run_serving)(args, world, rank, local)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return rc

    import numpy as np
    import torch

    import curplsh_b200 as cb
    import oracle
    from curplsh_b200 import synth

    torch.cuda.set_device(local)
    dev = f"cuda:{local}"
    wl = args.workload
    info = WORKLOADS[wl]
    n_db, _, dim, _ = synth.CONFIGS[wl]
    # every rank holds the same database and searches a full query batch (replicas)
    base, queries, k = synth.make(wl, backend="torch", device=dev)
    torch.cuda.synchronize()  # generated on torch's stream; the library orders its work on its own streams
    res = cb.DeviceResources(local)
    stream = torch.cuda.Stream(device=dev)
    Q = queries.shape[0]
    oi = torch.empty((Q, k), dtype=torch.int32, device=dev)
    od = torch.empty((Q, k), dtype=torch.float32, device=dev)

    # ---- recall of every form on a query subsample (rank 0), and the CPU baseline
    sub = torch.arange(0, Q, Q // RECALL_SAMPLE, device=dev)[:RECALL_SAMPLE]
    form_results = {}
    cpu = None
    if rank == 0 and not args.no_recall:
        base_h = base.cpu().numpy()
        qs_h = queries[sub].cpu().numpy()
        rate, rd, ri, cores = cpu_oracle_rate(base_h, qs_h, k, RECALL_SAMPLE)
        cpu = {"value": rate, "unit": "queries/s", "cores": cores, "kind": "port",
               "sample": f"{RECALL_SAMPLE} queries against all {n_db} rows (FP64 oracle, OpenMP)"}
    forms = [int(f) for f in (args.forms or info["forms"]).split(",") if f != ""]
    headline = info["headline"] if info["headline"] in forms else forms[0]
    indexes = {}
    for form in forms:
        ix = cb.IndexBF(res, dim, cb.IndexBFConfig(device=local, precision=form))
        ix.add(n_db, base)
        indexes[form] = ix
        ix.search_ex(Q, queries, k, oi, od, stream=stream)
        stream.synchronize()
        if rank == 0 and not args.no_recall:
            gi = oi[sub].cpu().numpy()
            gd = od[sub].cpu().numpy().astype(np.float64)
            rec, _ = oracle.recall_at_k(base_h, qs_h, gi, rd[:, :k])
            err = float(np.max(np.abs(gd - rd[:, :k]) / np.maximum(np.abs(rd[:, :k]), 1e-30)))
            form_results[FORMS[form]] = {"recall_at_k": rec, "max_rel_dist_err": err}

    # ---- timed region: device-resident queries, CUDA events on our stream
    peaks = load_peaks()
    flops = 2.0 * Q * n_db * dim
    timing = {}
    estimates = {}
    clocks = None

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
        sampler = ClockSampler(local) if form == headline else None
        if sampler:
            sampler.__enter__()
        fb0 = ix.fallback_count()
        ms = timed_searches(ix, args.steps)
        fb = ix.fallback_count() - fb0
        if sampler:
            sampler.__exit__(None, None, None)
            clocks = sampler.summary()
        ms = max_over_ranks(ms, world)
        # per-pass device times (events between passes on the same stream)
        passes = ix.search_profiled(Q, queries, k, oi, od, stream=stream)
        fused_ms = max_over_ranks(passes["fused_ms"], world)
        timing[form] = (ms, fused_ms, passes)
        rows, step, rank_r = ix.estimate_plan(Q, k, form)
        est = {"sample_rows": rows, "step": step, "rank": rank_r, "fallback_queries_timed": fb}
        if rows:
            # the same searches without the sampled bound estimate, for comparison
            cb.set_bound_estimate(False)
            for _ in range(2):
                ix.search_ex(Q, queries, k, oi, od, stream=stream)
            est["ms_per_search_without"] = max_over_ranks(timed_searches(ix, max(1, args.steps // 2)), world)
            cb.set_bound_estimate(True)
        estimates[form] = est
    # query prep, [sample pass + estimate merge,] fused tensor-core filter, merge + rerank
    launches_per_step = 5 if estimates[headline]["sample_rows"] else 3

    # ---- end to end through the C ABI: pinned host queries in, host results out
    qh = torch.empty((Q, dim), dtype=torch.float32, pin_memory=True)
    qh.copy_(queries.cpu())
    ih = torch.empty((Q, k), dtype=torch.int32, pin_memory=True)
    dh = torch.empty((Q, k), dtype=torch.float32, pin_memory=True)
    ix = indexes[headline]
    for _ in range(args.warmup):
        ix.search(Q, qh, k, ih, dh)
    barrier(world)
    e2e_ms = []
    for _ in range(args.steps):
        t = ix.search_profiled(Q, qh, k, ih, dh, stream=stream)
        e2e_ms.append(t["total_ms"])
    e2e = max_over_ranks(sum(e2e_ms) / len(e2e_ms), world)

    if rank == 0:
        ms, fused_ms, passes = timing[headline]
        hbm, bf16_burst, bf16_sust, peak_kind = peaks
        forms_out = {}
        for form in forms:
            name = FORMS[form]
            f_ms, f_fused, _ = timing[form]
            p_form = bf16_burst / 3.0 if form == 0 else (2 * bf16_burst if form == 2 else bf16_burst)
            forms_out[name] = {
                "queries_per_s": Q * world / (f_ms / 1e3), "ms_per_search": f_ms, "fused_ms": f_fused,
                "fused_tflops": flops / (f_fused / 1e3) / 1e12,
                "roofline_frac": flops / (f_fused / 1e3) / 1e12 / p_form,
                "peak_basis_tflops": p_form, "bound_estimate": estimates[form], **form_results.get(name, {}),
            }
        achieved = flops / (fused_ms / 1e3) / 1e12
        rec = form_results.get(FORMS[headline], {}).get("recall_at_k")
        rec_ok = rec is not None and rec >= 1.0
        line = {
            "metric": METRIC, "value": Q * world / (ms / 1e3), "unit": "queries/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": FORMS[headline].split("_")[0],
            "data": info["data"],
            "config": {"workload": wl, "N": n_db, "Q": Q, "d": dim, "k": k, "form": FORMS[headline],
                       "rerank_factor": 4, "l2": info["l2"],
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "recall_at_k": rec, "recall_ok": rec_ok,
            "forms": forms_out,
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": bf16_burst, "unit": "TFLOP/s",
                         "frac": achieved / bf16_burst, "traffic": load_traffic(wl, FORMS[headline]),
                         "kernel": f"fused_knn_kernel<{FORMS[headline]}>", "peak_kind": peak_kind + " bf16 burst",
                         "algorithmic": "2*Q*N*d flops per launch"},
            "cpu_baseline": cpu,
            "e2e": {"value": Q * world / (e2e / 1e3), "unit": "queries/s", "ms_per_step": e2e,
                    "h2d_bytes_per_step": Q * dim * 4, "d2h_bytes_per_step": Q * k * 8},
            "gpu_launches": launches_per_step * args.steps,
            "launches_per_step": ({"prep_rows_kernel": 1, "fused_knn_kernel": 2, "merge_rerank_kernel": 2}
                                  if launches_per_step == 5 else
                                  {"prep_rows_kernel": 1, "fused_knn_kernel": 1, "merge_rerank_kernel": 1}),
            "clocks": clocks,
            "passes_ms": {k_: v for k_, v in passes.items()},
            "passes_note": "prep_ms includes the sample pass and estimate merge when bound_estimate.sample_rows > 0; "
                           "fused_ms is the full-database fused launch the roofline is taken on",
        }
        print(json.dumps(line), flush=True)
    for ix in indexes.values():
        ix.close()
    res.close()
    barrier(world)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
