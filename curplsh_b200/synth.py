"""Seeded synthetic workloads with the shapes and value distributions of the
benchmark configurations (no dataset files are used; the reference only ships
loaders for SIFT/GIST files, include/dataset.h:14-45, which are not present).

Generated with torch on the requested device from a fixed seed, so a GPU run
and the CPU oracle see identical inputs (copy to host for the oracle).
"""
from __future__ import annotations

import torch

CONFIGS = {
    # name: (N, Q, d, k)
    "uniform_small": (10_000, 100, 128, 10),      # plain FP32, U[0,1)
    "mixture_int_1m": (1_000_000, 10_000, 128, 100),
    "sphere_10m": (10_000_000, 10_000, 96, 10),
}


def _gen(device, seed):
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    return g


def uniform(n: int, q: int, d: int, seed: int = 0, device="cuda"):
    """i.i.d. U[0,1) FP32 database and queries."""
    g = _gen(device, seed)
    base = torch.rand((n, d), generator=g, device=device)
    queries = torch.rand((q, d), generator=g, device=device)
    return base, queries


def mixture_int(n: int, q: int, d: int = 128, centroids: int = 1000, sigma: float = 12.0, seed: int = 1,
                device="cuda", chunk: int = 1 << 20):
    """Gaussian mixture: centroids uniform in [0,255]^d, per-point N(0, sigma^2),
    rounded to integers and clamped to [0,255], stored FP32.  Queries come from
    the same mixture."""
    g = _gen(device, seed)
    cent = torch.rand((centroids, d), generator=g, device=device) * 255.0

    def draw(m):
        out = torch.empty((m, d), device=device)
        for s in range(0, m, chunk):
            e = min(m, s + chunk)
            lab = torch.randint(0, centroids, (e - s,), generator=g, device=device)
            x = cent[lab] + sigma * torch.randn((e - s, d), generator=g, device=device)
            out[s:e] = x.round_().clamp_(0.0, 255.0)
        return out

    return draw(n), draw(q)


def sphere_mixture(n: int, q: int, d: int = 96, centroids: int = 4096, sigma: float = 0.05, seed: int = 2,
                   device="cuda", chunk: int = 1 << 20):
    """Gaussian mixture on the unit sphere: centroids are normalised Gaussians,
    points are normalise(c + N(0, sigma^2)).  Queries from the same mixture."""
    g = _gen(device, seed)
    cent = torch.randn((centroids, d), generator=g, device=device)
    cent = cent / cent.norm(dim=1, keepdim=True)

    def draw(m):
        out = torch.empty((m, d), device=device)
        for s in range(0, m, chunk):
            e = min(m, s + chunk)
            lab = torch.randint(0, centroids, (e - s,), generator=g, device=device)
            x = cent[lab] + sigma * torch.randn((e - s, d), generator=g, device=device)
            out[s:e] = x / x.norm(dim=1, keepdim=True)
        return out

    return draw(n), draw(q)


def batched_uneven_spec(seed: int = 3, num_dbs: int = 8, num_batches: int = 64, n_lo: int = 10_000,
                        n_hi: int = 2_000_000, q_lo: int = 1, q_hi: int = 4096, dims=(64, 128, 256, 512),
                        ks=(1, 10, 100, 1024)):
    """Shapes of the uneven batched workload: `num_dbs` resident databases with
    N log-uniform in [n_lo, n_hi] and d cycling through a shuffled `dims` (so
    every dimension occurs); `num_batches` query
    batches with sizes log-uniform in [q_lo, q_hi], each against a random
    database with k drawn from `ks`.  Returns (dbs [(n, d)], batches [(db, nq, k)])."""
    import numpy as np
    rng = np.random.default_rng(seed)
    dbs = []
    dim_order = [int(x) for x in rng.permutation(list(dims) * ((num_dbs + len(dims) - 1) // len(dims)))]
    for i in range(num_dbs):
        n = int(round(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi)))))
        dbs.append((n, dim_order[i]))
    batches = []
    for _ in range(num_batches):
        nq = int(round(np.exp(rng.uniform(np.log(q_lo), np.log(q_hi)))))
        db = int(rng.integers(num_dbs))
        k = int(rng.choice(ks))
        batches.append((db, nq, min(k, dbs[db][0])))
    return dbs, batches


def normal_bf16(rows: int, d: int, seed: int, device="cuda", chunk: int = 1 << 20):
    """i.i.d. N(0,1) values rounded to BF16, stored FP32."""
    g = _gen(device, seed)
    out = torch.empty((rows, d), device=device)
    for s in range(0, rows, chunk):
        e = min(rows, s + chunk)
        out[s:e] = torch.randn((e - s, d), generator=g, device=device).bfloat16().float()
    return out


def mixture_bf16(n: int, q: int, d: int = 256, centroids: int = 2048, sigma: float = 0.25, seed: int = 4,
                 device="cuda", chunk: int = 1 << 20):
    """Gaussian mixture with N(0,1) centroids and per-point N(0, sigma^2)
    offsets, values rounded to BF16 and stored FP32.  Queries come from the
    same mixture."""
    g = _gen(device, seed)
    cent = torch.randn((centroids, d), generator=g, device=device)

    def draw(m):
        out = torch.empty((m, d), device=device)
        for s in range(0, m, chunk):
            e = min(m, s + chunk)
            lab = torch.randint(0, centroids, (e - s,), generator=g, device=device)
            x = cent[lab] + sigma * torch.randn((e - s, d), generator=g, device=device)
            out[s:e] = x.bfloat16().float()
        return out

    return draw(n), draw(q)


def make(name: str, device="cuda", n: int | None = None, q: int | None = None):
    """Inputs of a named configuration (optionally with N or Q overridden)."""
    N, Q, d, k = CONFIGS[name]
    N = n or N
    Q = q or Q
    if name == "uniform_small":
        b, qq = uniform(N, Q, d, device=device)
    elif name == "mixture_int_1m":
        b, qq = mixture_int(N, Q, d, device=device)
    elif name == "sphere_10m":
        b, qq = sphere_mixture(N, Q, d, device=device)
    else:
        raise KeyError(name)
    return b, qq, k
