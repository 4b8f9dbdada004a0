"""Seeded synthetic workloads with the shapes and value distributions of the
benchmark configurations (no dataset files are used; the reference only ships
loaders for SIFT/GIST files, include/dataset.h:14-45, which are not present).

Every value comes from a counter-based SplitMix64 stream: output i of stream
(seed, s) is mix(key(seed, s) + (i + 1) * 0x9E3779B97F4A7C15), with the
SplitMix64 finaliser mix (shifts 30/27/31, multipliers 0xBF58476D1CE4E5B9 and
0x94D049BB133111EB).  From those 64-bit words:

* uniform FP32 in [0, 1): the top 24 bits times 2^-24 (exact);
* uniform FP64 in [0, 1): the top 53 bits times 2^-53;
* labels in [0, m): the top 32 bits times m, shifted right by 32;
* normals: Box-Muller on consecutive word pairs (2p, 2p + 1) in FP64,
  r = sqrt(-2 ln(1 - u1)), normal 2p = r cos(2 pi u2), normal 2p + 1 = r sin(2 pi u2).

Because element (row, column) of a matrix is output row * d + column of its
stream, any row range can be generated on its own (the first q queries of a
workload are the same whatever Q is), and the numpy backend (host) and the
torch backend (CUDA, int64 arithmetic that wraps modulo 2^64) produce the
same words and the same uniforms bit for bit.  Normals go through FP64
log/sqrt/cos/sin, whose last-bit rounding may differ between libraries; after
the cast to FP32 (or rounding to integers) such a difference survives in
about one value in 10^8 and moves it by one FP32 ulp.

This module imports nothing from the curplsh_b200 package, so it can be
loaded by file path without loading the library.
"""
from __future__ import annotations

import math

import numpy as np

CONFIGS = {
    # name: (N, Q, d, k)
    "uniform_small": (10_000, 100, 128, 10),      # plain FP32, U[0,1)
    "mixture_int_1m": (1_000_000, 10_000, 128, 100),
    "sphere_10m": (10_000_000, 10_000, 96, 10),
}

# seeds of the named workloads (recorded in the bench output)
SEEDS = {"uniform_small": 0, "mixture_int_1m": 1, "sphere_10m": 2, "serving": 4, "batched_uneven": 3}

_GAMMA = 0x9E3779B97F4A7C15
_M1 = 0xBF58476D1CE4E5B9
_M2 = 0x94D049BB133111EB
_MASK = (1 << 64) - 1

# streams of a workload
_S_CENT, _S_BASE_LAB, _S_BASE_VAL, _S_Q_LAB, _S_Q_VAL = 0, 1, 2, 3, 4


def _mix_int(z: int) -> int:
    z &= _MASK
    z = ((z ^ (z >> 30)) * _M1) & _MASK
    z = ((z ^ (z >> 27)) * _M2) & _MASK
    return z ^ (z >> 31)


def stream_key(seed: int, stream: int) -> int:
    """64-bit key of stream `stream` of seed `seed`."""
    return _mix_int(_mix_int(seed * _GAMMA + 0x5851F42D4C957F2D) ^ (stream * 0xD1B54A32D192ED03))


def _signed(c: int) -> int:
    return c - (1 << 64) if c >= (1 << 63) else c


class _Numpy:
    """uint64 numpy arithmetic (wraps modulo 2^64)."""

    name = "numpy"

    def words(self, key: int, start: int, count: int):
        i = np.arange(start + 1, start + 1 + count, dtype=np.uint64)
        with np.errstate(over="ignore"):
            z = np.uint64(key) + i * np.uint64(_GAMMA)
            z = (z ^ (z >> np.uint64(30))) * np.uint64(_M1)
            z = (z ^ (z >> np.uint64(27))) * np.uint64(_M2)
        return z ^ (z >> np.uint64(31))

    def top(self, z, bits: int):
        return z >> np.uint64(64 - bits)

    def f64(self, x):
        return x.astype(np.float64)

    def f32(self, x):
        return x.astype(np.float32)

    def i64(self, x):
        return x.astype(np.int64)

    def log(self, x):
        return np.log(x)

    def sqrt(self, x):
        return np.sqrt(x)

    def cos(self, x):
        return np.cos(x)

    def sin(self, x):
        return np.sin(x)

    def empty(self, shape, dtype):
        return np.empty(shape, dtype=dtype)

    def rint(self, x):
        return np.rint(x)

    def clip(self, x, lo, hi):
        return np.clip(x, lo, hi)

    def rownorm(self, x):
        return np.sqrt((x * x).sum(axis=1, keepdims=True))

    def bf16_round(self, x32):
        """Round FP32 values to the nearest BF16 (ties to even), kept as FP32."""
        b = x32.view(np.uint32)
        r = ((b >> np.uint32(16)) & np.uint32(1)) + np.uint32(0x7FFF)
        with np.errstate(over="ignore"):
            out = (b + r) & np.uint32(0xFFFF0000)
        return out.view(np.float32)

    def interleave(self, even, odd):
        out = np.empty(even.shape[0] * 2, dtype=np.float64)
        out[0::2] = even
        out[1::2] = odd
        return out


class _Torch:
    """int64 torch arithmetic on a CUDA device (multiplication wraps modulo 2^64;
    right shifts are made logical by masking)."""

    name = "torch"

    def __init__(self, device):
        import torch
        self.t = torch
        self.device = device

    def _srl(self, x, s: int):
        return (x >> s) & ((1 << (64 - s)) - 1)

    def words(self, key: int, start: int, count: int):
        t = self.t
        i = t.arange(start + 1, start + 1 + count, dtype=t.int64, device=self.device)
        z = i * _signed(_GAMMA) + _signed(key)
        z = (z ^ self._srl(z, 30)) * _signed(_M1)
        z = (z ^ self._srl(z, 27)) * _signed(_M2)
        return z ^ self._srl(z, 31)

    def top(self, z, bits: int):
        return self._srl(z, 64 - bits)

    def f64(self, x):
        return x.double()

    def f32(self, x):
        return x.float()

    def i64(self, x):
        return x.long()

    def log(self, x):
        return self.t.log(x)

    def sqrt(self, x):
        return self.t.sqrt(x)

    def cos(self, x):
        return self.t.cos(x)

    def sin(self, x):
        return self.t.sin(x)

    def empty(self, shape, dtype):
        t = self.t
        return t.empty(shape, dtype={np.float32: t.float32, np.float64: t.float64}[dtype], device=self.device)

    def rint(self, x):
        return self.t.round(x)  # round half to even, as np.rint

    def clip(self, x, lo, hi):
        return self.t.clamp(x, lo, hi)

    def rownorm(self, x):
        return self.t.sqrt((x * x).sum(dim=1, keepdim=True))

    def bf16_round(self, x32):
        return x32.bfloat16().float()

    def interleave(self, even, odd):
        return self.t.stack((even, odd), dim=1).reshape(-1)


def _backend(backend: str, device=None):
    if backend == "numpy":
        return _Numpy()
    if backend == "torch":
        return _Torch(device if device is not None else "cuda")
    raise ValueError(f"unknown backend {backend!r}")


def uniform_f32(B, key: int, start: int, count: int):
    """`count` uniform FP32 values in [0, 1) from outputs start.. of the stream."""
    return B.f32(B.top(B.words(key, start, count), 24)) * np.float32(2.0 ** -24)


def uniform_f64(B, key: int, start: int, count: int):
    return B.f64(B.top(B.words(key, start, count), 53)) * (2.0 ** -53)


def labels(B, key: int, start: int, count: int, m: int):
    """`count` labels in [0, m) (m < 2^31)."""
    return B.i64((B.top(B.words(key, start, count), 32) * m) >> 32)


def normals(B, key: int, start: int, count: int):
    """FP64 standard normals start .. start + count - 1 of the stream (Box-Muller
    over word pairs)."""
    p0 = start // 2
    p1 = (start + count + 1) // 2
    w = uniform_f64(B, key, 2 * p0, 2 * (p1 - p0))
    u1, u2 = w[0::2], w[1::2]
    r = B.sqrt(-2.0 * B.log(1.0 - u1))
    th = (2.0 * math.pi) * u2
    z = B.interleave(r * B.cos(th), r * B.sin(th))
    off = start - 2 * p0
    return z[off:off + count]


def _rows(B, n: int, d: int, chunk: int, fill):
    """An [n x d] FP32 matrix filled chunk by chunk by fill(r0, r1) -> [(r1-r0) x d].
    On the host, chunks of about a million values run on a thread pool (numpy
    releases the GIL in its loops); on a GPU they run one after another."""
    out = B.empty((n, d), np.float32)
    if B.name == "numpy":
        import concurrent.futures as cf
        import os
        rows = max(1, min(chunk, (1 << 20) // max(d, 1)))

        def work(r0):
            out[r0:min(n, r0 + rows)] = fill(r0, min(n, r0 + rows))

        with cf.ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 1)) as ex:
            list(ex.map(work, range(0, n, rows)))
        return out
    for r0 in range(0, n, chunk):
        r1 = min(n, r0 + chunk)
        out[r0:r1] = fill(r0, r1)
    return out


def uniform(n: int, q: int, d: int, seed: int = 0, backend: str = "numpy", device=None, chunk: int = 1 << 19):
    """i.i.d. U[0,1) FP32 database and queries."""
    B = _backend(backend, device)
    kb, kq = stream_key(seed, _S_BASE_VAL), stream_key(seed, _S_Q_VAL)
    base = _rows(B, n, d, chunk, lambda a, b: uniform_f32(B, kb, a * d, (b - a) * d).reshape(b - a, d))
    queries = _rows(B, q, d, chunk, lambda a, b: uniform_f32(B, kq, a * d, (b - a) * d).reshape(b - a, d))
    return base, queries


def _mixture(B, n, q, d, cent, sigma, seed, post, chunk):
    m = cent.shape[0]

    def draw(rows, s_lab, s_val):
        kl, kv = stream_key(seed, s_lab), stream_key(seed, s_val)

        def fill(a, b):
            lab = labels(B, kl, a, b - a, m)
            x = cent[lab] + sigma * normals(B, kv, a * d, (b - a) * d).reshape(b - a, d)
            return post(x)

        return _rows(B, rows, d, chunk, fill)

    return draw(n, _S_BASE_LAB, _S_BASE_VAL), draw(q, _S_Q_LAB, _S_Q_VAL)


def mixture_int(n: int, q: int, d: int = 128, centroids: int = 1000, sigma: float = 12.0, seed: int = 1,
                backend: str = "numpy", device=None, chunk: int = 1 << 19):
    """Gaussian mixture: centroids uniform in [0,255]^d, per-point N(0, sigma^2),
    rounded to integers (half to even) and clamped to [0,255], stored FP32.
    Queries come from the same mixture."""
    B = _backend(backend, device)
    cent = uniform_f64(B, stream_key(seed, _S_CENT), 0, centroids * d).reshape(centroids, d) * 255.0
    return _mixture(B, n, q, d, cent, sigma, seed, lambda x: B.f32(B.clip(B.rint(x), 0.0, 255.0)), chunk)


def sphere_mixture(n: int, q: int, d: int = 96, centroids: int = 4096, sigma: float = 0.05, seed: int = 2,
                   backend: str = "numpy", device=None, chunk: int = 1 << 19):
    """Gaussian mixture on the unit sphere: centroids are normalised Gaussians,
    points are normalise(c + N(0, sigma^2)) (FP64, stored FP32).  Queries from
    the same mixture."""
    B = _backend(backend, device)
    cent = normals(B, stream_key(seed, _S_CENT), 0, centroids * d).reshape(centroids, d)
    cent = cent / B.rownorm(cent)
    return _mixture(B, n, q, d, cent, sigma, seed, lambda x: B.f32(x / B.rownorm(x)), chunk)


def normal_bf16(rows: int, d: int, seed: int, backend: str = "numpy", device=None, chunk: int = 1 << 19):
    """i.i.d. N(0,1) values rounded to BF16, stored FP32."""
    B = _backend(backend, device)
    kv = stream_key(seed, _S_BASE_VAL)
    return _rows(B, rows, d, chunk,
                 lambda a, b: B.bf16_round(B.f32(normals(B, kv, a * d, (b - a) * d)).reshape(b - a, d)))


def mixture_bf16(n: int, q: int, d: int = 256, centroids: int = 2048, sigma: float = 0.25, seed: int = 4,
                 backend: str = "numpy", device=None, chunk: int = 1 << 19):
    """Gaussian mixture with N(0,1) centroids and per-point N(0, sigma^2)
    offsets, values rounded to BF16 and stored FP32.  Queries come from the
    same mixture."""
    B = _backend(backend, device)
    cent = normals(B, stream_key(seed, _S_CENT), 0, centroids * d).reshape(centroids, d)
    return _mixture(B, n, q, d, cent, sigma, seed, lambda x: B.bf16_round(B.f32(x)), chunk)


def batched_uneven_spec(seed: int = 3, num_dbs: int = 8, num_batches: int = 64, n_lo: int = 10_000,
                        n_hi: int = 2_000_000, q_lo: int = 1, q_hi: int = 4096, dims=(64, 128, 256, 512),
                        ks=(1, 10, 100, 1024)):
    """Shapes of the uneven batched workload: `num_dbs` resident databases with
    N log-uniform in [n_lo, n_hi] and d cycling through a shuffled `dims` (so
    every dimension occurs); `num_batches` query batches with sizes log-uniform
    in [q_lo, q_hi], each against a random database with k drawn from `ks`.
    Returns (dbs [(n, d)], batches [(db, nq, k)])."""
    B = _Numpy()
    u = uniform_f64(B, stream_key(seed, 0), 0, 4 * num_dbs + 4 * num_batches)
    pos = 0

    def nxt():
        nonlocal pos
        pos += 1
        return float(u[pos - 1])

    reps = (num_dbs + len(dims) - 1) // len(dims)
    pool = list(dims) * reps
    dim_order = []
    for _ in range(num_dbs):  # draw without replacement from the repeated dims
        dim_order.append(pool.pop(min(int(nxt() * len(pool)), len(pool) - 1)))
    dbs = []
    for i in range(num_dbs):
        n = int(round(math.exp(math.log(n_lo) + nxt() * (math.log(n_hi) - math.log(n_lo)))))
        dbs.append((n, dim_order[i]))
    batches = []
    for _ in range(num_batches):
        nq = int(round(math.exp(math.log(q_lo) + nxt() * (math.log(q_hi) - math.log(q_lo)))))
        db = min(int(nxt() * num_dbs), num_dbs - 1)
        k = ks[min(int(nxt() * len(ks)), len(ks) - 1)]
        batches.append((db, nq, min(k, dbs[db][0])))
    return dbs, batches


def make(name: str, backend: str = "numpy", device=None, n: int | None = None, q: int | None = None):
    """Inputs of a named configuration (optionally with N or Q overridden; the
    first rows of a smaller draw equal the first rows of the full one)."""
    N, Q, d, k = CONFIGS[name]
    N = n or N
    Q = q or Q
    seed = SEEDS[name]
    if name == "uniform_small":
        b, qq = uniform(N, Q, d, seed=seed, backend=backend, device=device)
    elif name == "mixture_int_1m":
        b, qq = mixture_int(N, Q, d, seed=seed, backend=backend, device=device)
    elif name == "sphere_10m":
        b, qq = sphere_mixture(N, Q, d, seed=seed, backend=backend, device=device)
    else:
        raise KeyError(name)
    return b, qq, k
