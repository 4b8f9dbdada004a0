"""The seeded input generator (curplsh_b200/synth.py): SplitMix64 words, the
derived uniforms and labels, and agreement of its host (numpy) and device
(torch) backends."""
import importlib.util
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _synth():
    spec = importlib.util.spec_from_file_location("curplsh_synth", os.path.join(ROOT, "curplsh_b200", "synth.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _splitmix64_scalar(state, count):
    """The published SplitMix64 generator, one output at a time."""
    out = []
    for _ in range(count):
        state = (state + 0x9E3779B97F4A7C15) & ((1 << 64) - 1)
        z = state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & ((1 << 64) - 1)
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & ((1 << 64) - 1)
        out.append(z ^ (z >> 31))
    return out


def test_words_are_splitmix64():
    s = _synth()
    B = s._Numpy()
    assert int(B.words(0, 0, 1)[0]) == 0xE220A8397B1DCDAF  # first output of SplitMix64 seeded with 0
    for key in (0, 1234567, (1 << 64) - 5):
        assert [int(x) for x in B.words(key, 0, 6)] == _splitmix64_scalar(key, 6)
        assert [int(x) for x in B.words(key, 3, 3)] == _splitmix64_scalar(key, 6)[3:]


def test_rows_are_independent_of_the_draw_size():
    s = _synth()
    b1, q1, _ = s.make("uniform_small")
    b2, q2 = s.uniform(300, 7, 128, seed=s.SEEDS["uniform_small"])
    assert np.array_equal(b1[:300], b2) and np.array_equal(q1[:7], q2)
    m1 = s.mixture_int(5000, 40)
    m2 = s.mixture_int(2000, 10)
    assert np.array_equal(m1[0][:2000], m2[0]) and np.array_equal(m1[1][:10], m2[1])


def test_distributions():
    s = _synth()
    B = s._Numpy()
    z = s.normals(B, s.stream_key(9, 0), 0, 400_000)
    assert abs(z.mean()) < 0.01 and abs(z.std() - 1) < 0.01 and abs((z ** 4).mean() - 3) < 0.05
    u = s.uniform_f32(B, s.stream_key(9, 1), 0, 100_000)
    assert u.dtype == np.float32 and u.min() >= 0 and u.max() < 1 and abs(u.mean() - 0.5) < 0.01
    lab = s.labels(B, s.stream_key(9, 2), 0, 100_000, 1000)
    assert lab.min() == 0 and lab.max() == 999
    b, q = s.mixture_int(3000, 10)
    assert b.dtype == np.float32 and np.array_equal(b, np.rint(b)) and b.min() >= 0 and b.max() <= 255
    b, q = s.sphere_mixture(3000, 10)
    assert np.allclose(np.linalg.norm(b, axis=1), 1, atol=1e-6)
    x = s.normal_bf16(100, 64, 3)
    assert np.array_equal(x.view(np.uint32) & 0xFFFF, np.zeros_like(x.view(np.uint32)))


def _compare_backends(device):
    s = _synth()
    N, T = s._Numpy(), s._Torch(device)
    key = s.stream_key(7, 2)
    assert np.array_equal(N.words(key, 1000, 50_000).view(np.int64), T.words(key, 1000, 50_000).cpu().numpy())
    assert np.array_equal(s.uniform_f32(N, key, 3, 50_000), s.uniform_f32(T, key, 3, 50_000).cpu().numpy())
    assert np.array_equal(s.uniform_f64(N, key, 3, 50_000), s.uniform_f64(T, key, 3, 50_000).cpu().numpy())
    assert np.array_equal(s.labels(N, key, 3, 50_000, 4096), s.labels(T, key, 3, 50_000, 4096).cpu().numpy())
    a = s.normals(N, key, 5, 50_001)
    b = s.normals(T, key, 5, 50_001).cpu().numpy()
    assert np.max(np.abs(a - b)) < 1e-14  # FP64 transcendental rounding may differ in the last bit
    for name in ("uniform_small",):
        x = s.make(name)
        y = s.make(name, backend="torch", device=device)
        assert np.array_equal(x[0], y[0].cpu().numpy()) and np.array_equal(x[1], y[1].cpu().numpy())
    x = s.mixture_int(20000, 50)
    y = s.mixture_int(20000, 50, backend="torch", device=device)
    assert np.array_equal(x[0], y[0].cpu().numpy()) and np.array_equal(x[1], y[1].cpu().numpy())
    x = s.sphere_mixture(20000, 50)
    y = s.sphere_mixture(20000, 50, backend="torch", device=device)
    assert (x[0] != y[0].cpu().numpy()).mean() < 1e-5


def test_numpy_and_torch_cpu_backends_agree():
    _compare_backends("cpu")


@pytest.mark.gpu
def test_numpy_and_torch_cuda_backends_agree():
    _compare_backends("cuda")
