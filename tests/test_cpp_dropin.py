"""The C++ drop-in headers (include/curplsh/*.h): they compile against the C
ABI here, and on a GPU the reference's smoke pattern runs through them."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = "/usr/local/cuda"


def _compile(out, src="test_index_bf.cpp"):
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("g++ not available")
    cmd = [cxx, "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), "-I", f"{CUDA}/include",
           os.path.join(ROOT, "tests", "cpp", src), "-L", os.path.join(ROOT, "curplsh_b200"),
           "-lcurplsh_b200", "-L", f"{CUDA}/lib64", "-lcudart", f"-Wl,-rpath,{os.path.join(ROOT, 'curplsh_b200')}",
           "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_cpp_headers_compile(tmp_path):
    _compile(str(tmp_path / "t"))


@pytest.mark.gpu
def test_cpp_dropin_runs_reference_pattern(tmp_path):
    exe = str(tmp_path / "t")
    _compile(exe)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "cpp drop-in ok" in r.stdout


def test_cpp_dataset_header_compiles(tmp_path):
    _compile(str(tmp_path / "td"), "test_dataset.cpp")


@pytest.mark.gpu
def test_cpp_dataset_search_recall(tmp_path):
    """include/curplsh/dataset.h: write a SIFT-style directory, load it with
    DatasetSIFT, search it with IndexBF and evaluate recall (1.0)."""
    exe = str(tmp_path / "td")
    _compile(exe, "test_dataset.cpp")
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "cpp dataset ok" in r.stdout


def test_cpp_device_memory_header_compiles(tmp_path):
    _compile(str(tmp_path / "tm"), "test_device_memory.cpp")


@pytest.mark.gpu
def test_cpp_device_memory_reservations(tmp_path):
    """include/curplsh/device_memory.h: stream-ordered reservations, moves, reuse."""
    exe = str(tmp_path / "tm")
    _compile(exe, "test_device_memory.cpp")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "cpp device memory ok" in r.stdout


def test_server_admission_and_step_forming(tmp_path):
    """The serving loop's scheduling rules (curplsh_b200/csrc/server_sched.h):
    first-fit arena with coalescing, first-come-first-served steps under the
    query cap, and halving a step until its memory fits -- on the host."""
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("g++ not available")
    exe = str(tmp_path / "ts")
    r = subprocess.run([cxx, "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "curplsh_b200", "csrc"),
                        os.path.join(ROOT, "tests", "cpp", "test_server_sched.cpp"), "-o", exe],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "server sched ok" in r.stdout, r.stdout + r.stderr
