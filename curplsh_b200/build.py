"""Build libcurplsh_b200.so in-tree with nvcc for sm_100a (B200).

    python curplsh_b200/build.py            # incremental
    python curplsh_b200/build.py --force    # rebuild everything

Run it as a script (or load it by path, as __graft_entry__.build() does):
importing the package itself loads the library, which may not exist yet.

Objects go to curplsh_b200/_build/ (git-ignored); the shared library lands at
curplsh_b200/libcurplsh_b200.so so that it travels with the source tree.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcurplsh_b200.so")
EXTRA_DEFINES: list[str] = []  # e.g. ["-DCURPLSH_FUSED_STATS"] for an instrumented build

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
          "-I", CSRC, "-I", os.path.join(ROOT, "include")]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return path


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def headers():
    out = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    out.append(os.path.join(ROOT, "include", "curplsh_b200.h"))
    return out


def _compile(src: str, force: bool, verbose_ptxas: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    common = COMMON + EXTRA_DEFINES
    newest_dep = max(os.path.getmtime(p) for p in headers() + [src])
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep:
        return obj
    cmd = [nvcc(), *ARCH, *common, "-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [nvcc(), *common, "-x", "cu", *ARCH, "-c", src, "-o", obj]
    if verbose_ptxas and src.endswith(".cu"):
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {os.path.basename(src)}:\n{res.stdout}\n{res.stderr}")
    if verbose_ptxas and res.stderr:
        sys.stderr.write(res.stderr)
    return obj


def build(force: bool = False, verbose_ptxas: bool = False, build_dir: str | None = None,
          lib: str | None = None) -> str:
    """Compile every source under csrc/ and link the shared library.  build_dir
    and lib redirect the outputs (used for instrumented side builds)."""
    global BUILD, LIB
    if build_dir:
        BUILD = build_dir
    if lib:
        LIB = lib
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, verbose_ptxas), srcs))
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        tmp = LIB + ".tmp"
        cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcuda"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
        os.replace(tmp, LIB)
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print ptxas register/smem usage")
    a = ap.parse_args()
    print(build(a.force, a.ptxas))


if __name__ == "__main__":
    main()
