"""Build the matcha_b200 CUDA library in-tree for sm_100a.

    python -m matcha_b200.build [--verbose]

Produces ``matcha_b200/_lib/libmatcha_b200.so`` from ``matcha_b200/csrc/*.cu`` and ``*.cpp`` with
nvcc (cross-compiles without a GPU).  The library exports the C ABI declared in
``include/matcha_b200.h``.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB_DIR = os.path.join(PKG, "_lib")
LIB = os.path.join(LIB_DIR, "libmatcha_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; set NVCC or put CUDA's bin directory on PATH")


def sources():
    return sorted(glob.glob(os.path.join(PKG, "csrc", "*.cu")) + glob.glob(os.path.join(PKG, "csrc", "*.cpp")))


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(PKG, "csrc", "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, obj: str, verbose: bool):
    cmd = [nvcc_path(), "-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC", "-c",
           "-I", os.path.join(ROOT, "include"), "-o", obj, src]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    return src, res


def build(verbose: bool = False, force: bool = False) -> str:
    """Compile every source to an object in matcha_b200/_build (in parallel), then link."""
    if not force and not needs_build():
        return LIB
    from concurrent.futures import ThreadPoolExecutor

    os.makedirs(LIB_DIR, exist_ok=True)
    obj_dir = os.path.join(PKG, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    srcs = sources()
    objs = [os.path.join(obj_dir, os.path.basename(s) + ".o") for s in srcs]
    with ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda so: _compile(so[0], so[1], verbose), zip(srcs, objs)))
    for src, res in results:
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed on {os.path.basename(src)}:\n" + res.stdout + res.stderr)
        if verbose:
            print(os.path.basename(src), res.stdout + res.stderr)
    tmp = LIB + ".tmp"
    cmd = [nvcc_path(), *ARCH, "-shared", "-o", tmp, *objs, "-lcuda"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + res.stdout + res.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force=True))
