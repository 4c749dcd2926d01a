"""Builds the in-tree CUDA library onemirror_b200/lib/libqmcrt.so for sm_100a.

Each translation unit is compiled by nvcc in parallel into
onemirror_b200/_build/, then linked into one shared library exporting the
C-ABI declared in include/qmcrt.h.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib", "libqmcrt.so")

SOURCES = ["host.cpp", "scene.cu", "trace.cu", "batch.cu", "adjoint.cu", "smooth.cu", "probe.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include")]
CUDA_ONLY = ["-lineinfo", "--expt-relaxed-constexpr"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _compile(src, verbose_ptxas=False):
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    path = os.path.join(CSRC, src)
    cmd = [nvcc(), "-c", path, "-o", obj] + ARCH + COMMON
    if src.endswith(".cu"):
        cmd += CUDA_ONLY
        if verbose_ptxas:
            cmd += ["-Xptxas", "-v"]
    else:
        cmd += ["-x", "cu"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), r.stderr))
    return obj, r.stderr


def _stale(objs):
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "qmcrt.h"), __file__]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose_ptxas=False):
    """Compile and link libqmcrt.so; returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    if not force and not _stale(None):
        return LIB
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose_ptxas), SOURCES))
    if verbose_ptxas:
        for _, err in results:
            sys.stderr.write(err)
    objs = [o for o, _ in results]
    cmd = [nvcc(), "-shared", "-o", LIB] + ARCH + objs + ["-Xcompiler", "-fPIC"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv))
