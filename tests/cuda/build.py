"""Builds tests/cuda/libcurand_ref.so (test-only cuRAND harness) for sm_100a."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libcurand_ref.so")


def build(force=False):
    src = os.path.join(HERE, "curand_ref.cu")
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) > os.path.getmtime(src):
        return LIB
    nvcc = "/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else "nvcc"
    subprocess.run([nvcc, "-O2", "-shared", "-Xcompiler", "-fPIC", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-o", LIB, src], check=True)
    return LIB


if __name__ == "__main__":
    print(build(True))
