"""Build recipe of ``libpds_b200.so`` (sm_100a), in-tree next to this file.

    python -m shapefromcaustics_b200.build [--force] [--verbose]

Compiles ``csrc/*.cu`` with nvcc for ``sm_100a`` only, links the CUDA runtime statically
(the library shares the process's primary context with torch) and writes the shared
library into the package directory, where ``shapefromcaustics_b200._lib`` loads it.
"""
import argparse
import glob
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libpds_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "-shared", "-cudart", "static",
]


def nvcc():
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    p = os.path.join(cuda, "bin", "nvcc")
    return p if os.path.exists(p) else "nvcc"


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale():
    if not os.path.isfile(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
    deps += glob.glob(os.path.join(INCLUDE, "*.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, ptxas_verbose=False):
    """Compile the library if any source is newer than it; returns its path."""
    if not force and not _stale():
        return LIB
    flags = list(NVCC_FLAGS)
    if ptxas_verbose:
        flags += ["-Xptxas", "-v"]
    cmd = [nvcc()] + flags + ["-I", INCLUDE, "-o", LIB + ".tmp"] + sources()
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose, a.ptxas_verbose))
