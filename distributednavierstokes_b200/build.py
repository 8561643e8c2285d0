"""Build libdnsb.so in-tree with nvcc for sm_100a.

    python -m distributednavierstokes_b200.build

nvcc cross-compiles without a GPU; the resulting .so sits next to this file
so that it travels with the source tree.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libdnsb.so")
SOURCES = ["dnsb.cu"]
HEADERS = ["common.cuh", "fft.cuh", "fft4.cuh", "spectral.cuh", "spectral4.cuh", "stencil.cuh",
           "tma.cuh", "ysolve.cuh", "gradmom.cuh", "zyz.cuh", "spsolver.cuh", "lowshells.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
]


def _nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _host_compiler():
    # the system g++ (some images point CXX at a compiler without its runtime)
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and os.path.exists(cand):
            return cand
    return None


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "dnsb.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    if not force and not needs_build():
        return OUT
    cmd = [_nvcc()] + NVCC_FLAGS
    hc = _host_compiler()
    if hc:
        cmd += ["-ccbin", hc]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    cmd += ["-o", OUT + ".tmp"] + [os.path.join(CSRC, s) for s in SOURCES]
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
