"""Build libdnsb.so in-tree with nvcc for sm_100a.

    python -m distributednavierstokes_b200.build [--force] [-v]

Each .cu translation unit is compiled to an object under _build/ (rebuilt
only when it or a header changed), then the objects are linked into the
shared library next to this file, so that it travels with the source tree.
nvcc cross-compiles without a GPU.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build")
OUT = os.path.join(HERE, "libdnsb.so")
SOURCES = ["dnsb.cu", "cnn.cu"]
INCLUDES = [os.path.join(ROOT, "include", h) for h in ("dnsb.h", "dnsb_cnn.h")]
# headers each translation unit includes (a change rebuilds its object)
HEADERS = {
    "dnsb.cu": ["common.cuh", "fft.cuh", "fft4.cuh", "spectral.cuh", "spectral4.cuh", "stencil.cuh",
                "tma.cuh", "ysolve.cuh", "gradmom.cuh", "zyz.cuh", "spsolver.cuh", "lowshells.cuh",
                "cnn_host.h"],
    "cnn.cu": ["cnn.cuh", "cnn_host.h"],
}

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]


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


def _obj(src):
    return os.path.join(BUILD, os.path.splitext(src)[0] + ".o")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _deps(src):
    return [os.path.join(CSRC, src)] + [os.path.join(CSRC, h) for h in HEADERS.get(src, [])] + INCLUDES


def needs_build():
    objs = [_obj(s) for s in SOURCES]
    return any(_stale(_obj(s), _deps(s)) for s in SOURCES) or _stale(OUT, objs)


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    hc = _host_compiler()
    base = [_nvcc()] + NVCC_FLAGS + (["-ccbin", hc] if hc else [])
    changed = False
    for s in SOURCES:
        o = _obj(s)
        if force or _stale(o, _deps(s)):
            cmd = base + (["-Xptxas", "-v"] if verbose else []) + ["-c", "-o", o + ".tmp", os.path.join(CSRC, s)]
            subprocess.run(cmd, check=True)
            os.replace(o + ".tmp", o)
            changed = True
    objs = [_obj(s) for s in SOURCES]
    if force or changed or _stale(OUT, objs):
        cmd = [_nvcc()] + ARCH + ["-shared"] + (["-ccbin", hc] if hc else []) + ["-o", OUT + ".tmp"] + objs
        subprocess.run(cmd, check=True)
        os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
