"""Build libddfmm_b200.so in-tree with nvcc for sm_100a.

All CUDA/C++ sources under csrc/ are compiled into one shared library with
the CUDA runtime linked statically, so the library loads (and exports its C
ABI) on machines without a GPU; CUDA calls then fail with DDFMM_ECUDA.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libddfmm_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# extra -D options for measuring build-time kernel variants against each other
# (e.g. DDFMM_NVCC_DEFINES="-DDDFMM_ZGEMM_BK=32 -DDDFMM_ZGEMM_MINB=1"; build(force=True))
DEFINES = os.environ.get("DDFMM_NVCC_DEFINES", "").split()


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def headers():
    inc = os.path.join(os.path.dirname(HERE), "include")
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh"))] + \
        [os.path.join(inc, f) for f in os.listdir(inc)]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(s) <= t for s in sources() + headers())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [NVCC, "-std=c++17", "-O3", "-lineinfo", *ARCH, *DEFINES, "-Xcompiler", "-fPIC", "-Xptxas", "-v" if verbose else "-O3",
               "-I", CSRC, "-x", "cu" if src.endswith(".cu") else "c++", "-c", src, "-o", obj]
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        objs.append(obj)
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError("nvcc failed on %s:\n%s" % (src, out))
        if verbose and out:
            print(out)
    tmp = LIB + ".tmp%d" % os.getpid()
    cmd = [NVCC, "-shared", *ARCH, "-cudart", "static", "-o", tmp, *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s%s" % (r.stdout, r.stderr))
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
