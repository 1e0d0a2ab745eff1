"""Build libowl.so (the sm_100a engine behind include/owl.h and the host drivers of
include/owl_host.h) in-tree.

    python -m gpuowl_b200.build            # or: python gpuowl_b200/build.py

Compiles gpuowl_b200/csrc/*.cu with nvcc for sm_100a only, gpuowl_b200/host/*.cpp
with the host compiler nvcc drives, and links gpuowl_b200/libowl.so. The build is skipped when the library is newer than
every source file.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
HOST = os.path.join(HERE, "host")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libowl.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
              "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def sources():
    out = []
    for d in (CSRC, HOST):
        for name in sorted(os.listdir(d)):
            if name.endswith((".cu", ".cuh", ".inc", ".hpp", ".h", ".cpp")):
                out.append(os.path.join(d, name))
    for name in sorted(os.listdir(INCLUDE)):
        out.append(os.path.join(INCLUDE, name))
    return out


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(s) <= t for s in sources())


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    cu = [os.path.join(CSRC, n) for n in sorted(os.listdir(CSRC)) if n.endswith(".cu")]
    cu += [os.path.join(HOST, n) for n in sorted(os.listdir(HOST)) if n.endswith(".cpp")]
    cmd = [nvcc()] + ARCH + NVCC_FLAGS + ["-shared", "-I", INCLUDE, "-I", CSRC, "-o", LIB + ".tmp"] + cu
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libowl.so")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
