"""Builds libpdgpu.so for sm_100a with nvcc, in-tree (peridem_b200/_lib/).

The FP64 kernels are compiled with --fmad=false so that every product and
sum rounds separately, as in the reference's x86-64 build; the runtime and
the mixed-precision kernels keep FMA contraction.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIB_DIR, "libpdgpu.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler",
          "-fvisibility=hidden", "-I", os.path.join(ROOT, "include")]

UNITS = [
    ("pdgpu_kernels.cu", ["--fmad=false"]),
    ("pdgpu_bonds_fp64.cu", ["--fmad=false"]),
    ("pdgpu_bonds_mixed.cu", ["-ftz=true"]),
    ("pdgpu_mixed.cu", []),
    ("pdgpu_noalloc.cu", ["--fmad=false"]),
    ("pdgpu_tc.cu", []),
    ("pdgpu_surrogate.cu", []),
    ("pdgpu_runtime.cu", []),
    ("pdgpu_decks.cu", ["--fmad=false"]),
    ("pdgpu_meshsize.cu", ["--fmad=false"]),
    ("pdgpu_strain.cu", ["--fmad=false"]),
]


def _nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def sources():
    return [os.path.join(CSRC, u) for u, _ in UNITS] + [
        os.path.join(CSRC, "pdgpu_internal.h"), os.path.join(CSRC, "pdgpu_bonds.cuh"),
        os.path.join(ROOT, "include", "pdgpu.h")]


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(s) <= t for s in sources())


def build(force=False, verbose=False):
    """Compile every unit for sm_100a and link libpdgpu.so; returns its path."""
    if not force and up_to_date():
        return LIB
    os.makedirs(os.path.join(LIB_DIR, "obj"), exist_ok=True)
    objs = []
    for unit, extra in UNITS:
        obj = os.path.join(LIB_DIR, "obj", unit.replace(".cu", ".o"))
        cmd = [_nvcc(), *ARCH, *COMMON, *extra, "-c", os.path.join(CSRC, unit), "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [_nvcc(), *ARCH, "-shared", "-o", LIB, *objs]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
