"""Build librtb200.so in-tree with nvcc for sm_100a.

Traversal (rt_trace.cu) is compiled with --fmad=false so the hit arithmetic
is the un-fused f32 sequence of the reference; the rest keeps FMA contraction.
Host code is compiled with -ffp-contract=off for the same reason (BVH build,
spectral tables).
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INC = os.path.join(HERE, "..", "include")
OUT = os.path.join(HERE, "librtb200.so")
BUILD = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
          "-I", CSRC, "-I", INC, "--expt-relaxed-constexpr"]
UNITS = [
    ("rt_trace.cu", ["--fmad=false"]),
    ("rt_shade.cu", []),
    ("rt_photon.cu", []),
    ("rt_output.cu", ["--fmad=false"]),
    ("rt_build.cu", ["--fmad=false"]),
    ("rt_guide.cu", ["--fmad=false"]),
    ("rt_host.cu", []),
]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _deps():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(INC, f) for f in os.listdir(INC)]


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(p) > t for p in _deps() + [__file__])


def build(force=False, verbose=False, ptxas_v=False):
    if not force and not needs_build():
        return OUT
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    for src, extra in UNITS:
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        cmd = [nvcc()] + ARCH + COMMON + extra + (["-Xptxas", "-v"] if ptxas_v else []) + \
              ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [nvcc()] + ARCH + ["-shared", "-o", OUT + ".tmp"] + objs + ["-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_v="-v" in sys.argv)
    print(OUT)
