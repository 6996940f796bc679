"""Build recipe for the CPU oracle (test infrastructure only).

Compiles oracle/rt_oracle.cpp into oracle/liboracle.so with the flags the
restatement needs: -ffp-contract=off (the reference is Rust, which never fuses
a*b+c into an FMA), AVX2 for the 8-wide slab test the reference uses
(src/bvh.rs:326-364), and -O3.  The reference itself (Rust, crates not vendored,
no toolchain) cannot be built here, so there is no oracle/_ref.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "rt_oracle.cpp")
OUT = os.path.join(HERE, "liboracle.so")
HDRS = [os.path.join(HERE, "..", "include", "rt_api.h"),
        os.path.join(HERE, "..", "include", "rt_spectral_tables.h")]

CXXFLAGS = ["-O3", "-std=c++17", "-mavx2", "-ffp-contract=off", "-fno-fast-math",
            "-fPIC", "-shared", "-pthread", "-Wall", "-Wno-unused-function"]


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(p) > t for p in [SRC] + HDRS)


def build(force=False, verbose=False):
    if not force and not needs_build():
        return OUT
    cmd = ["g++"] + CXXFLAGS + [SRC, "-o", OUT + ".tmp"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(OUT)
