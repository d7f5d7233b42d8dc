"""Build recipe for the CPU oracle (test infrastructure, not product code).

Two shared libraries are built from ``self_oracle.cpp`` into ``oracle/_build``:

* ``liboracle.so``      -- parity build: ``-O2 -ffp-contract=off`` so no FMA
  contraction changes the rounding of the restated Fortran expressions.
* ``liboracle_fast.so`` -- timed CPU baseline: ``-O3 -march=x86-64-v3`` (AVX2
  and FMA, portable to the GPU hosts) with OpenMP over elements.

The reference itself (Fortran + hipfort + MPI + HDF5) cannot be compiled in
this image, so no ``oracle/_ref`` build exists.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_build")
SRC = os.path.join(HERE, "self_oracle.cpp")

BUILDS = {
    "liboracle.so": ["-O2", "-ffp-contract=off"],
    "liboracle_fast.so": ["-O3", "-march=x86-64-v3", "-mtune=native"],
}


def build(force: bool = False) -> None:
    os.makedirs(OUT, exist_ok=True)
    for name, flags in BUILDS.items():
        dst = os.path.join(OUT, name)
        if not force and os.path.exists(dst) and os.path.getmtime(dst) >= os.path.getmtime(SRC):
            continue
        cmd = ["g++", "-std=c++17", "-fPIC", "-shared", "-fopenmp", *flags, "-o", dst, SRC]
        subprocess.run(cmd, check=True)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
