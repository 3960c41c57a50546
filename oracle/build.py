"""Build recipe for the oracle (TEST INFRASTRUCTURE ONLY).

Compiles ``oracle/negf_oracle.c`` with gcc into ``oracle/liboracle.so``.  The
library resolves LAPACK/BLAS at run time (``oracle_init``) from the ILP64
OpenBLAS that NumPy bundles, so nothing beyond gcc is needed to build it.

The reference itself (Fortran 90 + MPI + FFTW + LAPACK) cannot be compiled in
this image: there is no Fortran compiler, no MPI and no FFTW.  No
``oracle/_ref`` build exists for that reason.
"""
from __future__ import annotations

import glob
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
SRC = os.path.join(HERE, "negf_oracle.c")


def lapack_path() -> str:
    """Path of NumPy's bundled ILP64 OpenBLAS (exports scipy_zgetrf_64_ etc.)."""
    import numpy

    root = os.path.dirname(os.path.dirname(numpy.__file__))
    hits = sorted(glob.glob(os.path.join(root, "numpy.libs", "libscipy_openblas64_*.so")))
    if not hits:
        raise RuntimeError("NumPy's bundled ILP64 OpenBLAS was not found")
    return hits[0]


def build(force: bool = False) -> str:
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= max(os.path.getmtime(SRC),
                                             os.path.getmtime(os.path.join(HERE, "negf_oracle.h")))):
        return LIB
    cmd = ["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-std=gnu11", "-o", LIB, SRC, "-lm", "-ldl"]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
