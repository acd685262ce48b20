"""ORACLE -- test infrastructure only.

CPU FP64 restatement of the reference EPIC 3-D parcel step (see
oracle_core.hpp for what pins it).  Only tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline leg may import this package, and only as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libepic_oracle.so")
LIB_OMP = os.path.join(HERE, "_build", "libepic_oracle_omp.so")


def build(quiet: bool = True) -> None:
    """Compile the oracle (make in oracle/)."""
    out = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def load(threads: bool = False):
    """Return an EpicLib bound to the oracle (prefix epic_oracle_)."""
    from epic_b200.abi import EpicLib
    path = LIB_OMP if threads else LIB
    if not os.path.exists(path):
        build()
    lib = EpicLib(path, "epic_oracle_")
    f = lib.lib.epic_oracle_eigen
    f.argtypes = [C.c_int64, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int]
    f.restype = C.c_int
    g = lib.lib.epic_oracle_transform
    g.argtypes = [C.c_int, C.c_int64, C.c_int, C.POINTER(C.c_double)]
    g.restype = C.c_int
    return lib


def eigen(lib, A6: np.ndarray, values_only: bool = False):
    A6 = np.ascontiguousarray(A6, dtype=np.float64).reshape(-1, 6)
    n = len(A6)
    D = np.empty((n, 3))
    V = np.empty((n, 9))
    P = C.POINTER(C.c_double)
    lib.lib.epic_oracle_eigen(n, A6.ctypes.data_as(P), D.ctypes.data_as(P), V.ctypes.data_as(P),
                              int(values_only))
    return D, V.reshape(n, 3, 3).transpose(0, 2, 1)  # V[i][:, j] = eigenvector j


def transform(lib, kind: str, x: np.ndarray) -> np.ndarray:
    """kind in {'forfft','revfft','dst','dct'}; x is (m, n) (dct: (m, n+1))."""
    k = {"forfft": 0, "revfft": 1, "dst": 2, "dct": 3}[kind]
    x = np.array(x, dtype=np.float64, order="C")
    m = x.shape[0]
    n = x.shape[1] - 1 if kind == "dct" else x.shape[1]
    lib.lib.epic_oracle_transform(k, m, n, x.ctypes.data_as(C.POINTER(C.c_double)))
    return x
