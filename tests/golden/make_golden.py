"""Regenerate tests/golden/scherzinger_BDV.npz from the reference's golden
vectors (unit-tests/3d/B.asc, D.asc, V.asc, produced by numpy.linalg.eigh in
unit-tests/3d/numpy_eigh.py).  Run once where the reference tree is mounted:

    python tests/golden/make_golden.py /path/to/epic
"""
import os
import sys

import numpy as np

if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_golden.py <path of the reference source tree>")
ref = sys.argv[1]
d = os.path.join(ref, "unit-tests", "3d")
B = np.loadtxt(os.path.join(d, "B.asc"), skiprows=1)
D = np.loadtxt(os.path.join(d, "D.asc"), skiprows=1)
V = np.loadtxt(os.path.join(d, "V.asc"), skiprows=1)
out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "scherzinger_BDV.npz")
np.savez_compressed(out, B=B, D=D, V=V)
print("wrote", out, B.shape, D.shape, V.shape)
