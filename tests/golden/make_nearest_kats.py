"""Regenerate tests/golden/nearest_kats.json from the reference's nearest-parcel
unit tests (unit-tests/3d/test_mpi_nearest_5.f90 .. _20.f90), read as text.

Every one of those tests places the same constellation of parcels in each
cell (i, j) of the layer k = 1 of a 10 x 10 x 10 grid on the unit cube (loop
j outer, i inner), runs find_nearest with lambda_max = 5 and min_vratio = 8,
and checks the number of merges against a stated count, for one or more
constellations in turn.  This script records, per test and constellation,
the parcels of one cell as (x offset, y offset, volume factor) -- offsets as
sign, grid axis and factor of the cell width, in the order the test fills
the container -- and the expected count.  Factors written as single
precision literals are stored as their single precision value.

    python tests/golden/make_nearest_kats.py <path of the reference source tree>
"""
import json
import os
import re
import sys

import numpy as np

if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_nearest_kats.py <path of the reference source tree>")
D = os.path.join(sys.argv[1], "unit-tests", "3d")


def literal(tok):
    t = tok.lower()
    if t.endswith("d0"):
        return float(t[:-2])
    return float(np.float32(float(t)))   # default real


POS = re.compile(r"parcels%position\((\d),\s*l\)\s*=\s*([xyz])\s*(?:([+-])\s*(?:dx\((\d)\)\s*\*\s*([0-9.d]+)|([0-9.d]+)\s*\*\s*dx\((\d)\)))?\s*$")
VOL = re.compile(r"parcels%volume\(l\)\s*=\s*([0-9.d]+)\s*\*\s*vmin")


def placements(text):
    out = {}
    for m in re.finditer(r"subroutine (cell_placement(?:_\d+)?)\(.*?\n(.*?)end subroutine \1", text, re.S):
        name, body = m.group(1), m.group(2)
        parcels, cur = [], None
        for ln in body.splitlines():
            ln = ln.split("!")[0].strip()
            if not ln:
                continue
            p = POS.match(ln)
            if p:
                comp, base = int(p.group(1)), p.group(2)
                assert base == "xyz"[comp - 1], ln
                if cur is None:
                    cur = {"off": [None, None], "vol": None}
                if comp < 3:
                    if p.group(3):
                        axis = int(p.group(4) or p.group(7))
                        fac = literal(p.group(5) or p.group(6))
                        cur["off"][comp - 1] = [1 if p.group(3) == "+" else -1, axis, fac]
                    else:
                        cur["off"][comp - 1] = [0, comp, 0.0]
                continue
            v = VOL.match(ln)
            if v:
                cur["vol"] = literal(v.group(1))
                continue
            if re.match(r"l\s*=\s*l\s*\+\s*1$", ln):
                parcels.append(cur)
                cur = None
                continue
            assert "position" not in ln and "volume" not in ln, ln
        out[name] = parcels
    return out


def cases(text, places):
    """The constellations run by the main program and their expected merges."""
    main = text.split("contains")[0]
    seq = re.findall(r"call parcel_setup(?:\((\d+)\))?|call check_result\((\d+)\)|check_array\(2\)\s*==\s*(\d+)\)", text)
    calls = re.findall(r"call parcel_setup(?:\((\d+)\))?", main)
    checks = re.findall(r"call check_result\((\d+)\)", main)
    if not checks:
        checks = re.findall(r"check_array\(2\)\s*==\s*(\d+)\)", text)
    assert len(calls) == len(checks), (calls, checks)
    out = []
    for c, n in zip(calls, checks):
        name = "cell_placement" + (f"_{c}" if c else "")
        out.append({"setup": int(c) if c else 0, "expected": int(n), "cell": places[name]})
    return out


def header(text):
    t = {}
    for key, pat in (("lambda_max", r"parcel%lambda_max\s*=\s*(\w+)"), ("min_vratio", r"parcel%min_vratio\s*=\s*([0-9.d]+)"),
                     ("nx", r"\bnx\s*=\s*(\d+)"), ("ny", r"\bny\s*=\s*(\d+)"), ("nz", r"\bnz\s*=\s*(\d+)")):
        t[key] = re.search(pat, text).group(1)
    assert t["lambda_max"] == "five" and t["nx"] == t["ny"] == t["nz"] == "10", t
    assert "box%lo(3)+1, box%lo(3)+1" in text and "extent = (/one, one, one/)" in text
    return {"lambda_max": 5.0, "min_vratio": literal(t["min_vratio"]), "n": 10}


out = {}
for k in range(5, 21):
    f = os.path.join(D, f"test_mpi_nearest_{k}.f90")
    text = open(f).read()
    out[f"test_mpi_nearest_{k}"] = dict(header(text), cases=cases(text, placements(text)))
dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "nearest_kats.json")
with open(dst, "w") as fh:
    json.dump(out, fh, indent=1)
print("wrote", dst, sum(len(v["cases"]) for v in out.values()), "constellations")
