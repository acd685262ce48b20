"""The C ABI library loads and exports every symbol its headers declare
(no device calls: runs without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(epic_(?:gpu|srv|nc)_[a-z0-9_]+)\s*\(", text)))


@pytest.mark.parametrize("header", ["epic_gpu.h", "epic_gpu_testing.h", "epic_serve.h", "epic_nc.h"])
def test_library_exports_declared_symbols(header):
    import epic_b200
    lib = ctypes.CDLL(epic_b200.LIB_PATH)
    names = _declared(header)
    assert len(names) >= {"epic_gpu.h": 30, "epic_serve.h": 5, "epic_nc.h": 9}.get(header, 2)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_library_resolves_every_symbol():
    """RTLD_NOW: a symbol the library uses but does not define fails here, on
    the CPU, instead of at first use on a GPU."""
    import epic_b200
    ctypes.CDLL(epic_b200.LIB_PATH, mode=os.RTLD_NOW)


def test_binding_covers_abi():
    import epic_b200
    lib = epic_b200.load()      # binds every signature of epic_b200/abi.py
    assert lib.prefix == "epic_gpu_"


def test_oracle_exports_same_abi(olib):
    names = [n.replace("epic_gpu_", "epic_oracle_") for n in _declared("epic_gpu.h")
             if not n.startswith(("epic_gpu_get_stream", "epic_gpu_profile", "epic_gpu_kernel_time",
                                  "epic_gpu_launch_count", "epic_gpu_apply_vortcor_noalloc", "epic_gpu_autotune"))]
    missing = [n for n in names if not hasattr(olib.lib, n)]
    assert not missing, missing


def test_config_struct_matches_header():
    """sizeof(epic_cfg) / sizeof(epic_step_info) of the ctypes mirror match C."""
    import subprocess, tempfile
    from epic_b200.abi import EpicCfg, EpicStepInfo
    src = ('#include "epic_gpu.h"\n#include <stdio.h>\n#include <stddef.h>\n'
           'int main(){printf("%zu %zu %zu\\n", sizeof(epic_cfg), sizeof(epic_step_info), offsetof(epic_cfg, capacity));}')
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe])
        a, b, off = map(int, subprocess.check_output([exe]).split())
    assert a == ctypes.sizeof(EpicCfg) and b == ctypes.sizeof(EpicStepInfo)
    assert off == EpicCfg.capacity.offset


def test_every_struct_mirror_matches_c_layout():
    """Size and every field offset of each ctypes mirror (config, step info,
    initial-state spec, tuning, server request and result) equal the C
    compiler's for the headers."""
    import subprocess, tempfile
    from epic_b200.abi import EpicCfg, EpicStepInfo, EpicInitSpec, EpicTuning
    from epic_b200.serve import EpicRequest, EpicResult
    mirrors = {"epic_cfg": EpicCfg, "epic_step_info": EpicStepInfo, "epic_init_spec": EpicInitSpec,
               "epic_tuning": EpicTuning, "epic_request": EpicRequest, "epic_result": EpicResult}
    lines = ['#include "epic_gpu.h"', '#include "epic_serve.h"', "#include <stdio.h>", "#include <stddef.h>",
             "int main(){"]
    for cname, py in mirrors.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write("\n".join(lines))
        exe = os.path.join(d, "t")
        subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe])
        out = subprocess.check_output([exe]).decode().split("\n")
    for ln in filter(None, out):
        cname, what, val = ln.split()
        py = mirrors[cname]
        got = ctypes.sizeof(py) if what == "size" else getattr(py, what).offset
        assert got == int(val), (cname, what, got, val)


def test_fortran_config_type_matches_mirror():
    """The Fortran shim's bind(C) epic_cfg lists the same fields, in the same
    order, with the same kinds and array lengths as the C struct (through its
    ctypes mirror, checked against C above).  Textual: no Fortran compiler in
    this image."""
    import ctypes as C
    from epic_b200.abi import EpicCfg
    text = open(os.path.join(ROOT, "fortran", "epic_gpu_iface.f90")).read()
    body = re.search(r"type, bind\(C\) :: epic_cfg\n(.*?)end type epic_cfg", text, re.S).group(1)
    kinds = {"c_int32_t": C.c_int32, "c_int64_t": C.c_int64, "c_double": C.c_double}
    fields = []
    for ln in body.splitlines():
        ln = ln.split("!")[0].strip()
        if not ln:
            continue
        m = re.match(r"(?:integer|real)\((c_\w+)\)\s*::\s*(.*)", ln)
        assert m, ln
        for item in re.findall(r"(\w+)(?:\((\d+)\))?", m.group(2)):
            name, dim = item
            t = kinds[m.group(1)]
            fields.append((name, t * int(dim) if dim else t))
    mirror = [(n, t) for n, t in EpicCfg._fields_]
    assert [n for n, _ in fields] == [n for n, _ in mirror]
    for (n, t), (_, u) in zip(fields, mirror):
        assert C.sizeof(t) == C.sizeof(u) and getattr(t, "_type_", None) == getattr(u, "_type_", None), n


def test_fortran_interfaces_match_c_prototypes():
    """Every bind(C) function of the Fortran shim names a declared C entry
    point and passes as many arguments as its prototype."""
    text = open(os.path.join(ROOT, "fortran", "epic_gpu_iface.f90")).read()
    hdr = "".join(open(os.path.join(ROOT, "include", h)).read() for h in os.listdir(os.path.join(ROOT, "include")))
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    protos = {}
    for m in re.finditer(r"\b(epic_\w+)\s*\(([^;{]*?)\)\s*;", hdr):
        args = m.group(2).strip()
        protos[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    found = 0
    for m in re.finditer(r"(?:function|subroutine)\s+\w+\s*\(([^)]*)\)\s*&?\s*bind\(C,\s*name=\"(\w+)\"\)", text):
        args, cname = m.group(1).strip(), m.group(2)
        assert cname in protos, cname
        n = 0 if not args else args.count(",") + 1
        assert n == protos[cname], (cname, n, protos[cname])
        found += 1
    assert found == len(re.findall(r"bind\(C,\s*name=", text)) >= 17


def test_library_has_no_undefined_own_symbols():
    """Every function of the library's own namespace is defined: a shared
    library links with undefined symbols and would only fail when loaded."""
    import subprocess
    lib = os.path.join(ROOT, "epic_b200", "libepic_b200.so")
    if not os.path.exists(lib):
        pytest.skip("library not built")
    out = subprocess.check_output(["nm", "-D", "--undefined-only", lib]).decode()
    own = [ln for ln in out.splitlines() if "epic" in ln.lower()]
    assert not own, own
