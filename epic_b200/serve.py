"""Served ensembles of independent EPIC simulations on one GPU
(include/epic_serve.h, bound through ctypes).

A request is a configuration (grid, options, precision form), a device-side
initial state (epic_init_spec) and a number of steps.  The server runs up to
`slots` requests at a time, each on its own context and CUDA stream, and
admits queued requests first come, first served as slots and device memory
free up.
"""
from __future__ import annotations

import ctypes as C
import math

from . import abi, initial, load


class EpicRequest(C.Structure):
    _fields_ = [("cfg", abi.EpicCfg), ("init", abi.EpicInitSpec), ("steps", C.c_int32), ("tune", C.c_int32)]


class EpicResult(C.Structure):
    _fields_ = [
        ("id", C.c_int64), ("status", C.c_int32), ("slot", C.c_int32),
        ("t_submit", C.c_double), ("t_start", C.c_double), ("t_done", C.c_double),
        ("parcel_steps", C.c_int64), ("n_parcels", C.c_int64), ("t_final", C.c_double),
        ("ke", C.c_double), ("enstrophy", C.c_double), ("device_bytes", C.c_double),
        ("message", C.c_char * 160),
    ]

    def as_dict(self) -> dict:
        d = {name: getattr(self, name) for name, _ in self._fields_}
        d["message"] = d["message"].decode(errors="replace")
        return d


def _bind(lib):
    L = lib.lib
    L.epic_srv_create.argtypes = [C.c_int32, C.c_double, C.POINTER(C.c_void_p)]
    L.epic_srv_submit.argtypes = [C.c_void_p, C.POINTER(EpicRequest), C.POINTER(C.c_int64)]
    L.epic_srv_wait.argtypes = [C.c_void_p, C.c_int64, C.POINTER(EpicResult)]
    L.epic_srv_counts.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.epic_srv_set_policy.argtypes = [C.c_void_p, C.c_int32]
    L.epic_srv_destroy.argtypes = [C.c_void_p]
    L.epic_srv_destroy.restype = None
    for f in (L.epic_srv_create, L.epic_srv_submit, L.epic_srv_wait, L.epic_srv_counts, L.epic_srv_set_policy):
        f.restype = C.c_int
    return L


def request(kind: str, n: tuple, seed: int = 1, klm=(1, 1, 1), steps: int = 100, precision: int = 1,
            lib=None, tune: bool = False, **options) -> EpicRequest:
    """A request for a thermal or Beltrami simulation on an n = (nx, ny, nz)
    grid with the benchmark workloads' domains and options; tune lets a new
    context pick its launch shapes by timing (epic_gpu_autotune)."""
    lib = lib or load()
    nx, ny, nz = n
    if kind == "thermal":
        extent = (6.28, 6.28, 6.28 * nz / nx)
        lower = (-0.5 * extent[0], -0.5 * extent[1], 0.0)
        opts = dict(min_vratio=40.0, lambda_max=4.0, bndry_zeta_zero=(1, 1))
        spec = abi.init_spec(abi.INIT_THERMAL, seed=seed, bubbles=((0.0, 0.0, 1.5 * nz / nx, 0.5),))
    elif kind == "beltrami":
        extent = (2 * math.pi, 2 * math.pi, math.pi)
        lower = (-math.pi, -math.pi, -0.5 * math.pi)
        opts = dict(min_vratio=40.0, lambda_max=4.0, bndry_zeta_zero=beltrami_zeta_flags(n, klm))
        spec = abi.init_spec(abi.INIT_BELTRAMI, klm=klm)
    else:
        raise KeyError(kind)
    # room for the splits of the stretched Beltrami shapes
    opts.update(precision=precision, keep_order=0, capacity=4 * nx * ny * nz * 8 + 1024)
    opts.update(options)
    r = EpicRequest()
    r.cfg = lib.default_config(nx, ny, nz, lower, extent, **opts)
    r.init = spec
    r.steps = steps
    r.tune = int(tune)
    return r


def beltrami_zeta_flags(n, klm):
    """set_zeta_boundary_flag of the gridded Beltrami vertical vorticity."""
    import numpy as np
    nx, ny, nz = n
    lower = (-math.pi, -math.pi, -0.5 * math.pi)
    dx = (2 * math.pi / nx, 2 * math.pi / ny, math.pi / nz)
    X, Y, Z = np.meshgrid(lower[0] + np.arange(nx) * dx[0], lower[1] + np.arange(ny) * dx[1],
                          lower[2] + np.arange(nz + 1) * dx[2], indexing="ij")
    zg = initial.beltrami_vorticity(np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1), *klm)[:, 2].reshape(X.shape)
    return initial.zeta_boundary_flags(zg)


ARRIVAL = 0          # EPIC_SRV_ARRIVAL
SHORTEST_FIRST = 1   # EPIC_SRV_SHORTEST_FIRST
POLICIES = {"arrival": ARRIVAL, "shortest-first": SHORTEST_FIRST}


class Server:
    """epic_server: submit(request) -> id; wait(id) -> result dict.  policy:
    admission order, "arrival" or "shortest-first" (smallest estimated work,
    cells x parcels per cell x steps, first)."""

    def __init__(self, slots: int = 4, hbm_fraction: float = 0.8, lib=None, policy: str = "arrival"):
        code = POLICIES[policy]
        self.lib = lib or load()
        self.L = _bind(self.lib)
        h = C.c_void_p()
        rc = self.L.epic_srv_create(slots, hbm_fraction, C.byref(h))
        if rc != 0:
            raise abi.EpicError(rc, "epic_srv_create", "server creation failed")
        self.h = h
        rc = self.L.epic_srv_set_policy(self.h, code)
        if rc != 0:
            self.close()
            raise abi.EpicError(rc, "epic_srv_set_policy", policy)

    def submit(self, req: EpicRequest) -> int:
        i = C.c_int64()
        rc = self.L.epic_srv_submit(self.h, C.byref(req), C.byref(i))
        if rc != 0:
            raise abi.EpicError(rc, "epic_srv_submit", "")
        return i.value

    def wait(self, rid: int) -> dict:
        r = EpicResult()
        rc = self.L.epic_srv_wait(self.h, rid, C.byref(r))
        if rc != 0:
            raise abi.EpicError(rc, "epic_srv_wait", "")
        return r.as_dict()

    def counts(self):
        q, r, d = C.c_int64(), C.c_int64(), C.c_int64()
        self.L.epic_srv_counts(self.h, C.byref(q), C.byref(r), C.byref(d))
        return q.value, r.value, d.value

    def close(self):
        if getattr(self, "h", None):
            self.L.epic_srv_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
