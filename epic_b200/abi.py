"""ctypes binding of the C ABI declared in include/epic_gpu.h.

The same binding drives any library that exports the ABI under a symbol
prefix (the CUDA product exports ``epic_gpu_*``).  Arrays follow the
reference's Fortran layouts: parcel attributes are C-contiguous ``(n, c)``
float64 arrays (= Fortran ``(c, n)``), gridded fields are ``(nx, ny, nz+3)``
float64 arrays with z fastest and z running from -1 to nz+1.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

EPIC_OK = 0
ERROR_NAMES = {
    1: "EPIC_ERR_CONFIG",
    2: "EPIC_ERR_CAPACITY",
    3: "EPIC_ERR_NUMERICAL",
    4: "EPIC_ERR_CUDA",
    5: "EPIC_ERR_TIMEOUT",
    6: "EPIC_ERR_ARG",
    7: "EPIC_ERR_STATE",
    8: "EPIC_ERR_PARCEL_COUNT",
    9: "EPIC_ERR_IO",
}

# field ids (enum epic_field_id)
VELOG = (0, 1, 2)
VORTG = (3, 4, 5)
VTEND = (6, 7, 8)
VELGRADG = tuple(range(9, 17))
TBUOYG, DBUOYG, HUMG, VOLG, NPARG, NSPARG = 17, 18, 19, 20, 21, 22
FIELD_NAMES = {
    **{VELOG[i]: f"velog_{c}" for i, c in enumerate("xyz")},
    **{VORTG[i]: f"vortg_{c}" for i, c in enumerate("xyz")},
    **{VTEND[i]: f"vtend_{c}" for i, c in enumerate("xyz")},
    **{VELGRADG[i]: n for i, n in enumerate(
        ["dudx", "dudy", "dudz", "dvdx", "dvdy", "dvdz", "dwdx", "dwdy"])},
    TBUOYG: "tbuoyg", DBUOYG: "dbuoyg", HUMG: "humg", VOLG: "volg",
    NPARG: "nparg", NSPARG: "nsparg",
}

PRECISION_FP64 = 0
PRECISION_MIXED = 1


class EpicCfg(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("lower", C.c_double * 3), ("extent", C.c_double * 3),
        ("size_factor", C.c_double), ("grow_factor", C.c_double), ("shrink_factor", C.c_double),
        ("n_per_cell", C.c_int32),
        ("lambda_max", C.c_double), ("min_vratio", C.c_double),
        ("correction_iters", C.c_int32),
        ("gradient_pref", C.c_double), ("max_compression", C.c_double),
        ("t_initial", C.c_double), ("t_limit", C.c_double), ("alpha", C.c_double),
        ("precise_stop", C.c_int32), ("use_fixed_dt", C.c_int32),
        ("fixed_dt", C.c_double),
        ("rk_order", C.c_int32),
        ("gravity", C.c_double), ("L_v", C.c_double), ("c_p", C.c_double),
        ("theta_0", C.c_double), ("q_0", C.c_double), ("height_c", C.c_double),
        ("ang_vel", C.c_double), ("lat_degrees", C.c_double),
        ("l_planetary_vorticity", C.c_int32),
        ("bndry_zeta_zero", C.c_int32 * 2),
        ("capacity", C.c_int64),
        ("precision", C.c_int32),
        ("keep_order", C.c_int32),
        ("damping_vorticity_prefactor", C.c_double),
        ("damping_scalars_prefactor", C.c_double),
        ("damping_vorticity", C.c_int32),
        ("damping_surface_vorticity", C.c_int32),
        ("damping_scalars", C.c_int32),
        ("damping_surface_scalars", C.c_int32),
        ("labels", C.c_int32),
        ("label_seed", C.c_int32),
    ]


class EpicStepInfo(C.Structure):
    _fields_ = [
        ("t", C.c_double), ("dt", C.c_double),
        ("n_parcels", C.c_int64), ("n_splits", C.c_int64), ("n_merges", C.c_int64),
        ("parcel_stats", C.c_double * 18),
        ("field_stats", C.c_double * 11),
    ]


INIT_THERMAL, INIT_BELTRAMI, INIT_DEFAULT = 0, 1, 2


class EpicInitSpec(C.Structure):
    """epic_init_spec of include/epic_gpu.h (device-side initial states)."""
    _fields_ = [
        ("kind", C.c_int32), ("n_per_cell", C.c_int32), ("seed", C.c_uint64),
        ("k", C.c_int32), ("l", C.c_int32), ("m", C.c_int32),
        ("n_bubbles", C.c_int32), ("bubble", (C.c_double * 4) * 4),
    ]


def init_spec(kind, n_per_cell=8, seed=1234, klm=(1, 1, 1), bubbles=((0.0, 0.0, 1.5, 0.5),)) -> EpicInitSpec:
    s = EpicInitSpec()
    s.kind = kind
    s.n_per_cell = n_per_cell
    s.seed = seed
    s.k, s.l, s.m = klm
    s.n_bubbles = len(bubbles)
    for b, row in enumerate(bubbles):
        for q in range(4):
            s.bubble[b][q] = row[q]
    return s


class EpicTuning(C.Structure):
    """epic_tuning of include/epic_gpu.h (autotuner choices and times)."""
    _fields_ = [("lg_par2grid", C.c_int32), ("lg_vol2grid", C.c_int32), ("fft_path", C.c_int32),
                ("reserved", C.c_int32), ("ms_par2grid", C.c_double), ("ms_vol2grid", C.c_double),
                ("ms_fft", C.c_double)]


class EpicError(RuntimeError):
    def __init__(self, code: int, func: str, msg: str):
        self.code = code
        super().__init__(f"{func} failed with {ERROR_NAMES.get(code, code)}: {msg}")


_D = C.POINTER(C.c_double)
_I32 = C.POINTER(C.c_int32)
_I64 = C.POINTER(C.c_int64)
_VP = C.c_void_p

# name -> argtypes (after the prefix); every function returns int unless noted
_SIGNATURES = {
    "default_config": [C.POINTER(EpicCfg)],
    "create": [C.POINTER(EpicCfg), C.POINTER(_VP)],
    "sync": [_VP],
    "set_parcels": [_VP, C.c_int64, _D, _D, _D, _D, _D, _D],
    "get_parcels": [_VP, C.c_int64, _I64, _D, _D, _D, _D, _D, _D],
    "num_parcels": [_VP, _I64],
    "get_labels": [_VP, C.c_int64, _I64, _I64, _D],
    "set_labels": [_VP, C.c_int64, _I64, _D],
    "get_parcel_rk": [_VP, C.c_int64, _I64, _D, _D, _D, _D],
    "set_parcel_rk": [_VP, C.c_int64, _D, _D, _D],
    "get_field": [_VP, C.c_int, _D],
    "set_field": [_VP, C.c_int, _D],
    "init_correction": [_VP],
    "apply_vortcor": [_VP],
    "par2grid": [_VP, C.c_int],
    "vor2vel": [_VP],
    "vorticity_tendency": [_VP],
    "time_step": [_VP, C.c_double, _D],
    "grid2par": [_VP, C.c_int],
    "rk_step": [_VP, _D, _D],
    "merge": [_VP, _I64],
    "get_merge_pairs": [_VP, C.c_int64, _I64, _I32, _I32],
    "split": [_VP, _I64],
    "apply_laplace": [_VP, C.c_int],
    "apply_gradient": [_VP, C.c_int],
    "vol2grid": [_VP, C.c_int],
    "parcel_diagnostics": [_VP, _D],
    "field_diagnostics": [_VP, _D],
    "step": [_VP, _D, C.POINTER(EpicStepInfo)],
    "parcel_damp": [_VP, C.c_double],
    "set_bndry_fluxes": [_VP, _D, _D],
    "apply_bndry_fluxes": [_VP, C.c_double],
    "init_from_grids": [_VP, _D, _D, _D, _I32],
}


def _ptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(_D)


def _f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        a = a.reshape(shape)
    return a


class EpicLib:
    """Thin typed wrapper around one shared library exporting the ABI."""

    def __init__(self, path: str, prefix: str):
        if not os.path.exists(path):
            raise FileNotFoundError(
                f"EPIC library {path} is missing; build it first "
                "(python -m epic_b200.build)")
        self.path = path
        self.prefix = prefix
        self.lib = C.CDLL(path)
        self.fn = {}
        for name, args in _SIGNATURES.items():
            f = getattr(self.lib, prefix + name)
            f.argtypes = args
            f.restype = C.c_int
            self.fn[name] = f
        # entry points only the CUDA library has
        for name, args in (("init_state", [_VP, C.POINTER(EpicInitSpec)]),
                           ("autotune", [_VP, C.POINTER(EpicTuning)]),
                           ("write_parcels_nc", [_VP, C.c_char_p, C.c_double]),
                           ("read_parcels_nc", [_VP, C.c_char_p, _D]),
                           ("write_fields_nc", [_VP, C.c_char_p, C.c_double]),
                           ("init_from_field_file", [_VP, C.c_char_p, _I32])):
            if hasattr(self.lib, prefix + name):
                f = getattr(self.lib, prefix + name)
                f.argtypes = args
                f.restype = C.c_int
                self.fn[name] = f
        d = getattr(self.lib, prefix + "destroy")
        d.argtypes = [_VP]
        d.restype = None
        self.fn["destroy"] = d
        e = getattr(self.lib, prefix + "last_error")
        e.argtypes = [_VP]
        e.restype = C.c_char_p
        self.fn["last_error"] = e

    def default_config(self, nx, ny, nz, lower, extent, **kw) -> EpicCfg:
        cfg = EpicCfg()
        self.fn["default_config"](C.byref(cfg))
        cfg.nx, cfg.ny, cfg.nz = int(nx), int(ny), int(nz)
        for k in range(3):
            cfg.lower[k] = float(lower[k])
            cfg.extent[k] = float(extent[k])
        for k, v in kw.items():
            if k == "bndry_zeta_zero":
                cfg.bndry_zeta_zero[0], cfg.bndry_zeta_zero[1] = int(v[0]), int(v[1])
            else:
                setattr(cfg, k, v)
        return cfg


class EpicContext:
    """One simulation context (epic_ctx*) of a library."""

    def __init__(self, lib: EpicLib, cfg: EpicCfg):
        self.lib = lib
        self.cfg = cfg
        self.nx, self.ny, self.nz = cfg.nx, cfg.ny, cfg.nz
        h = _VP()
        rc = lib.fn["create"](C.byref(cfg), C.byref(h))
        if rc != EPIC_OK:
            raise EpicError(rc, lib.prefix + "create", "context creation failed")
        self.h = h

    # -- plumbing ---------------------------------------------------------
    def _call(self, name, *args):
        rc = self.lib.fn[name](self.h, *args)
        if rc != EPIC_OK:
            msg = self.lib.fn["last_error"](self.h)
            raise EpicError(rc, self.lib.prefix + name, msg.decode(errors="replace") if msg else "")
        return rc

    def close(self):
        if getattr(self, "h", None):
            self.lib.fn["destroy"](self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def field_shape(self):
        return (self.nx, self.ny, self.nz + 3)

    # -- parcels ----------------------------------------------------------
    def set_parcels(self, pos, vor, B, vol, buoy, hum=None):
        n = len(vol)
        pos = _f64(pos, (n, 3)); vor = _f64(vor, (n, 3)); B = _f64(B, (n, 5))
        vol = _f64(vol, (n,)); buoy = _f64(buoy, (n,))
        hum = _f64(hum, (n,)) if hum is not None else np.zeros(n)
        self._keep = (pos, vor, B, vol, buoy, hum)
        self._call("set_parcels", C.c_int64(n), _ptr(pos), _ptr(vor), _ptr(B), _ptr(vol),
                   _ptr(buoy), _ptr(hum))

    def num_parcels(self) -> int:
        n = C.c_int64()
        self._call("num_parcels", C.byref(n))
        return n.value

    def get_parcels(self) -> dict:
        n = self.num_parcels()
        out = dict(pos=np.empty((n, 3)), vor=np.empty((n, 3)), B=np.empty((n, 5)),
                   vol=np.empty(n), buoy=np.empty(n), hum=np.empty(n))
        nn = C.c_int64()
        self._call("get_parcels", C.c_int64(n), C.byref(nn), _ptr(out["pos"]), _ptr(out["vor"]),
                   _ptr(out["B"]), _ptr(out["vol"]), _ptr(out["buoy"]), _ptr(out["hum"]))
        return out

    def get_labels(self):
        """(label int64 (n,), dilution (n,)) of the parcels (cfg.labels = 1)."""
        n = self.num_parcels()
        lab, dil = np.empty(n, dtype=np.int64), np.empty(n)
        nn = C.c_int64()
        self._call("get_labels", C.c_int64(n), C.byref(nn), lab.ctypes.data_as(_I64), _ptr(dil))
        return lab, dil

    def set_labels(self, label, dilution):
        lab = np.ascontiguousarray(label, dtype=np.int64)
        dil = _f64(dilution, (len(lab),))
        self._call("set_labels", C.c_int64(len(lab)), lab.ctypes.data_as(_I64), _ptr(dil))

    def get_parcel_rk(self) -> dict:
        n = self.num_parcels()
        out = dict(delta_pos=np.empty((n, 3)), delta_vor=np.empty((n, 3)),
                   strain=np.empty((n, 8)), delta_b=np.empty((n, 5)))
        nn = C.c_int64()
        self._call("get_parcel_rk", C.c_int64(n), C.byref(nn), _ptr(out["delta_pos"]),
                   _ptr(out["delta_vor"]), _ptr(out["strain"]), _ptr(out["delta_b"]))
        return out

    def set_parcel_rk(self, delta_pos, delta_vor, delta_b):
        n = len(delta_pos)
        a = _f64(delta_pos, (n, 3)); b = _f64(delta_vor, (n, 3)); c = _f64(delta_b, (n, 5))
        self._call("set_parcel_rk", C.c_int64(n), _ptr(a), _ptr(b), _ptr(c))

    # -- fields -----------------------------------------------------------
    def get_field(self, fid: int) -> np.ndarray:
        out = np.empty(self.field_shape)
        self._call("get_field", C.c_int(fid), _ptr(out))
        return out

    def set_field(self, fid: int, arr):
        a = _f64(arr, self.field_shape)
        self._call("set_field", C.c_int(fid), _ptr(a))

    # -- step pieces ------------------------------------------------------
    def sync(self):
        self._call("sync")

    def init_correction(self):
        self._call("init_correction")

    def apply_vortcor(self):
        self._call("apply_vortcor")

    def par2grid(self, reuse=False):
        self._call("par2grid", C.c_int(int(reuse)))

    def vol2grid(self, reuse=False):
        self._call("vol2grid", C.c_int(int(reuse)))

    def vor2vel(self):
        self._call("vor2vel")

    def vorticity_tendency(self):
        self._call("vorticity_tendency")

    def time_step(self, t: float) -> float:
        dt = C.c_double()
        self._call("time_step", C.c_double(t), C.byref(dt))
        return dt.value

    def grid2par(self, add=False):
        self._call("grid2par", C.c_int(int(add)))

    def init_state(self, spec: "EpicInitSpec"):
        self._call("init_state", C.byref(spec))

    def autotune(self) -> dict:
        t = EpicTuning()
        self._call("autotune", C.byref(t))
        return {name: getattr(t, name) for name, _ in t._fields_ if name != "reserved"}

    def rk_step(self, t: float):
        tt = C.c_double(t)
        dt = C.c_double()
        self._call("rk_step", C.byref(tt), C.byref(dt))
        return tt.value, dt.value

    def merge(self) -> int:
        n = C.c_int64()
        self._call("merge", C.byref(n))
        return n.value

    def merge_pairs(self):
        """(isma, iclo) of the last merge, 1-based, in merge order."""
        n = C.c_int64()
        # the count first (a zero capacity only reports it)
        self.lib.fn["get_merge_pairs"](self.h, C.c_int64(0), C.byref(n), None, None)
        cap = max(n.value, 1)
        isma = np.empty(cap, dtype=np.int32)
        iclo = np.empty(cap, dtype=np.int32)
        n = C.c_int64()
        self._call("get_merge_pairs", C.c_int64(cap), C.byref(n),
                   isma.ctypes.data_as(_I32), iclo.ctypes.data_as(_I32))
        return isma[:n.value].copy(), iclo[:n.value].copy()

    def split(self) -> int:
        n = C.c_int64()
        self._call("split", C.byref(n))
        return n.value

    def apply_laplace(self, reuse=False):
        self._call("apply_laplace", C.c_int(int(reuse)))

    def apply_gradient(self, reuse=True):
        self._call("apply_gradient", C.c_int(int(reuse)))

    def parcel_diagnostics(self) -> np.ndarray:
        st = np.zeros(18)
        self._call("parcel_diagnostics", _ptr(st))
        return st

    def field_diagnostics(self) -> np.ndarray:
        st = np.zeros(11)
        self._call("field_diagnostics", _ptr(st))
        return st

    def parcel_damp(self, dt: float):
        self._call("parcel_damp", C.c_double(dt))

    def init_from_grids(self, vortg, tbuoyg, humg=None):
        """parcel_default + init_refine + init_parcels_from_grids +
        set_zeta_boundary_flag; vortg (3, nx, ny, nz+3), tbuoyg and humg
        (nx, ny, nz+3).  Returns the zeta boundary flags."""
        v = _f64(vortg, (3,) + self.field_shape)
        b = _f64(tbuoyg, self.field_shape)
        h = _f64(humg, self.field_shape) if humg is not None else None
        flags = np.zeros(2, dtype=np.int32)
        self._call("init_from_grids", _ptr(v), _ptr(b), _ptr(h), flags.ctypes.data_as(_I32))
        return int(flags[0]), int(flags[1])

    # -- files in the reference's netCDF layout (include/epic_nc.h) --------
    def write_parcels_nc(self, path, t: float):
        self._call("write_parcels_nc", os.fsencode(path), C.c_double(t))

    def read_parcels_nc(self, path) -> float:
        """Parcels (and zeta flags) from a parcel file; returns its time."""
        t = C.c_double()
        self._call("read_parcels_nc", os.fsencode(path), C.byref(t))
        return t.value

    def write_fields_nc(self, path, t: float):
        self._call("write_fields_nc", os.fsencode(path), C.c_double(t))

    def init_from_field_file(self, path):
        """init_from_grids on the vorticity, buoyancy and humidity of a field
        file's last record; returns the zeta boundary flags."""
        flags = np.zeros(2, dtype=np.int32)
        self._call("init_from_field_file", os.fsencode(path), flags.ctypes.data_as(_I32))
        return int(flags[0]), int(flags[1])

    def set_bndry_fluxes(self, bflux=None, hflux=None):
        """bflux, hflux: (nx, ny) arrays (= the reference's (ny, nx) Fortran
        datasets); bflux None turns the fluxes off."""
        shape = (self.nx, self.ny)
        b = _f64(bflux, shape) if bflux is not None else None
        h = _f64(hflux, shape) if hflux is not None else None
        self._call("set_bndry_fluxes", _ptr(b), _ptr(h))

    def apply_bndry_fluxes(self, dt: float):
        self._call("apply_bndry_fluxes", C.c_double(dt))

    def step(self, t: float):
        tt = C.c_double(t)
        info = EpicStepInfo()
        self._call("step", C.byref(tt), C.byref(info))
        return tt.value, info
