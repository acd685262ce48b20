"""Parcel and field files in the reference's netCDF layout (include/epic_nc.h),
host arrays only: the classic-format writer and reader of the library,
without a device.

Parcel arrays follow EpicContext.get_parcels: pos, vor (n, 3), B (n, 5),
vol, buoy, hum (n,).  Fields follow EpicContext.get_field: (nx, ny, nz+3),
z fastest, rows z = -1 .. nz+1 (the files hold rows 0 .. nz)."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .abi import EpicError, _D, _I32, _I64, _f64, _ptr


class NcFiles:
    def __init__(self, lib):
        """lib: an EpicLib of the CUDA library (epic_b200.load())."""
        self.lib = lib.lib
        L = self.lib
        L.epic_nc_last_error.argtypes = []
        L.epic_nc_last_error.restype = C.c_char_p
        L.epic_nc_info.argtypes = [C.c_char_p, C.c_char_p, _I32, _D, _D, _I64, _I64, _D, _I32]
        L.epic_nc_write_parcels.argtypes = [C.c_char_p, _I32, _D, _D, _I32, C.c_double, C.c_int64,
                                            _D, _D, _D, _D, _D, _D]
        L.epic_nc_read_parcels.argtypes = [C.c_char_p, C.c_int64, _I64, _D, _D, _D, _D, _D, _D]
        L.epic_nc_read_field.argtypes = [C.c_char_p, C.c_char_p, C.c_int64, _I32, _D, _D, _D]
        L.epic_nc_write_field_file.argtypes = [C.c_char_p, _I32, _D, _D, _I32, C.c_double, C.c_int,
                                               C.POINTER(C.c_char_p), C.POINTER(C.c_char_p), C.POINTER(_D)]
        L.epic_nc_read_variable.argtypes = [C.c_char_p, C.c_char_p, C.c_int64, C.c_int64, _I64, _D]
        for f in (L.epic_nc_info, L.epic_nc_write_parcels, L.epic_nc_read_parcels, L.epic_nc_read_field,
                  L.epic_nc_write_field_file, L.epic_nc_read_variable):
            f.restype = C.c_int

    def _check(self, rc, name):
        if rc != 0:
            raise EpicError(rc, name, self.lib.epic_nc_last_error().decode(errors="replace"))

    @staticmethod
    def _box(ncells, origin, extent):
        return (np.ascontiguousarray(ncells, dtype=np.int32), _f64(origin, (3,)), _f64(extent, (3,)))

    def info(self, path) -> dict:
        ft = C.create_string_buffer(16)
        nc = np.zeros(3, dtype=np.int32)
        og, ex = np.zeros(3), np.zeros(3)
        npar, nst, t = C.c_int64(), C.c_int64(), C.c_double()
        z = np.zeros(2, dtype=np.int32)
        self._check(self.lib.epic_nc_info(os.fsencode(path), ft, nc.ctypes.data_as(_I32), _ptr(og), _ptr(ex),
                                          C.byref(npar), C.byref(nst), C.byref(t), z.ctypes.data_as(_I32)),
                    "epic_nc_info")
        return dict(file_type=ft.value.decode(errors="replace"), ncells=tuple(int(v) for v in nc), origin=tuple(og),
                    extent=tuple(ex), n_parcels=npar.value, n_steps=nst.value, t=t.value,
                    zeta=(int(z[0]), int(z[1])))

    def write_parcels(self, path, ncells, origin, extent, t, p: dict, zeta=(0, 0)):
        n = len(p["vol"])
        nc, og, ex = self._box(ncells, origin, extent)
        arrs = (_f64(p["pos"], (n, 3)), _f64(p["vor"], (n, 3)), _f64(p["B"], (n, 5)), _f64(p["vol"], (n,)),
                _f64(p["buoy"], (n,)), _f64(p["hum"], (n,)) if p.get("hum") is not None else None)
        z = np.ascontiguousarray(zeta, dtype=np.int32)
        self._check(self.lib.epic_nc_write_parcels(os.fsencode(path), nc.ctypes.data_as(_I32), _ptr(og), _ptr(ex),
                                                   z.ctypes.data_as(_I32), C.c_double(t), C.c_int64(n),
                                                   *[_ptr(a) for a in arrs]), "epic_nc_write_parcels")

    def read_parcels(self, path) -> dict:
        n = self.info(path)["n_parcels"]
        out = dict(pos=np.empty((n, 3)), vor=np.empty((n, 3)), B=np.empty((n, 5)), vol=np.empty(n),
                   buoy=np.empty(n), hum=np.empty(n))
        m = C.c_int64()
        self._check(self.lib.epic_nc_read_parcels(os.fsencode(path), C.c_int64(n), C.byref(m), _ptr(out["pos"]),
                                                  _ptr(out["vor"]), _ptr(out["B"]), _ptr(out["vol"]),
                                                  _ptr(out["buoy"]), _ptr(out["hum"])), "epic_nc_read_parcels")
        return out

    def write_field_file(self, path, ncells, origin, extent, t, fields: dict, units: dict | None = None,
                         zeta=(0, 0)):
        """fields: name -> (nx, ny, nz+3) array (rows 0 .. nz are written)."""
        nc, og, ex = self._box(ncells, origin, extent)
        shape = (int(nc[0]), int(nc[1]), int(nc[2]) + 3)
        names = list(fields)
        arrs = [_f64(fields[k], shape) for k in names]
        cn = (C.c_char_p * len(names))(*[k.encode() for k in names])
        cu = (C.c_char_p * len(names))(*[((units or {}).get(k) or "1").encode() for k in names])
        cd = (_D * len(names))(*[_ptr(a) for a in arrs])
        z = np.ascontiguousarray(zeta, dtype=np.int32)
        self._check(self.lib.epic_nc_write_field_file(os.fsencode(path), nc.ctypes.data_as(_I32), _ptr(og), _ptr(ex),
                                                      z.ctypes.data_as(_I32), C.c_double(t), C.c_int(len(names)),
                                                      cn, cu, cd), "epic_nc_write_field_file")

    def read_variable(self, path, name, record=0) -> np.ndarray:
        """Any numeric variable (one record) as a flat float64 array."""
        n = C.c_int64()
        self._check(self.lib.epic_nc_read_variable(os.fsencode(path), name.encode(), C.c_int64(record), C.c_int64(0),
                                                   C.byref(n), None), "epic_nc_read_variable")
        out = np.empty(n.value)
        self._check(self.lib.epic_nc_read_variable(os.fsencode(path), name.encode(), C.c_int64(record),
                                                   C.c_int64(n.value), C.byref(n), _ptr(out)), "epic_nc_read_variable")
        return out

    def read_field(self, path, name, ncells, origin, extent, step=-1) -> np.ndarray:
        nc, og, ex = self._box(ncells, origin, extent)
        out = np.zeros((int(nc[0]), int(nc[1]), int(nc[2]) + 3))
        self._check(self.lib.epic_nc_read_field(os.fsencode(path), name.encode(), C.c_int64(step),
                                                nc.ctypes.data_as(_I32), _ptr(og), _ptr(ex), _ptr(out)),
                    "epic_nc_read_field")
        return out
