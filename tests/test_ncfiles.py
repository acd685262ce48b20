"""Parcel and field files in the reference's netCDF layout (include/epic_nc.h).

The library's classic-format writer and reader are checked against an
independent implementation of the format, scipy.io.netcdf_file (CDF-1 and
CDF-2): files the library writes read back in scipy with the reference's
names, dimensions, attributes and values (parcel_netcdf.f90:100-200,
field_netcdf.f90:100-250, netcdf_writer.f90:374-600), and files scipy writes
read in the library.  CDF-5 is checked by a round trip and a hand-built
header.  The GPU cases write and read through a context."""
import math
import os
import struct

import numpy as np
import pytest
from scipy.io import netcdf_file

from epic_b200 import abi
from epic_b200.ncfiles import NcFiles
from tests.conftest import rel_err

BOX = dict(ncells=(8, 6, 4), origin=(-math.pi, -math.pi, 0.0), extent=(2 * math.pi, 2 * math.pi, math.pi))


@pytest.fixture(scope="module")
def nc():
    import epic_b200
    return NcFiles(epic_b200.load())


def _parcels(n, seed=1):
    r = np.random.default_rng(seed)
    return dict(pos=r.normal(size=(n, 3)), vor=r.normal(size=(n, 3)), B=r.normal(size=(n, 5)),
                vol=r.random(n), buoy=r.normal(size=n), hum=r.random(n))


def _fields(seed=2):
    r = np.random.default_rng(seed)
    nx, ny, nz = BOX["ncells"]
    return {k: r.normal(size=(nx, ny, nz + 3)) for k in ("x_vorticity", "y_vorticity", "z_vorticity", "buoyancy")}


def test_parcel_file_layout_in_scipy(nc, tmp_path):
    p = _parcels(257)
    f = str(tmp_path / "run_0000000001_parcels.nc")
    nc.write_parcels(f, t=2.5, p=p, zeta=(1, 0), **BOX)
    assert open(f, "rb").read(4) == b"CDF\x02"
    with netcdf_file(f, "r", mmap=False) as d:
        assert d.file_type == b"parcels"
        assert list(d.ncells) == list(BOX["ncells"])
        assert np.array_equal(d.extent, BOX["extent"]) and np.array_equal(d.origin, BOX["origin"])
        assert d.l_lower_boundry_zeta_zero == b"true" and d.l_upper_boundry_zeta_zero == b"false"
        assert d.dimensions["n_parcels"] == 257 and d.dimensions["world%size"] == 1
        assert d.dimensions["t"] is None and d.variables["t"][:].tolist() == [2.5]
        assert d.variables["t"].axis == b"T" and d.variables["t"].calendar == b"proleptic_gregorian"
        names = {"x_position": ("pos", 0), "y_position": ("pos", 1), "z_position": ("pos", 2),
                 "x_vorticity": ("vor", 0), "y_vorticity": ("vor", 1), "z_vorticity": ("vor", 2),
                 "B11": ("B", 0), "B12": ("B", 1), "B13": ("B", 2), "B22": ("B", 3), "B23": ("B", 4),
                 "volume": ("vol", None), "buoyancy": ("buoy", None), "humidity": ("hum", None)}
        for name, (k, c) in names.items():
            v = d.variables[name]
            assert v.dimensions == ("t", "n_parcels") and v.shape == (1, 257), name
            want = p[k][:, c] if c is not None else p[k]
            assert np.array_equal(v[0], want), name
        assert d.variables["x_position"].units == b"m" and d.variables["B11"].units == b"m^2"
        assert d.variables["volume"].units == b"m^3" and d.variables["x_vorticity"].units == b"1/s"
        assert d.variables["start_index"][:].tolist() == [1]
        assert d.variables["xhi"][:].tolist() == [7] and d.variables["yhi"][:].tolist() == [5]


@pytest.mark.parametrize("version", [2, 5])
def test_parcel_round_trip(nc, tmp_path, monkeypatch, version):
    if version == 5:
        monkeypatch.setenv("EPIC_NC_VERSION", "5")
    p = _parcels(1000, seed=version)
    f = str(tmp_path / "p.nc")
    nc.write_parcels(f, t=0.75, p=p, zeta=(0, 1), **BOX)
    assert open(f, "rb").read(4) == b"CDF" + bytes([version])
    info = nc.info(f)
    assert info["file_type"] == "parcels" and info["n_parcels"] == 1000 and info["n_steps"] == 1
    assert info["t"] == 0.75 and info["zeta"] == (0, 1) and info["ncells"] == BOX["ncells"]
    q = nc.read_parcels(f)
    for k in p:
        assert np.array_equal(q[k], p[k]), k


def test_empty_parcel_file_refused(nc, tmp_path):
    """A fixed dimension of length 0 would be the record dimension of the
    classic format: an empty parcel file is refused."""
    with pytest.raises(abi.EpicError) as e:
        nc.write_parcels(str(tmp_path / "e.nc"), t=0.0, p=_parcels(0), **BOX)
    assert e.value.code == 9


@pytest.mark.parametrize("version", [1, 2])
def test_scipy_parcel_file_reads(nc, tmp_path, version):
    """A parcel file from another writer (as the reference's tools make them),
    without humidity: the absent attribute is zero (parcel_netcdf.f90:600-700)."""
    p = _parcels(50, seed=5)
    f = str(tmp_path / "s.nc")
    with netcdf_file(f, "w", version=version) as d:
        d.file_type = b"parcels"
        d.ncells = np.array(BOX["ncells"], dtype=np.int32)
        d.extent = np.array(BOX["extent"])
        d.origin = np.array(BOX["origin"])
        d.createDimension("t", None)   # scipy wants the record dimension first
        d.createDimension("n_parcels", 50)
        t = d.createVariable("t", "d", ("t",))
        t[0] = 4.0
        for name, (k, c) in {"x_position": ("pos", 0), "y_position": ("pos", 1), "z_position": ("pos", 2),
                             "B11": ("B", 0), "B12": ("B", 1), "B13": ("B", 2), "B22": ("B", 3),
                             "B23": ("B", 4), "volume": ("vol", None), "x_vorticity": ("vor", 0),
                             "y_vorticity": ("vor", 1), "z_vorticity": ("vor", 2),
                             "buoyancy": ("buoy", None)}.items():
            v = d.createVariable(name, "d", ("t", "n_parcels"))
            v[0, :] = p[k][:, c] if c is not None else p[k]
    info = nc.info(f)
    assert info["t"] == 4.0 and info["zeta"] == (-1, -1)
    q = nc.read_parcels(f)
    for k in ("pos", "vor", "B", "vol", "buoy"):
        assert np.array_equal(q[k], p[k]), k
    assert np.array_equal(q["hum"], np.zeros(50))


def test_parcel_file_errors(nc, tmp_path):
    f = str(tmp_path / "bad.nc")
    with netcdf_file(f, "w") as d:   # no B11
        d.file_type = b"parcels"
        d.ncells = np.array(BOX["ncells"], dtype=np.int32)
        d.extent = np.array(BOX["extent"])
        d.origin = np.array(BOX["origin"])
        d.createDimension("n_parcels", 3)
        d.createVariable("volume", "d", ("n_parcels",))[:] = 1.0
    with pytest.raises(abi.EpicError) as e:
        nc.read_parcels(f)
    assert e.value.code == 9 and "B11" in str(e.value)
    h = str(tmp_path / "hdf.nc")
    open(h, "wb").write(b"\x89HDF\r\n\x1a\n" + bytes(100))
    with pytest.raises(abi.EpicError) as e:
        nc.info(h)
    assert e.value.code == 9 and "HDF5" in str(e.value)
    with pytest.raises(abi.EpicError):
        nc.info(str(tmp_path / "missing.nc"))
    g = str(tmp_path / "g.nc")
    nc.write_field_file(g, t=0.0, fields=_fields(), **BOX)
    with pytest.raises(abi.EpicError):   # a field file is not a parcel file
        nc.read_parcels(g)


def test_field_file_layout_in_scipy(nc, tmp_path):
    fl = _fields()
    f = str(tmp_path / "run_fields.nc")
    nc.write_field_file(f, t=1.25, fields=fl, units={"buoyancy": "m/s^2"}, **BOX)
    nx, ny, nz = BOX["ncells"]
    with netcdf_file(f, "r", mmap=False) as d:
        assert d.file_type == b"fields"
        assert d.dimensions["x"] == nx and d.dimensions["y"] == ny and d.dimensions["z"] == nz + 1
        dx = np.array(BOX["extent"]) / np.array(BOX["ncells"])
        assert np.allclose(d.variables["x"][:], BOX["origin"][0] + np.arange(nx) * dx[0], rtol=0, atol=1e-15)
        assert np.allclose(d.variables["z"][:], BOX["origin"][2] + np.arange(nz + 1) * dx[2], rtol=0, atol=1e-15)
        assert d.variables["x"].axis == b"X" and d.variables["z"].axis == b"Z"
        assert d.variables["t"][:].tolist() == [1.25]
        for name, a in fl.items():
            v = d.variables[name]
            assert v.dimensions == ("t", "z", "y", "x")
            # file (z, y, x), x fastest  <->  field layout (x, y, z+1), z fastest
            assert np.array_equal(v[0], np.transpose(a[:, :, 1:-1], (2, 1, 0))), name
        assert d.variables["buoyancy"].units == b"m/s^2"


def test_field_file_reads_scipy_and_own(nc, tmp_path):
    nx, ny, nz = BOX["ncells"]
    fl = _fields(seed=9)
    f = str(tmp_path / "s_fields.nc")
    with netcdf_file(f, "w", version=2) as d:   # two records; the last is read by default
        d.file_type = b"fields"
        d.ncells = np.array(BOX["ncells"], dtype=np.int32)
        d.extent = np.array(BOX["extent"])
        d.origin = np.array(BOX["origin"])
        d.createDimension("t", None)
        for k, n in (("x", nx), ("y", ny), ("z", nz + 1)):
            d.createDimension(k, n)
        d.createVariable("t", "d", ("t",))[:] = [0.0, 3.0]
        v = d.createVariable("buoyancy", "d", ("t", "z", "y", "x"))
        v[0] = 0.0
        v[1] = np.transpose(fl["buoyancy"][:, :, 1:-1], (2, 1, 0))
        w = d.createVariable("humidity", "f", ("t", "z", "y", "x"))   # FP32 converts
        w[1] = np.full((nz + 1, ny, nx), 0.25, dtype=np.float32)
    assert nc.info(f)["n_steps"] == 2 and nc.info(f)["t"] == 3.0
    b = nc.read_field(f, "buoyancy", **BOX)
    assert np.array_equal(b[:, :, 1:-1], fl["buoyancy"][:, :, 1:-1])
    assert np.all(b[:, :, 0] == 0) and np.all(b[:, :, -1] == 0)
    assert np.all(nc.read_field(f, "buoyancy", step=0, **BOX) == 0)
    assert np.all(nc.read_field(f, "humidity", **BOX)[:, :, 1:-1] == 0.25)
    with pytest.raises(abi.EpicError):
        nc.read_field(f, "x_vorticity", **BOX)
    with pytest.raises(abi.EpicError):   # another box
        nc.read_field(f, "buoyancy", ncells=(8, 6, 5), origin=BOX["origin"], extent=BOX["extent"])
    g = str(tmp_path / "own.nc")
    nc.write_field_file(g, t=0.0, fields=fl, **BOX)
    for k in fl:
        assert np.array_equal(nc.read_field(g, k, **BOX)[:, :, 1:-1], fl[k][:, :, 1:-1])


def test_cdf5_header_by_hand(nc, tmp_path):
    """A minimal CDF-5 parcel file assembled from the format description
    (64-bit counts, lengths, sizes and offsets) reads in the library."""
    def u32(v): return struct.pack(">I", v)
    def u64(v): return struct.pack(">Q", v)
    def name(s):
        b = s.encode()
        return u64(len(b)) + b + bytes((-len(b)) % 4)
    def att_text(k, s):
        b = s.encode()
        return name(k) + u32(2) + u64(len(b)) + b + bytes((-len(b)) % 4)
    def att(k, typ, fmt, vals):
        return name(k) + u32(typ) + u64(len(vals)) + struct.pack(">" + fmt * len(vals), *vals)
    n = 3
    vals = {v: np.arange(n) + 10.0 * i for i, v in enumerate(
        ("x_position", "y_position", "z_position", "B11", "B12", "B13", "B22", "B23", "volume", "buoyancy"))}
    gatts = [att_text("file_type", "parcels"), att("ncells", 4, "i", [8, 6, 4]),
             att("extent", 6, "d", list(BOX["extent"])), att("origin", 6, "d", list(BOX["origin"]))]
    head = b"CDF\x05" + u64(0) + u32(10) + u64(1) + name("n_parcels") + u64(n)
    head += u32(12) + u64(len(gatts)) + b"".join(gatts)
    var_hdr_len = lambda v: len(name(v)) + 8 + 8 + 4 + 8 + 4 + 8 + 8
    hlen = len(head) + 4 + 8 + sum(var_hdr_len(v) for v in vals)
    body, vh, off = b"", b"", hlen
    for v, a in vals.items():
        vh += name(v) + u64(1) + u64(0) + u32(0) + u64(0) + u32(6) + u64(8 * n) + u64(off)
        body += struct.pack(">%dd" % n, *a)
        off += 8 * n
    data = head + u32(11) + u64(len(vals)) + vh
    assert len(data) == hlen
    f = tmp_path / "c5.nc"
    f.write_bytes(data + body)
    q = nc.read_parcels(str(f))
    assert np.array_equal(q["pos"][:, 1], vals["y_position"]) and np.array_equal(q["B"][:, 4], vals["B23"])
    assert np.array_equal(q["vol"], vals["volume"]) and np.array_equal(q["vor"], np.zeros((n, 3)))


# ---- through a context (GPU) -------------------------------------------------

@pytest.mark.gpu
def test_context_parcel_file_restart(glib, nc, tmp_path):
    from epic_b200 import initial, make_context_device
    spec = initial.device_spec("thermal-32")
    a = make_context_device(spec, glib, keep_order=0)
    t, _ = a.step(0.0)
    t, _ = a.step(t)
    f = str(tmp_path / "a_parcels.nc")
    a.write_parcels_nc(f, t)
    pa = a.get_parcels()
    q = nc.read_parcels(f)
    for k in pa:
        assert np.array_equal(q[k], pa[k]), k
    b = abi.EpicContext(glib, a.cfg)
    assert b.read_parcels_nc(f) == t
    pb = b.get_parcels()
    for k in pa:
        assert np.array_equal(pb[k], pa[k]), k
    b.init_correction()
    ta, ia = a.step(t)
    tb, ib = b.step(t)
    assert ia.n_parcels == ib.n_parcels
    assert rel_err(np.array(ib.parcel_stats), np.array(ia.parcel_stats)) < 1e-9
    a.close()
    b.close()


@pytest.mark.gpu
def test_context_field_file(glib, nc, tmp_path):
    from epic_b200 import initial, make_context_device
    a = make_context_device(initial.device_spec("thermal-32"), glib, keep_order=0)
    t, _ = a.step(0.0)
    f = str(tmp_path / "a_fields.nc")
    a.write_fields_nc(f, t)
    cfg = a.cfg
    box = dict(ncells=(cfg.nx, cfg.ny, cfg.nz), origin=tuple(cfg.lower), extent=tuple(cfg.extent))
    info = nc.info(f)
    assert info["file_type"] == "fields" and info["t"] == t
    for name, fid in (("x_velocity", abi.VELOG[0]), ("z_vorticity", abi.VORTG[2]), ("buoyancy", abi.TBUOYG),
                      ("volume", abi.VOLG), ("nparg", abi.NPARG)):
        got = nc.read_field(f, name, **box)[:, :, 1:-1]
        assert np.array_equal(got, a.get_field(fid)[:, :, 1:-1]), name
    with pytest.raises(abi.EpicError):   # a field file is not a restart parcel file
        abi.EpicContext(glib, cfg).read_parcels_nc(f)
    a.close()


@pytest.mark.gpu
def test_init_from_field_file_parity(olib, glib, nc, tmp_path):
    """epic_gpu_init_from_field_file on a field file equals the oracle's
    init_from_grids on the same fields (halo rows zero, as after
    read_netcdf_fields)."""
    from tests.test_init_from_grids import BELTRAMI_DOMAIN, _grids
    n = (16, 16, 8)
    lower, extent = BELTRAMI_DOMAIN["lower"], BELTRAMI_DOMAIN["extent"]
    vor, b, h = _grids(n, lower, extent)
    for a in (vor[0], vor[1], vor[2], b, h):
        a[:, :, 0] = 0.0
        a[:, :, -1] = 0.0
    f = str(tmp_path / "init_fields.nc")
    nc.write_field_file(f, ncells=n, origin=lower, extent=extent, t=0.0,
                        fields={"x_vorticity": vor[0], "y_vorticity": vor[1], "z_vorticity": vor[2],
                                "buoyancy": b, "humidity": h})
    cfg_o = olib.default_config(*n, lower, extent)
    cfg_g = glib.default_config(*n, lower, extent)
    oc, gc = abi.EpicContext(olib, cfg_o), abi.EpicContext(glib, cfg_g)
    fo = oc.init_from_grids(vor, b, h)
    fg = gc.init_from_field_file(f)
    assert fo == fg
    po, pg = oc.get_parcels(), gc.get_parcels()
    assert len(po["vol"]) == len(pg["vol"])
    for k in ("pos", "vol", "B"):
        assert rel_err(pg[k], po[k]) < 1e-15, k
    for k in ("vor", "buoy", "hum"):
        assert rel_err(pg[k], po[k]) < 1e-13, k
    bad = abi.EpicContext(glib, glib.default_config(16, 16, 4, lower, extent))
    with pytest.raises(abi.EpicError) as e:   # the file's box is not the context's
        bad.init_from_field_file(f)
    assert e.value.code == 9


def test_corrupt_files_give_errors_not_crashes(nc, tmp_path):
    """Truncated files and random byte changes in the header or the data of
    a valid parcel file and field file: every read returns either data or
    EPIC_ERR_IO (a crash would end the test process).  Seeded."""
    rng = np.random.default_rng(12)
    good_p = str(tmp_path / "good_p.nc")
    nc.write_parcels(good_p, t=1.0, p=_parcels(40), **BOX)
    good_f = str(tmp_path / "good_f.nc")
    nc.write_field_file(good_f, t=0.0, fields=_fields(), **BOX)
    for src in (good_p, good_f):
        raw = bytearray(open(src, "rb").read())
        for trial in range(200):
            b = bytearray(raw)
            kind = trial % 4
            if kind == 0:
                b = b[:int(rng.integers(0, len(b)))]
            else:
                # header bytes (1, 2: all-ones bytes make huge counts) or anywhere (3)
                hi = min(len(b), 600) if kind < 3 else len(b)
                for _ in range(int(rng.integers(1, 6))):
                    b[int(rng.integers(0, hi))] = 0xFF if kind == 2 else int(rng.integers(0, 256))
            f = str(tmp_path / "bad.nc")
            open(f, "wb").write(bytes(b))
            try:
                info = nc.info(f)
            except abi.EpicError as e:
                assert e.code == 9
                continue
            try:
                if info["file_type"] == "parcels" and 0 <= info["n_parcels"] <= 10000:
                    nc.read_parcels(f)
                else:
                    nc.read_field(f, "buoyancy", **BOX)
            except abi.EpicError as e:
                assert e.code in (6, 9)
