"""The start of a run from a field file (utils.f90:223-234): parcel_default,
init_refine, init_parcels_from_grids and set_zeta_boundary_flag.

The oracle is checked against the Python restatement of the same steps
(regular positions and shapes from epic_b200/initial.py, trilinear
interpolation in numpy, zeta flags from initial.zeta_boundary_flags), then the
device against the oracle."""
import math

import numpy as np
import pytest

from epic_b200 import abi, initial
from tests.conftest import rel_err

BELTRAMI_DOMAIN = dict(lower=(-math.pi, -math.pi, -0.5 * math.pi), extent=(2 * math.pi, 2 * math.pi, math.pi))


def _grids(n, lower, extent, zeta_wall=True):
    """Beltrami vorticity (k, l, m) = (1, 1, 1) on the grid (zeta is zero on
    both walls, so both flags are set), a buoyancy and a humidity field; the
    fields are (nx, ny, nz+3) with z = -1 .. nz+1 (halo rows filled too)."""
    nx, ny, nz = n
    dx = np.array(extent) / np.array(n)
    X, Y, Z = np.meshgrid(lower[0] + np.arange(nx) * dx[0], lower[1] + np.arange(ny) * dx[1],
                          lower[2] + np.arange(-1, nz + 2) * dx[2], indexing="ij")
    pts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    vor = initial.beltrami_vorticity(pts, 1, 1, 1).T.reshape(3, nx, ny, nz + 3)
    if not zeta_wall:
        vor[2] += 0.3
    b = (0.5 * np.exp(-(X ** 2 + Y ** 2 + (Z - 0.2) ** 2) / 0.5)).reshape(nx, ny, nz + 3)
    h = (1e-3 * (1 + np.cos(X) * np.sin(2 * Y))).reshape(nx, ny, nz + 3)
    return np.ascontiguousarray(vor), b, h


def _trilinear_np(f, pos, lower, dx, n):
    nx, ny, nz = n
    xyz = (pos - np.array(lower)) / dx
    i0 = np.floor(xyz).astype(int)
    p = xyz - i0
    out = np.zeros(len(pos))
    for di in (0, 1):
        for dj in (0, 1):
            for dk in (0, 1):
                w = (p[:, 0] if di else 1 - p[:, 0]) * (p[:, 1] if dj else 1 - p[:, 1]) * \
                    (p[:, 2] if dk else 1 - p[:, 2])
                out += w * f[(i0[:, 0] + di) % nx, (i0[:, 1] + dj) % ny, i0[:, 2] + dk + 1]
    return out


def _ctx(lib, n, lower, extent, **kw):
    cfg = lib.default_config(*n, lower, extent, **kw)
    return abi.EpicContext(lib, cfg)


@pytest.mark.parametrize("zeta_wall", [True, False])
def test_oracle_init_from_grids(olib, zeta_wall):
    n = (16, 16, 8)
    lower, extent = BELTRAMI_DOMAIN["lower"], BELTRAMI_DOMAIN["extent"]
    vor, b, h = _grids(n, lower, extent, zeta_wall)
    oc = _ctx(olib, n, lower, extent)
    flags = oc.init_from_grids(vor, b, h)
    p = oc.get_parcels()
    pos, vol, B = initial.regular_parcels(*n, lower, extent)
    assert np.array_equal(p["pos"], pos) and np.array_equal(p["vol"], vol) and np.array_equal(p["B"], B)
    dx = np.array(extent) / np.array(n)
    for k in range(3):
        assert rel_err(p["vor"][:, k], _trilinear_np(vor[k], pos, lower, dx, n)) < 1e-13
    assert rel_err(p["buoy"], _trilinear_np(b, pos, lower, dx, n)) < 1e-13
    assert rel_err(p["hum"], _trilinear_np(h, pos, lower, dx, n)) < 1e-13
    assert flags == initial.zeta_boundary_flags(vor[2][:, :, 1:-1])
    assert flags == ((1, 1) if zeta_wall else (0, 0))


def test_oracle_init_refine(olib):
    """Flat cells (dx / dz = 5 >= lambda_max): parcel_default's spheroids are
    split (init_refine) until parcel 1's aspect ratio is below lambda_max."""
    n = (8, 8, 4)
    lower, extent = (0.0, 0.0, 0.0), (8.0, 8.0, 0.8)
    vor, b, h = _grids(n, lower, extent)
    oc = _ctx(olib, n, lower, extent)
    oc.init_from_grids(vor, b, h)
    npar = oc.num_parcels()
    assert npar > 8 * 8 * 8 * 4 and npar % (8 * 8 * 4 * 8) == 0
    p = oc.get_parcels()
    assert np.isclose(p["vol"].sum(), 8.0 * 8.0 * 0.8, rtol=1e-13)


def test_oracle_init_n_per_cell_not_a_cube(olib):
    """int(64 ** (1/3)) is 3 in FP64, so the reference refuses 64 per cell
    (parcel_init.f90:113-121) as it refuses 10."""
    for npc in (10, 64):
        oc = _ctx(olib, (8, 8, 8), (0, 0, 0), (1, 1, 1), n_per_cell=npc)
        with pytest.raises(abi.EpicError) as e:
            oc.init_from_grids(*_grids((8, 8, 8), (0, 0, 0), (1, 1, 1)))
        assert e.value.code == 1


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["beltrami", "refine"])
def test_init_from_grids_parity(olib, glib, case):
    if case == "beltrami":
        n, lower, extent = (16, 16, 8), BELTRAMI_DOMAIN["lower"], BELTRAMI_DOMAIN["extent"]
    else:
        n, lower, extent = (8, 8, 4), (0.0, 0.0, 0.0), (8.0, 8.0, 0.8)
    vor, b, h = _grids(n, lower, extent)
    oc, gc = _ctx(olib, n, lower, extent), _ctx(glib, n, lower, extent)
    fo = oc.init_from_grids(vor, b, h)
    fg = gc.init_from_grids(vor, b, h)
    assert fo == fg
    a, r = gc.get_parcels(), oc.get_parcels()
    assert len(a["vol"]) == len(r["vol"])
    for k in ("pos", "vol", "B"):
        assert rel_err(a[k], r[k]) < 1e-15, k
    for k in ("vor", "buoy", "hum"):
        assert rel_err(a[k], r[k]) < 1e-13, k
    # and the run from there
    oc.init_correction()
    gc.init_correction()
    to = tg = 0.0
    for _ in range(2):
        to, io = oc.step(to)
        tg, ig = gc.step(tg)
        assert io.n_parcels == ig.n_parcels
        assert rel_err(np.array(ig.parcel_stats), np.array(io.parcel_stats)) < 1e-9
