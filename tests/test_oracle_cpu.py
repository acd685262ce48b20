"""The oracle against the reference's own known answers (CPU only).

Golden vectors: unit-tests/3d/{B,D,V}.asc (tests/golden/scherzinger_BDV.npz).
Analytic KATs restated from unit-tests/3d: test_scherzinger_2, test_mpi_vor2vel,
test_mpi_trilinear, test_mpi_grid2par, test_mpi_nearest_1..4,
test_mpi_laplace_correction_3d; the transforms against numpy."""
import math
import os

import numpy as np
import pytest

import oracle
from epic_b200 import abi, initial, make_context

F32 = lambda x: float(np.float32(x))  # noqa: E731  Fortran single-precision literal


def test_scherzinger_golden(olib):
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "scherzinger_BDV.npz"))
    D, V = oracle.eigen(olib, g["B"])
    err = 0.0
    for n in range(len(D)):
        e = np.abs(g["D"][n] - D[n]).sum()
        Q = g["V"][n].reshape(3, 3)
        for k in range(3):
            q = Q[k].copy()
            if q[0] / V[n][0, k] < 0:
                q = -q
            e = max(e, np.abs(q - V[n][:, k]).sum())
        err = max(err, e)
    assert err < 1e-12          # test_scherzinger_2.f90:47
    Dv, _ = oracle.eigen(olib, g["B"], values_only=True)
    assert np.abs(Dv - g["D"]).max() < 1e-12


@pytest.mark.parametrize("n", [8, 16, 48, 64, 96, 128])
def test_transforms(olib, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal((3, n))
    y = oracle.transform(olib, "forfft", x)
    X = np.fft.fft(x, axis=1) / np.sqrt(n)
    ref = np.zeros_like(x)
    for k in range(0, n // 2 + 1):
        ref[:, k] = X[:, k].real
    for k in range(1, (n + 1) // 2):
        ref[:, n - k] = X[:, k].imag
    assert np.abs(y - ref).max() < 1e-13
    assert np.abs(oracle.transform(olib, "revfft", y) - x).max() < 1e-13
    xs = rng.standard_normal((2, n)); xs[:, -1] = 0
    j = np.arange(1, n)
    S = np.sqrt(2 / n) * np.sin(np.pi * np.outer(j, j) / n)
    assert np.abs(oracle.transform(olib, "dst", xs)[:, :n - 1] - xs[:, :n - 1] @ S.T).max() < 1e-12
    xc = rng.standard_normal((2, n + 1))
    jj = np.arange(n + 1); w = np.ones(n + 1); w[0] = w[-1] = 0.5
    Cm = np.sqrt(2 / n) * np.cos(np.pi * np.outer(jj, jj) / n) * w[None, :]
    yc = oracle.transform(olib, "dct", xc)
    assert np.abs(yc - xc @ Cm.T).max() < 1e-12
    assert np.abs(oracle.transform(olib, "dct", yc) - xc).max() < 1e-12   # self-inverse


def test_vor2vel_taylor_green(olib):
    """test_mpi_vor2vel.f90: 64^3, max err < 1e-14."""
    nx = ny = nz = 64
    lower = (-math.pi, -math.pi, -0.5 * math.pi)
    extent = (2 * math.pi,) * 3
    ctx = abi.EpicContext(olib, olib.default_config(nx, ny, nz, lower, extent))
    dx = np.array(extent) / 64
    X, Y, Z = np.meshgrid(lower[0] + np.arange(nx) * dx[0], lower[1] + np.arange(ny) * dx[1],
                          lower[2] + np.arange(-1, nz + 2) * dx[2], indexing="ij")
    ctx.set_field(abi.VORTG[0], -3.0 * np.sin(X) * np.cos(Y) * np.cos(Z))
    ctx.set_field(abi.VORTG[1], 3.0 * np.cos(X) * np.sin(Y) * np.cos(Z))
    ctx.set_field(abi.VORTG[2], 0.0 * X)
    ctx.vor2vel()
    ref = [np.cos(X) * np.sin(Y) * np.sin(Z), np.sin(X) * np.cos(Y) * np.sin(Z), -2 * np.sin(X) * np.sin(Y) * np.cos(Z)]
    err = max(np.abs(ctx.get_field(abi.VELOG[i])[:, :, 1:-1] - ref[i][:, :, 1:-1]).max() for i in range(3))
    assert err < 1e-14


def test_trilinear_conservation(olib):
    """test_mpi_trilinear.f90: 32^3, 27 parcels per cell, constant vorticity."""
    n = 32
    lower = (-1.5, -1.5, -1.5)
    extent = (0.4, 0.4, 0.4)
    pos, vol, B = initial.regular_parcels(n, n, n, lower, extent, 27)
    cfg = olib.default_config(n, n, n, lower, extent, min_vratio=27.0, n_per_cell=27)
    ctx = abi.EpicContext(olib, cfg)
    vor = np.zeros((len(vol), 3)); vor[:, 0] = 1.5
    ctx.set_parcels(pos, vor, B, vol, np.zeros(len(vol)))
    ctx.par2grid(False)
    ngrid = n * n * (n + 1)
    vcell = np.prod(np.array(extent) / n)
    sx = ctx.get_field(abi.VORTG[0])[:, :, 1:-1].sum()
    sv = ctx.get_field(abi.VOLG)[:, :, 1:-1].sum()
    assert abs(sx - 1.5 * ngrid) < 1e-10          # reference bound 1e-15 with its order
    assert abs(sv - ngrid * vcell) < 3e-14


def test_grid2par_constant_fields(olib):
    """test_mpi_grid2par.f90: constant fields interpolate to the constant."""
    s = initial.thermal(16, seed=1)
    ctx = make_context(s, olib)
    vals = {}
    for k, fid in enumerate(list(abi.VELOG) + list(abi.VELGRADG) + list(abi.VTEND)):
        vals[fid] = 0.5 + k
        ctx.set_field(fid, np.full(ctx.field_shape, vals[fid]))
    ctx.grid2par(False)
    rk = ctx.get_parcel_rk()
    for c in range(3):
        assert np.abs(rk["delta_pos"][:, c] - vals[abi.VELOG[c]]).max() < 1e-14
        assert np.abs(rk["delta_vor"][:, c] - vals[abi.VTEND[c]]).max() < 1e-14
    for c in range(8):
        assert np.abs(rk["strain"][:, c] - vals[abi.VELGRADG[c]]).max() < 1e-13


def _nearest_case(olib, placement):
    """A 10^3 unit box with one z layer of cells (test_mpi_nearest_*); works
    with any library binding (oracle or CUDA)."""
    nx = 10
    dx = 0.1
    vcell = dx ** 3
    vmin = vcell / 8.0
    pos, vol = [], []
    for j in range(nx):
        for i in range(nx):
            for (px, py, v) in placement(i, j, dx):
                pos.append((px, py, 1.5 * dx)); vol.append(v * vmin)
    pos = np.array(pos); vol = np.array(vol)
    r2 = (0.75 * vol / math.pi) ** (2.0 / 3.0)
    B = np.zeros((len(vol), 5)); B[:, 0] = r2; B[:, 3] = r2
    cfg = olib.default_config(nx, nx, nx, (0, 0, 0), (1, 1, 1), lambda_max=5.0, min_vratio=8.0)
    ctx = abi.EpicContext(olib, cfg)
    ctx.set_parcels(pos, np.zeros((len(vol), 3)), B, vol, np.arange(len(vol), dtype=float))
    return ctx, len(vol)


def _p1(i, j, dx):   # test_mpi_nearest_1.f90:113-153 (a = b)
    x, y = (0.5 + i) * dx, (0.5 + j) * dx
    out = [(x, y, 1.1)]
    out += [(x + m * dx * F32(0.45), y, 0.9) for m in (-1, 1)]
    out += [(x, y + m * dx * F32(0.45), 0.9) for m in (-1, 1)]
    return out


def _p2(i, j, dx):   # test_mpi_nearest_2.f90:112-153 ((2) a = b)
    x, y = (0.5 + i) * dx, (0.5 + j) * dx
    out = [(x, y, 1.1)]
    out += [(x + m * dx * F32(0.44), y + dx * F32(0.44), 0.9) for m in (-1, 1)]
    out += [(x + m * dx * F32(0.44), y - dx * F32(0.44), 0.9) for m in (-1, 1)]
    return out


def _p3(i, j, dx):   # test_mpi_nearest_3.f90:95-135 (a - B)
    x, y = (0.5 + i) * dx, (0.500001 + j) * dx
    return [(x + 0.1 * dx, y, 1.1), (x + dx * 0.35, y, 0.9), (x - 0.42 * dx, y, 1.1)]


def _p4(i, j, dx):   # test_mpi_nearest_4.f90:95-135 ((2) a - B)
    x, y = (0.500001 + i) * dx, (0.5 + j) * dx
    return [(x, y + 0.1 * dx, 1.1), (x, y + dx * 0.35, 0.9), (x, y - 0.42 * dx, 1.1)]


def _load_kats():
    import json
    with open(os.path.join(os.path.dirname(__file__), "golden", "nearest_kats.json")) as f:
        return json.load(f)


NEAREST_KATS = [(name, c["setup"], c["expected"], c["cell"]) for name, t in sorted(_load_kats().items())
                for c in t["cases"]]


def kat_placement(cell):
    """The constellation of one cell of a test_mpi_nearest_5.._20 case: each
    parcel at the cell centre (x, y) moved by sign x (cell width x factor)
    along x and y, in the reference's evaluation order x + dx(k) * c."""
    def place(i, j, dx):
        x, y = (0.5 + i) * dx, (0.5 + j) * dx
        out = []
        for p in cell:
            q = []
            for base, (sgn, _axis, fac) in zip((x, y), p["off"]):
                q.append(base + dx * fac if sgn > 0 else base - dx * fac if sgn < 0 else base)
            out.append((q[0], q[1], p["vol"]))
        return out
    return place


@pytest.mark.parametrize("name,setup,expected,cell", NEAREST_KATS,
                         ids=[f"{n[9:]}-{s}" for n, s, _, _ in NEAREST_KATS])
def test_nearest_reference_kats(olib, name, setup, expected, cell):
    """unit-tests/3d/test_mpi_nearest_5.f90 .. _20.f90 (fixture made from
    them by tests/golden/make_nearest_kats.py): chains of small and big
    parcels across the periodic edges (a = b - c, a - b - C, a - B - c,
    a - b = c - d, a - b - c = d, ...); the number of merges equals the count
    each test states, and no parcel is lost."""
    ctx, n0 = _nearest_case(olib, kat_placement(cell))
    nm = ctx.merge()
    assert nm == expected
    assert ctx.num_parcels() == n0 - nm


@pytest.mark.parametrize("placement,expected", [(_p1, 200), (_p2, 200), (_p3, 100), (_p4, 100)])
def test_nearest_constellations(olib, placement, expected):
    ctx, n0 = _nearest_case(olib, placement)
    nm = ctx.merge()
    assert nm == expected
    assert ctx.num_parcels() == n0 - nm


def test_laplace_correction_reduces_volume_error(olib):
    """test_mpi_laplace_correction_3d.f90: the volume error decreases."""
    s = initial.thermal(16, seed=9)
    rng = np.random.default_rng(9)
    s.pos = s.pos + rng.uniform(-0.25, 0.25, s.pos.shape) * s.dx[None, :]
    s.pos[:, 2] = np.clip(s.pos[:, 2], 1e-6, s.extent[2] - 1e-6)
    ctx = make_context(s, olib)
    errs = []
    for it in range(6):
        ctx.vol2grid(False)
        v = ctx.get_field(abi.VOLG)[:, :, 1:-1]
        errs.append(np.abs(v / np.prod(s.dx) - 1).max())
        ctx.apply_laplace(False)
        ctx.apply_gradient(True)
    assert errs[-1] < errs[0]
    assert all(b <= a * 1.05 for a, b in zip(errs, errs[1:]))


@pytest.mark.parametrize("kind", ["thermal", "beltrami"])
def test_oracle_init_state_matches_generator(olib, kind):
    """epic_oracle_init_state builds the same parcels as epic_b200/initial.py
    (same arithmetic, same counter RNG): positions, shapes and volumes bit for
    bit; buoyancy and vorticity to the last bit of exp/sin/cos (numpy's
    vectorised exp is not glibc's)."""
    from epic_b200 import abi
    if kind == "thermal":
        bubbles = ((0.0, 0.0, 1.5, 0.5), (-0.75, 0.3, 2.0, 0.3))
        s = initial.thermal(8, 8, 6, seed=11, bubbles=bubbles)
        spec = abi.init_spec(abi.INIT_THERMAL, seed=11, bubbles=bubbles)
    else:
        s = initial.beltrami(8, 2, 1, 2)
        spec = abi.init_spec(abi.INIT_BELTRAMI, klm=(2, 1, 2))
    cfg = olib.default_config(s.nx, s.ny, s.nz, s.lower, s.extent, **s.options)
    ctx = abi.EpicContext(olib, cfg)
    ctx.init_state(spec)
    p = ctx.get_parcels()
    for key in ("pos", "B", "vol", "hum"):
        assert np.array_equal(p[key], getattr(s, key).reshape(p[key].shape)), key
    for key in ("buoy", "vor"):
        np.testing.assert_allclose(p[key], getattr(s, key).reshape(p[key].shape), rtol=4e-16, atol=1e-18)
