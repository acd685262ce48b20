"""Synthetic initial states of the benchmark configurations.

Parcels are placed like the reference's ``init_regular_positions``
(parcel_init.f90:108-152): cell by cell with z outermost, n_per_dim^3
parcels per cell at the sub-cell centres, loop order k, j, i inside a cell.
Shapes follow ``parcel_default`` (parcel_init.f90:31-100): for isotropic
cells B11 = B22 = (abc)^(2/3), other entries 0, i.e. spheres of volume
Vcell / n_per_cell.

Random perturbations use a counter-based generator (SplitMix64 keyed by
seed, parcel index and component) so that any two programs produce
bit-identical inputs from the same seed.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

_GOLD = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(x: np.ndarray) -> np.ndarray:
    x = (x + _GOLD).astype(np.uint64)
    z = x
    z = (z ^ (z >> np.uint64(30))) * _M1
    z = (z ^ (z >> np.uint64(27))) * _M2
    return z ^ (z >> np.uint64(31))


def uniform(seed: int, index: np.ndarray, comp: int) -> np.ndarray:
    """U[0, 1) keyed by (seed, parcel index, component)."""
    with np.errstate(over="ignore"):
        key = (np.uint64(seed) * _GOLD) ^ (index.astype(np.uint64) * np.uint64(16) + np.uint64(comp))
        r = splitmix64(splitmix64(key))
    return (r >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


@dataclass
class Setup:
    """Grid, options and parcel arrays of one run (Fortran (c, n) layouts as (n, c))."""
    name: str
    nx: int
    ny: int
    nz: int
    lower: tuple
    extent: tuple
    options: dict = field(default_factory=dict)
    pos: np.ndarray = None
    vor: np.ndarray = None
    B: np.ndarray = None
    vol: np.ndarray = None
    buoy: np.ndarray = None
    hum: np.ndarray = None
    steps: int = 1

    @property
    def n(self) -> int:
        return len(self.vol)

    @property
    def dx(self):
        return np.array(self.extent) / np.array([self.nx, self.ny, self.nz])

    def arrays(self):
        return (self.pos, self.vor, self.B, self.vol, self.buoy, self.hum)


def regular_parcels(nx, ny, nz, lower, extent, n_per_cell=8, shape="reference"):
    """Positions, volumes and B of init_regular_positions / parcel_default.

    shape="reference" uses parcel_default's aspect ratio lam = max cell
    spacing ratio (spheroids B11 = B22 = (lam abc)^(2/3)); shape="sphere"
    forces lam = 1 (spheres of volume Vcell / n_per_cell)."""
    npd = round(n_per_cell ** (1.0 / 3.0))
    if npd ** 3 != n_per_cell:
        raise ValueError("n_per_cell must be a cube")
    dx = np.array(extent, dtype=np.float64) / np.array([nx, ny, nz], dtype=np.float64)
    im = 1.0 / npd
    iz, iy, ix, k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), np.arange(1, npd + 1),
                                      np.arange(1, npd + 1), np.arange(1, npd + 1), indexing="ij")
    corner = [lower[0] + ix * dx[0], lower[1] + iy * dx[1], lower[2] + iz * dx[2]]
    x = corner[0] + dx[0] * (i - 0.5) * im
    y = corner[1] + dx[1] * (j - 0.5) * im
    z = corner[2] + dx[2] * (k - 0.5) * im
    pos = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    n = len(pos)
    vcell = dx[0] * dx[1] * dx[2]
    vol = np.full(n, vcell / n_per_cell)
    lam = max(dx[0] / dx[1], dx[1] / dx[0], dx[0] / dx[2], dx[2] / dx[0], dx[1] / dx[2], dx[2] / dx[1])
    if shape == "sphere":
        lam = 1.0
    abc = 0.75 * vol * (1.0 / math.pi)
    l23 = (lam * abc) ** (2.0 / 3.0)
    B = np.zeros((n, 5))
    B[:, 0] = l23
    B[:, 3] = l23
    return pos, vol, B


def zeta_boundary_flags(zeta_grid: np.ndarray, zeta_tol: float = float(np.float32(1.0e-3))):
    """set_zeta_boundary_flag (parameters.f90:168-217) for a gridded zeta (nx, ny, nz+1)."""
    nx, ny, nzp = zeta_grid.shape
    nz = nzp - 1
    nhcelli = 1.0 / (nx * ny)
    val_i = np.sum(zeta_grid[:, :, 1:nz] ** 2)
    val_b = np.array([np.sum(zeta_grid[:, :, 0] ** 2), np.sum(zeta_grid[:, :, nz] ** 2)])
    rms_i = math.sqrt(val_i * nhcelli / (nz - 1))
    rms_b = np.sqrt(val_b * nhcelli)
    thres = zeta_tol * rms_i + np.finfo(np.float64).eps
    return (int(rms_b[0] < thres), int(rms_b[1] < thres))


def beltrami_vorticity(pos, k=1, l=1, m=1):
    """get_flow_vorticity (models/3d/beltrami_3d.f90:103-122)."""
    kk, ll, mm = float(k), float(l), float(m)
    alpha = math.sqrt(kk ** 2 + ll ** 2 + mm ** 2)
    fk2l2 = alpha / float(k ** 2 + l ** 2)
    x, y, z = pos[:, 0], pos[:, 1], pos[:, 2]
    cosmz, sinmz = np.cos(mm * z), np.sin(mm * z)
    s, c = np.sin(kk * x + ll * y), np.cos(kk * x + ll * y)
    return np.stack([fk2l2 * (kk * mm * sinmz - ll * alpha * cosmz) * s,
                     fk2l2 * (ll * mm * sinmz + kk * alpha * cosmz) * s,
                     alpha * cosmz * c], axis=1)


def beltrami(n=32, k=1, l=1, m=1, n_per_cell=8, steps=50) -> Setup:
    """Beltrami flow: domain 2pi x 2pi x pi, n^3 grid, spheres of volume
    Vcell / n_per_cell, omega = u (Beltrami modes k, l, m)."""
    lower = (-math.pi, -math.pi, -0.5 * math.pi)
    extent = (2 * math.pi, 2 * math.pi, math.pi)
    pos, vol, B = regular_parcels(n, n, n, lower, extent, n_per_cell, shape="sphere")
    vor = beltrami_vorticity(pos, k, l, m)
    dx = np.array(extent) / n
    gx = lower[0] + np.arange(n) * dx[0]
    gy = lower[1] + np.arange(n) * dx[1]
    gz = lower[2] + np.arange(n + 1) * dx[2]
    X, Y, Z = np.meshgrid(gx, gy, gz, indexing="ij")
    zg = beltrami_vorticity(np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1), k, l, m)[:, 2].reshape(X.shape)
    flags = zeta_boundary_flags(zg)
    s = Setup("beltrami", n, n, n, lower, extent,
              options=dict(min_vratio=40.0, lambda_max=4.0, bndry_zeta_zero=flags),
              pos=pos, vor=vor, B=B, vol=vol, buoy=np.zeros(len(vol)), hum=np.zeros(len(vol)), steps=steps)
    return s


def thermal(nx=128, ny=None, nz=None, extent=(6.28, 6.28, 6.28), seed=1234, n_per_cell=8,
            bubbles=((0.0, 0.0, 1.5, 0.5),), steps=200, name="thermal") -> Setup:
    """Rising thermal: Gaussian buoyancy b = a exp(-r^2 / 0.5^2) plus seeded
    U(-1e-3, 1e-3) noise on b and U(-0.1 dx, 0.1 dx) on each position
    component (z kept inside the domain); zero vorticity and humidity."""
    ny = ny or nx
    nz = nz or nx
    lower = (-0.5 * extent[0], -0.5 * extent[1], 0.0)
    pos, vol, B = regular_parcels(nx, ny, nz, lower, extent, n_per_cell)
    n = len(vol)
    idx = np.arange(n, dtype=np.uint64)
    dx = np.array(extent) / np.array([nx, ny, nz])
    for c in range(3):
        pos[:, c] += (2.0 * uniform(seed, idx, c) - 1.0) * 0.1 * dx[c]
    upper = lower[2] + extent[2]
    pos[:, 2] = np.clip(pos[:, 2], lower[2], np.nextafter(upper, lower[2]))
    b = np.zeros(n)
    for (cx, cy, cz, amp) in bubbles:
        r2 = (pos[:, 0] - cx) ** 2 + (pos[:, 1] - cy) ** 2 + (pos[:, 2] - cz) ** 2
        b += amp * np.exp(-r2 / 0.25)
    b += (2.0 * uniform(seed, idx, 3) - 1.0) * 1.0e-3
    return Setup(name, nx, ny, nz, lower, extent,
                 options=dict(min_vratio=40.0, lambda_max=4.0, bndry_zeta_zero=(1, 1)),
                 pos=pos, vor=np.zeros((n, 3)), B=B, vol=vol, buoy=b, hum=np.zeros(n), steps=steps)


def config(name: str, **kw) -> Setup:
    """Named workloads: 'beltrami-32' (32^3, 262,144 parcels), 'thermal-128'
    (128^3, 16.8M parcels), 'thermal-256x256x128' (domain 6.28 x 6.28 x 3.14,
    67.1M parcels: the mixed-precision workload) plus small test variants."""
    if name == "beltrami-32":
        return beltrami(32, **kw)
    if name == "thermal-128":
        return thermal(128, **kw)
    if name == "thermal-256x256x128":
        return thermal(256, 256, 128, extent=(6.28, 6.28, 3.14), steps=100, name=name, **kw)
    if name.startswith("beltrami-"):
        return beltrami(int(name.split("-")[1]), **kw)
    if name.startswith("thermal-"):
        return thermal(int(name.split("-")[1]), **kw)
    raise KeyError(name)


@dataclass
class DeviceSpec:
    """A workload whose parcels are generated on the device (epic_gpu_init_state):
    grid, domain, options and the generator's parameters, no host arrays."""
    name: str
    nx: int
    ny: int
    nz: int
    lower: tuple
    extent: tuple
    options: dict
    kind: str                 # "thermal" or "beltrami"
    seed: int = 1234
    bubbles: tuple = ((0.0, 0.0, 1.5, 0.5),)
    klm: tuple = (1, 1, 1)
    n_per_cell: int = 8
    steps: int = 1

    @property
    def n(self) -> int:
        return self.nx * self.ny * self.nz * self.n_per_cell

    @property
    def dx(self):
        return np.array(self.extent) / np.array([self.nx, self.ny, self.nz])

    def init_spec(self):
        from . import abi
        if self.kind == "thermal":
            return abi.init_spec(abi.INIT_THERMAL, self.n_per_cell, self.seed, bubbles=self.bubbles)
        return abi.init_spec(abi.INIT_BELTRAMI, self.n_per_cell, klm=self.klm)


def device_spec(name: str) -> DeviceSpec:
    """Device-generated versions of the named workloads, plus
    'thermal2-512x512x256': two Gaussian thermals (b = 0.5 and 0.3 at
    x = -0.75 and +0.75, z = 1.5) on 512x512x256 cells of 6.28 x 6.28 x 3.14,
    536,870,912 parcels (the large mixed-precision run)."""
    def thermal_spec(nx, ny, nz, extent, bubbles, steps):
        lower = (-0.5 * extent[0], -0.5 * extent[1], 0.0)
        return DeviceSpec(name, nx, ny, nz, lower, extent,
                          dict(min_vratio=40.0, lambda_max=4.0, bndry_zeta_zero=(1, 1)),
                          "thermal", bubbles=bubbles, steps=steps)
    if name == "thermal2-512x512x256":
        return thermal_spec(512, 512, 256, (6.28, 6.28, 3.14), ((-0.75, 0.0, 1.5, 0.5), (0.75, 0.0, 1.5, 0.3)), 50)
    if name == "thermal-256x256x128":
        return thermal_spec(256, 256, 128, (6.28, 6.28, 3.14), ((0.0, 0.0, 1.5, 0.5),), 100)
    if name.startswith("thermal-"):
        n = int(name.split("-")[1])
        return thermal_spec(n, n, n, (6.28, 6.28, 6.28), ((0.0, 0.0, 1.5, 0.5),), 200)
    if name.startswith("beltrami-"):
        n = int(name.split("-")[1])
        lower = (-math.pi, -math.pi, -0.5 * math.pi)
        extent = (2 * math.pi, 2 * math.pi, math.pi)
        from .serve import beltrami_zeta_flags
        return DeviceSpec(name, n, n, n, lower, extent,
                          dict(min_vratio=40.0, lambda_max=4.0, bndry_zeta_zero=beltrami_zeta_flags((n, n, n), (1, 1, 1))),
                          "beltrami", steps=50)
    raise KeyError(name)
