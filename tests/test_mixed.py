"""Mixed-precision form (EPIC_PRECISION_MIXED) against the FP64 oracle and the
plain FP64 GPU path.

The mixed form keeps vorticity, B, buoyancy, humidity, the RK accumulators of
vorticity and B and the support vectors in FP32, accumulates par2grid and
interpolates grid2par in FP32, and keeps positions, volume, delta_pos and the
B33 volume constraint in FP64.  Tolerances are relative to the field or
quantity scale.
"""
import numpy as np
import pytest

from epic_b200 import abi, make_context
from tests.helpers import pair, small_state

pytestmark = pytest.mark.gpu

MIXED = 1
FIELD_TOL = 2e-6      # one par2grid / vor2vel in FP32 against FP64
DRIFT_TOL = 1e-5      # energy / enstrophy after many steps, mixed vs plain


def _rel(a, b):
    scale = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() / scale


def test_mixed_par2grid_vs_oracle(olib, glib):
    s = small_state("thermal")
    oc = make_context(s, olib)
    gc = make_context(s, glib, precision=MIXED)
    oc.par2grid(False)
    gc.par2grid(False)
    for fid in list(abi.VORTG) + [abi.TBUOYG, abi.VOLG]:
        assert _rel(gc.get_field(fid), oc.get_field(fid)) < FIELD_TOL, fid


def test_mixed_rk_step_vs_oracle(olib, glib):
    s = small_state("thermal")
    oc = make_context(s, olib)
    gc = make_context(s, glib, precision=MIXED)
    _, dto = oc.rk_step(0.0)
    _, dtg = gc.rk_step(0.0)
    assert abs(dtg - dto) / dto < 1e-5
    po, pg = oc.get_parcels(), gc.get_parcels()
    assert np.abs(pg["pos"] - po["pos"]).max() < 1e-6 * s.dx.min()
    for key in ("vor", "B"):
        assert _rel(pg[key], po[key]) < 1e-5, key
    for fid in list(abi.VELOG):
        assert _rel(gc.get_field(fid), oc.get_field(fid)) < 1e-5, fid


def test_mixed_store_round_trip(glib):
    """set_parcels / get_parcels of the mixed store: FP64 positions and volume
    come back exactly, FP32 attributes rounded once."""
    s = small_state("beltrami")
    gc = make_context(s, glib, precision=MIXED)
    p = gc.get_parcels()
    assert np.array_equal(p["pos"], s.pos)
    assert np.array_equal(p["vol"], s.vol)
    assert np.array_equal(p["vor"], s.vor.astype(np.float32).astype(np.float64))
    assert np.array_equal(p["B"], s.B.astype(np.float32).astype(np.float64))


@pytest.mark.parametrize("kind,steps,dt", [("thermal", 100, 0.05), ("beltrami", 100, 0.02)])
def test_mixed_drift_vs_plain(glib, kind, steps, dt):
    """Energy and enstrophy of the mixed form track the plain FP64 run of the
    same seed within 1e-5 relative after 100 full steps (merge, split and
    corrections on).  The step is fixed so that both runs compare the same
    times: with the adaptive step the thermal reaches its turbulent phase,
    where any rounding difference, FP64 ones included, grows."""
    s = small_state(kind, small_frac=0.02)
    runs = {}
    for prec in (0, MIXED):
        c = make_context(s, glib, precision=prec, keep_order=0, use_fixed_dt=1, fixed_dt=dt,
                         capacity=4 * s.n)
        t = 0.0
        for _ in range(steps):
            t, info = c.step(t)
        runs[prec] = (info.parcel_stats[1], info.parcel_stats[12], c.get_field(abi.VELOG[2]))
    ke0, en0, w0 = runs[0]
    ke1, en1, w1 = runs[MIXED]
    assert abs(ke1 - ke0) / abs(ke0) < DRIFT_TOL
    assert abs(en1 - en0) / abs(en0) < DRIFT_TOL


def test_mixed_par2grid_box_windows(olib, glib):
    """The mixed form's two-limb fixed-point windows (box-ordered store)
    against the oracle after one full step."""
    s = small_state("thermal", small_frac=0.02, seed=5)
    oc = make_context(s, olib)
    gc = make_context(s, glib, precision=MIXED, keep_order=0)
    oc.step(0.0)
    gc.step(0.0)
    oc.par2grid(False)
    gc.par2grid(False)
    for fid in list(abi.VORTG) + [abi.TBUOYG, abi.VOLG]:
        assert _rel(gc.get_field(fid), oc.get_field(fid)) < 1e-5, fid


@pytest.mark.parametrize("shape,path", [((128, 128, 32), 0), ((128, 128, 32), 1), ((128, 128, 32), 2),
                                        ((64, 64, 64), 1), ((128, 128, 128), 1), ((16, 16, 16), 1),
                                        ((48, 48, 48), 1), ((96, 96, 48), 1), ((96, 96, 48), 2)])
def test_mixed_vor2vel_fft_paths(glib, shape, path):
    """Taylor-Green vorticity (test_mpi_vor2vel.f90) through each horizontal
    FFT path in the mixed form, whose spectral work is FP32: velocity within
    FIELD_TOL of the exact solution's scale."""
    import math
    nx, ny, nz = shape
    lower = (-math.pi, -math.pi, -0.5 * math.pi)
    extent = (2 * math.pi, 2 * math.pi, 2 * math.pi)
    ctx = abi.EpicContext(glib, glib.default_config(nx, ny, nz, lower, extent, precision=MIXED))
    glib.lib.epic_gpu_test_set_fft_path(ctx.h, path)
    dx = np.array(extent) / np.array([nx, ny, nz])
    X, Y, Z = np.meshgrid(lower[0] + np.arange(nx) * dx[0], lower[1] + np.arange(ny) * dx[1],
                          lower[2] + np.arange(-1, nz + 2) * dx[2], indexing="ij")
    ctx.set_field(abi.VORTG[0], -3.0 * np.sin(X) * np.cos(Y) * np.cos(Z))
    ctx.set_field(abi.VORTG[1], 3.0 * np.cos(X) * np.sin(Y) * np.cos(Z))
    ctx.set_field(abi.VORTG[2], 0.0 * X)
    ctx.vor2vel()
    ref = [np.cos(X) * np.sin(Y) * np.sin(Z), np.sin(X) * np.cos(Y) * np.sin(Z), -2.0 * np.sin(X) * np.sin(Y) * np.cos(Z)]
    for i in range(3):
        assert np.abs(ctx.get_field(abi.VELOG[i])[:, :, 1:-1] - ref[i][:, :, 1:-1]).max() < FIELD_TOL * 2.0, i
    ctx.close()
