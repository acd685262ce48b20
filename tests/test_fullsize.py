"""Size-independent properties at the benchmark sizes, where the oracle would
take too long: the rising thermal on 128^3 (16,777,216 parcels, plain FP64)
and on 256x256x128 (67,108,864 parcels, mixed form).

* par2grid conserves the parcel moments: the trapezoid sum over z of the
  gridded volume equals the parcels' total volume, and of vortg * volg and
  tbuoyg * volg their volume-weighted vorticity and buoyancy (the z folds of
  parcel_interpl.f90:256-275 double the boundary rows and move the halo rows
  inward, which the trapezoid weights undo);
* the total parcel volume is invariant under a full step (merge and split
  conserve it, parcel_merge.f90:47-108, parcel_split.f90:37-198);
* vor2vel is linear: doubling the vorticity doubles the velocity exactly
  (every operation is linear and scaling by 2 commutes with rounding), and
  the velocity of a sum is the sum of the velocities to rounding."""
import numpy as np
import pytest

from epic_b200 import abi, initial, make_context_device
from tests.conftest import rel_err

pytestmark = pytest.mark.gpu


def _trap(f):
    """Trapezoid sum over z = 0 .. nz of a (nx, ny, nz+3) field."""
    g = f[:, :, 1:-1]
    return g[:, :, 1:-1].sum() + 0.5 * (g[:, :, 0].sum() + g[:, :, -1].sum())


@pytest.fixture(scope="module")
def thermal128(glib):
    ctx = make_context_device(initial.device_spec("thermal-128"), glib, keep_order=0)
    t, _ = ctx.step(0.0)
    yield ctx, t
    ctx.close()


def test_par2grid_moments_128(thermal128):
    ctx, _ = thermal128
    ctx.par2grid(False)
    p = ctx.get_parcels()
    vol = p["vol"]
    volg = ctx.get_field(abi.VOLG)
    assert rel_err(_trap(volg), vol.sum()) < 1e-12
    for c in (0, 1):   # the z component is zeroed on walls with the zeta flag set
        m = (vol * p["vor"][:, c]).sum()
        scale = (vol * np.abs(p["vor"][:, c])).sum()
        assert abs(_trap(ctx.get_field(abi.VORTG[c]) * volg) - m) < 1e-11 * scale
    mb = (vol * p["buoy"]).sum()   # humidity is zero: the total buoyancy is the buoyancy
    assert abs(_trap(ctx.get_field(abi.TBUOYG) * volg) - mb) < 1e-11 * (vol * np.abs(p["buoy"])).sum()


def test_volume_invariant_over_steps_128(thermal128):
    ctx, t = thermal128
    totals = []
    for _ in range(3):
        t, info = ctx.step(t)
        totals.append(info.parcel_stats[4] * info.parcel_stats[11])   # mean volume x parcels
    vdomain = 6.28 ** 3
    for v in totals:
        assert abs(v - vdomain) < 1e-9 * vdomain
    assert max(totals) - min(totals) < 1e-12 * vdomain


def test_vor2vel_linear_128(thermal128):
    ctx, _ = thermal128
    rng = np.random.default_rng(3)
    shape = ctx.field_shape
    w1 = [rng.normal(size=shape) for _ in range(3)]
    w2 = [rng.normal(size=shape) for _ in range(3)]

    def vel(w):
        for c in range(3):
            ctx.set_field(abi.VORTG[c], w[c])
        ctx.vor2vel()
        return np.stack([ctx.get_field(abi.VELOG[c])[:, :, 1:-1] for c in range(3)])

    u1 = vel(w1)
    u2 = vel(w2)
    assert np.array_equal(vel([2.0 * w for w in w1]), 2.0 * u1)
    u12 = vel([a + b for a, b in zip(w1, w2)])
    assert rel_err(u12, u1 + u2) < 1e-12


def test_mixed_256x256x128_steps(glib):
    ctx = make_context_device(initial.device_spec("thermal-256x256x128"), glib, precision=1, keep_order=0)
    t = 0.0
    totals, n = [], []
    for _ in range(3):
        t, info = ctx.step(t)
        totals.append(info.parcel_stats[4] * info.parcel_stats[11])
        n.append(info.n_parcels)
        assert np.isfinite(info.parcel_stats[1]) and info.dt > 0
    vdomain = 6.28 * 6.28 * 3.14
    for v in totals:
        assert abs(v - vdomain) < 1e-9 * vdomain   # volumes stay FP64 in the mixed form
    assert n[0] >= 256 * 256 * 128 * 8
    ctx.close()
