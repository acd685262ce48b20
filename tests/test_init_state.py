"""Device-side initial states (epic_gpu_init_state) against the Python
generators of the same workloads (epic_b200/initial.py): positions, volumes
and shapes bit for bit, buoyancy and vorticity to the last bits of exp, sin
and cos."""
import numpy as np
import pytest

from epic_b200 import abi, initial, make_context

pytestmark = pytest.mark.gpu


def _ctx_from_spec(glib, setup, spec):
    cfg = glib.default_config(setup.nx, setup.ny, setup.nz, setup.lower, setup.extent, **setup.options)
    ctx = abi.EpicContext(glib, cfg)
    ctx.init_state(spec)
    return ctx


def _check(ctx, s):
    p = ctx.get_parcels()
    assert len(p["vol"]) == s.n
    assert np.array_equal(p["pos"], s.pos)
    assert np.array_equal(p["vol"], s.vol)
    assert np.array_equal(p["B"], s.B)
    np.testing.assert_allclose(p["buoy"], s.buoy, rtol=4e-16, atol=1e-18)
    np.testing.assert_allclose(p["vor"], s.vor, rtol=4e-16, atol=4e-16)
    assert np.array_equal(p["hum"], s.hum)


@pytest.mark.parametrize("shape,seed", [((16, 16, 16), 7), ((32, 16, 8), 99)])
def test_init_thermal(glib, shape, seed):
    nx, ny, nz = shape
    bubbles = ((0.0, 0.0, 1.5, 0.5), (-0.75, 0.3, 2.0, 0.3))
    s = initial.thermal(nx, ny, nz, seed=seed, bubbles=bubbles)
    ctx = _ctx_from_spec(glib, s, abi.init_spec(abi.INIT_THERMAL, seed=seed, bubbles=bubbles))
    _check(ctx, s)


@pytest.mark.parametrize("klm", [(1, 1, 1), (2, 1, 2)])
def test_init_beltrami(glib, klm):
    s = initial.beltrami(16, *klm)
    ctx = _ctx_from_spec(glib, s, abi.init_spec(abi.INIT_BELTRAMI, klm=klm))
    _check(ctx, s)


def test_init_then_step_matches_host_state(glib):
    """A step from the device-generated state equals a step from the uploaded
    host state (the same inputs)."""
    s = initial.thermal(16, seed=3)
    a = _ctx_from_spec(glib, s, abi.init_spec(abi.INIT_THERMAL, seed=3))
    a.init_correction()
    b = make_context(s, glib)
    ta, ia = a.step(0.0)
    tb, ib = b.step(0.0)
    assert abs(ia.dt - ib.dt) <= 1e-12 * ib.dt
    assert abs(ia.parcel_stats[1] - ib.parcel_stats[1]) <= 1e-10 * abs(ib.parcel_stats[1])
