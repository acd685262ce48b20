"""Damping (parcel_damping.f90) and surface fluxes (bndry_fluxes.f90).

The reference has no tests for either; its design statements are the pins:
perturbation damping "nudges all the parcels associated with a grid point to
the grid point value ... in a conservative manner" (parcel_damping.f90:2-6),
so scalar damping keeps sum(V h) and sum(V b) (checked on the oracle here and
on the device at a size the oracle would take minutes for); the flux of a
uniform field has the closed form fac * 2 dxi(3) F (bndry_fluxes.f90:160-170,
232-238).  The device is then held to the oracle call by call."""
import numpy as np
import pytest

from epic_b200 import make_context
from tests.conftest import rel_err
from tests.helpers import small_state

MODES = {
    "vorticity": dict(damping_vorticity=1),
    "scalars": dict(damping_scalars=1),
    "surface": dict(damping_surface_vorticity=1, damping_surface_scalars=1),
    "mixed_kinds": dict(damping_vorticity=1, damping_surface_scalars=1),
}
PREF = dict(damping_vorticity_prefactor=3.0, damping_scalars_prefactor=5.0)


def _state(seed=11, n=16):
    s = small_state("thermal", n=n, seed=seed)
    rng = np.random.default_rng(seed + 1)
    # humidity and buoyancy with structure on the grid scale, so that the
    # gridded values differ from the parcels' own
    s.hum = np.abs(rng.normal(0.0, 1e-3, s.n)) + 1e-3 * (1 + np.sin(3 * s.pos[:, 0]))
    s.buoy = s.buoy + rng.uniform(-1e-2, 1e-2, s.n)
    return s


def _moments(ctx):
    p = ctx.get_parcels()
    return np.array([np.sum(p["vol"] * p["hum"]), np.sum(p["vol"] * p["buoy"])])


# ---------------------------------------------------------------------------
# oracle (CPU)

@pytest.mark.parametrize("mode", ["scalars", "surface"])
def test_oracle_scalar_damping_conserves(olib, mode):
    s = _state()
    oc = make_context(s, olib, **MODES[mode], **PREF)
    m0 = _moments(oc)
    before = oc.get_parcels()
    oc.parcel_damp(0.4)
    after = oc.get_parcels()
    changed = np.abs(after["hum"] - before["hum"]) > 0
    assert changed.sum() > (0.5 * s.n if mode == "scalars" else 0.02 * s.n)
    assert rel_err(_moments(oc), m0) < 1e-12
    if mode == "surface":
        # only parcels within two cells of a surface can change
        z = before["pos"][:, 2]
        far = (z > s.lower[2] + 2 * s.dx[2]) & (z < s.lower[2] + s.extent[2] - 2 * s.dx[2])
        assert not np.any(changed & far)


def test_oracle_damping_flags_conflict(olib):
    from epic_b200 import abi
    s = _state()
    for bad in (dict(damping_vorticity=1, damping_surface_vorticity=1),
                dict(damping_scalars=1, damping_surface_scalars=1)):
        with pytest.raises(abi.EpicError) as e:
            make_context(s, olib, **bad)
        assert e.value.code == 1


def test_oracle_uniform_flux_closed_form(olib):
    s = _state()
    oc = make_context(s, olib)
    F, H, dt = 0.3, -0.02, 0.25
    oc.set_bndry_fluxes(np.full((s.nx, s.ny), F), np.full((s.nx, s.ny), H))
    p0 = oc.get_parcels()
    oc.apply_bndry_fluxes(dt)
    p1 = oc.get_parcels()
    dxi = 1.0 / s.dx[2]
    zdepth = s.lower[2] + s.dx[2]
    z = p0["pos"][:, 2]
    fac = np.where(z < zdepth, (zdepth - z) * dxi * dt, 0.0)
    assert np.count_nonzero(fac) > 0.05 * s.n
    assert np.allclose(p1["buoy"] - p0["buoy"], fac * 2 * dxi * F, rtol=1e-12, atol=1e-15)
    assert np.allclose(p1["hum"] - p0["hum"], fac * 2 * dxi * H, rtol=1e-12, atol=1e-15)


def test_oracle_flux_time_step_bound(olib):
    s = _state()
    a = make_context(s, olib)
    b = make_context(s, olib)
    F = 50.0
    b.set_bndry_fluxes(np.full((s.nx, s.ny), F))
    _, dt0 = a.rk_step(0.0)
    _, dt1 = b.rk_step(0.0)
    bound = 0.2 * (s.dx[2] / (2 * F / s.dx[2])) ** (1.0 / 3.0)
    assert dt1 == pytest.approx(min(dt0, bound), rel=1e-14)
    assert dt1 < dt0


# ---------------------------------------------------------------------------
# device against the oracle

def _pair(s, olib, glib, **kw):
    return make_context(s, olib, **kw), make_context(s, glib, **kw)


def _cmp(oc, gc, tol):
    a, b = gc.get_parcels(), oc.get_parcels()
    assert len(a["vol"]) == len(b["vol"])
    for k in a:
        e = rel_err(a[k], b[k])
        assert e < tol, f"parcel {k}: rel err {e:.3e}"


@pytest.mark.gpu
@pytest.mark.parametrize("mode", list(MODES))
def test_parcel_damp_parity(olib, glib, mode):
    s = _state()
    oc, gc = _pair(s, olib, glib, **MODES[mode], **PREF)
    p0 = oc.get_parcels()
    oc.parcel_damp(0.4)
    gc.parcel_damp(0.4)
    _cmp(oc, gc, 1e-10)
    # the damping did something measurable
    p1 = oc.get_parcels()
    moved = max(rel_err(p1["vor"], p0["vor"]), rel_err(p1["hum"], p0["hum"]))
    assert moved > 1e-6


@pytest.mark.gpu
def test_parcel_damp_mixed_form(olib, glib):
    s = _state()
    kw = dict(**MODES["mixed_kinds"], **PREF)
    oc = make_context(s, olib, **kw)
    gc = make_context(s, glib, precision=1, **kw)
    oc.parcel_damp(0.4)
    gc.parcel_damp(0.4)
    a, b = gc.get_parcels(), oc.get_parcels()
    for k in ("vor", "hum", "buoy"):
        assert rel_err(a[k], b[k]) < 2e-6, k


@pytest.mark.gpu
def test_bndry_fluxes_parity(olib, glib):
    s = _state()
    rng = np.random.default_rng(5)
    bf = rng.uniform(-1, 1, (s.nx, s.ny))
    hf = rng.uniform(-1e-2, 1e-2, (s.nx, s.ny))
    oc, gc = _pair(s, olib, glib)
    for c in (oc, gc):
        c.set_bndry_fluxes(bf, hf)
        c.apply_bndry_fluxes(0.3)
    _cmp(oc, gc, 1e-13)


@pytest.mark.gpu
@pytest.mark.parametrize("fixed", [False, True])
def test_full_steps_damping_fluxes(olib, glib, fixed):
    """Three steps with vorticity and scalar damping and surface fluxes; the
    adaptive dt is bounded by the flux (bndry_fluxes_time_step)."""
    s = _state()
    kw = dict(damping_vorticity=1, damping_scalars=1, **PREF)
    if fixed:
        kw.update(use_fixed_dt=1, fixed_dt=0.05)
    oc, gc = _pair(s, olib, glib, **kw)
    rng = np.random.default_rng(9)
    bf = 5.0 + rng.uniform(-1, 1, (s.nx, s.ny))
    hf = rng.uniform(0, 1e-3, (s.nx, s.ny))
    oc.set_bndry_fluxes(bf, hf)
    gc.set_bndry_fluxes(bf, hf)
    to = tg = 0.0
    for _ in range(3):
        to, io = oc.step(to)
        tg, ig = gc.step(tg)
        assert io.n_parcels == ig.n_parcels
        assert rel_err(ig.dt, io.dt) < 1e-12
        assert rel_err(np.array(ig.parcel_stats), np.array(io.parcel_stats)) < 1e-9
    _cmp(oc, gc, 1e-9)


@pytest.mark.gpu
def test_scalar_damping_conserves_large(glib):
    """sum(V h) and sum(V b) through scalar damping on a 64^3 grid (2.1M parcels)."""
    s = _state(n=64)
    gc = make_context(s, glib, keep_order=0, **MODES["scalars"], **PREF)
    m0 = _moments(gc)
    gc.parcel_damp(0.4)
    assert rel_err(_moments(gc), m0) < 1e-11
