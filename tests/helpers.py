"""Shared inputs for the parity tests."""
import math

import numpy as np

from epic_b200 import initial


def small_state(kind="thermal", n=16, seed=7, small_frac=0.0, stretch=False):
    """A perturbed initial state on an n^3 grid.

    small_frac > 0 turns that fraction of parcels (chosen by a seeded RNG,
    biased to the periodic edges) into small parcels V < vmin to exercise
    merging; stretch deforms the shapes to exercise splitting."""
    if kind == "thermal":
        s = initial.thermal(n, seed=seed)
    else:
        s = initial.beltrami(n)
    rng = np.random.default_rng(seed)
    if kind == "beltrami":
        # a little position noise so that no two parcels are equidistant
        s.pos = s.pos + rng.uniform(-0.05, 0.05, s.pos.shape) * s.dx[None, :]
        s.pos[:, 2] = np.clip(s.pos[:, 2], s.lower[2] + 1e-9, s.lower[2] + s.extent[2] - 1e-9)
    s.vor = s.vor + rng.uniform(-0.1, 0.1, s.vor.shape)
    s.hum = np.abs(rng.normal(0.0, 1e-3, s.n))
    if small_frac > 0:
        vmin = np.prod(s.dx) / s.options["min_vratio"]
        pick = rng.random(s.n) < small_frac
        # make parcels near the x/y edges small more often
        edge = (np.abs(s.pos[:, 0] - s.lower[0]) < 0.6 * s.dx[0]) | \
               (np.abs(s.pos[:, 0] - s.lower[0] - s.extent[0]) < 0.6 * s.dx[0]) | \
               (np.abs(s.pos[:, 1] - s.lower[1]) < 0.6 * s.dx[1]) | \
               (np.abs(s.pos[:, 1] - s.lower[1] - s.extent[1]) < 0.6 * s.dx[1])
        pick |= edge & (rng.random(s.n) < 4 * small_frac)
        newv = rng.uniform(0.3, 0.95, s.n) * vmin
        scale = (newv / s.vol) ** (2.0 / 3.0)
        s.vol = np.where(pick, newv, s.vol)
        s.B = s.B * np.where(pick, scale, 1.0)[:, None]
    if stretch:
        # random volume-preserving deformation B -> M B M^T (stored upper part)
        Bf = np.zeros((s.n, 3, 3))
        abc = 0.75 * s.vol / math.pi
        Bf[:, 0, 0] = s.B[:, 0]; Bf[:, 1, 1] = s.B[:, 3]
        Bf[:, 2, 2] = abc ** 2 / (s.B[:, 0] * s.B[:, 3])
        # three distinct stretch factors: exactly degenerate eigenvalues
        # would leave the in-plane eigenvectors (and so the support points)
        # undetermined up to rounding
        l1 = rng.uniform(1.05, 2.2, s.n)
        l2 = rng.uniform(0.5, 0.95, s.n)
        A = np.zeros((s.n, 3, 3))
        A[:, 0, 0] = l1; A[:, 1, 1] = l2; A[:, 2, 2] = 1.0 / (l1 * l2)
        q, _ = np.linalg.qr(rng.normal(size=(s.n, 3, 3)))
        M = q @ A @ np.transpose(q, (0, 2, 1))
        Bn = M @ Bf @ np.transpose(M, (0, 2, 1))
        s.B = np.stack([Bn[:, 0, 0], Bn[:, 0, 1], Bn[:, 0, 2], Bn[:, 1, 1], Bn[:, 1, 2]], 1)
    return s


def pair(setup, olib, glib, init=True, **overrides):
    """Oracle and GPU contexts loaded with the same state."""
    from epic_b200 import make_context
    oc = make_context(setup, olib, **overrides)
    gc = make_context(setup, glib, **overrides)
    return oc, gc


def parcel_errors(a, b, extent):
    """Relative errors (to the largest |value| of b) of every parcel attribute
    of a against b, parcel by parcel in container order.  Horizontal position
    differences are taken modulo the period: a parcel within rounding of a
    periodic edge may be stored on either side of it (apply_periodic_bc,
    parcel_bc.f90:17-40, truncates (x - centre) * 2 / L, so one ulp decides)."""
    out = {}
    for k in a:
        x = np.asarray(a[k], dtype=np.float64)
        y = np.asarray(b[k], dtype=np.float64)
        d = x - y
        if k == "pos":
            for c in (0, 1):
                d[:, c] -= extent[c] * np.round(d[:, c] / extent[c])
        out[k] = float(np.abs(d).max() / max(np.abs(y).max(), 1e-300)) if len(y) else 0.0
    return out
