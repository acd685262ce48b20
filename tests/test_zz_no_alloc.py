"""The allocation-free vorticity correction against the regular entry point.

Callers whose device memory belongs to another runtime's pool or budget, or
whose time loop must not take the implicit synchronisation of cudaMalloc,
use epic_gpu_apply_vortcor_noalloc on device arrays they own; its only
scratch is a fixed array inside the library.  This test calls it through the
C ABI twice in a row and checks each result against epic_gpu_apply_vortcor
on the same state (1e-10 relative, the plain FP64 tolerance of the parity
tests).  The file is named to be collected last."""
import ctypes as C

import numpy as np
import pytest

from tests.conftest import rel_err
from tests.helpers import small_state

pytestmark = pytest.mark.gpu


def _fn(glib):
    f = glib.lib.epic_gpu_apply_vortcor_noalloc
    f.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_void_p]
    f.restype = C.c_int
    return f


def test_noalloc_vortcor_matches_regular(glib):
    import torch
    from epic_b200 import make_context

    s = small_state("beltrami")
    n = s.n
    ctx = make_context(s, glib)            # vor_bar from the initial state
    vbar = (s.vor * s.vol[:, None]).sum(0) / s.vol.sum()
    f = _fn(glib)
    rng = np.random.default_rng(21)
    for trial in range(2):
        vor_new = s.vor + rng.normal(0.1 * (trial + 1), 0.2, size=(n, 3))
        # regular path: context-owned device state
        ctx.set_parcels(s.pos, vor_new, s.B, s.vol, s.buoy, s.hum)
        ctx.apply_vortcor()
        ref = ctx.get_parcels()["vor"]
        # allocation-free path on caller-owned device arrays ((n, 3) C order = Fortran (3, n))
        d_vol = torch.tensor(s.vol, dtype=torch.float64, device="cuda")
        d_vor = torch.tensor(vor_new, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        vb = (C.c_double * 3)(*vbar)
        dv = (C.c_double * 3)()
        rc = f(n, d_vol.data_ptr(), d_vor.data_ptr(), vb, dv, None)
        assert rc == 0
        torch.cuda.synchronize()
        out = d_vor.cpu().numpy()
        assert rel_err(out, ref) < 1e-10
        expect = (vor_new * s.vol[:, None]).sum(0) / s.vol.sum() - vbar
        assert np.allclose(np.array(dv[:]), expect, rtol=1e-10, atol=1e-14)


def test_noalloc_rejects_oversize(glib):
    import torch
    f = _fn(glib)
    d = torch.zeros(3, dtype=torch.float64, device="cuda")
    vb = (C.c_double * 3)(0.0, 0.0, 0.0)
    # beyond the stated maximum of 67,108,864 parcels: refused before any launch
    assert f(67108864 + 1, d.data_ptr(), d.data_ptr(), vb, None, None) == 2   # EPIC_ERR_CAPACITY


def test_noalloc_on_caller_stream_without_readback(glib):
    """On a stream the caller owns and with dvor_out = NULL (no copy, no
    synchronisation by the library), vor is still corrected: the caller
    synchronises its own stream and compares with the regular path."""
    import torch
    from epic_b200 import make_context

    s = small_state("thermal")
    n = s.n
    ctx = make_context(s, glib)
    vbar = (s.vor * s.vol[:, None]).sum(0) / s.vol.sum()
    vor_new = s.vor + np.random.default_rng(5).normal(0.05, 0.1, size=(n, 3))
    ctx.set_parcels(s.pos, vor_new, s.B, s.vol, s.buoy, s.hum)
    ctx.apply_vortcor()
    ref = ctx.get_parcels()["vor"]
    f = _fn(glib)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        d_vol = torch.tensor(s.vol, dtype=torch.float64, device="cuda")
        d_vor = torch.tensor(vor_new, dtype=torch.float64, device="cuda")
    stream.synchronize()
    vb = (C.c_double * 3)(*vbar)
    assert f(n, d_vol.data_ptr(), d_vor.data_ptr(), vb, None, C.c_void_p(stream.cuda_stream)) == 0
    stream.synchronize()
    assert rel_err(d_vor.cpu().numpy(), ref) < 1e-10
