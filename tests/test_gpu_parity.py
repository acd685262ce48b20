"""Parity of the CUDA step with the FP64 oracle, call by call, on identical
inputs.  Tolerances: 1e-10 relative for the plain FP64 path (the per-call
bar; observed differences are rounding, ~1e-14); merge pairs, split counts
and parcel counts bit-exact."""
import math

import numpy as np
import pytest

from epic_b200 import abi, initial, make_context
from tests.conftest import rel_err
from tests.helpers import pair, parcel_errors, small_state

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _fields(ctx, ids):
    return {i: ctx.get_field(i) for i in ids}


def _cmp_fields(oc, gc, ids, tol=TOL, rows=slice(None)):
    for i in ids:
        a = gc.get_field(i)[:, :, rows]
        b = oc.get_field(i)[:, :, rows]
        e = rel_err(a, b)
        assert e < tol, f"{abi.FIELD_NAMES[i]}: rel err {e:.3e}"


def _cmp_parcels(oc, gc, tol=TOL):
    a, b = gc.get_parcels(), oc.get_parcels()
    assert len(a["vol"]) == len(b["vol"])
    ext = np.array(gc.cfg.extent[:])
    for k, e in parcel_errors(a, b, ext).items():
        assert e < tol, f"parcel {k}: rel err {e:.3e}"


def test_eigen_golden_gpu(glib):
    """test_scherzinger_2 on the device (atol 1e-12), both arithmetic modes."""
    import ctypes as C
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "scherzinger_BDV.npz"))
    f = glib.lib.epic_gpu_test_eigen
    P = C.POINTER(C.c_double)
    f.argtypes = [C.c_int64, P, P, P, C.c_int, C.c_int]
    A = np.ascontiguousarray(g["B"])
    for exact in (0, 1):
        D = np.empty((len(A), 3)); V = np.empty((len(A), 9))
        assert f(len(A), A.ctypes.data_as(P), D.ctypes.data_as(P), V.ctypes.data_as(P), exact, 0) == 0
        err = 0.0
        for n in range(len(A)):
            e = np.abs(g["D"][n] - D[n]).sum()
            Q = g["V"][n].reshape(3, 3)
            for k in range(3):
                q = Q[k].copy(); v = V[n, 3 * k:3 * k + 3]
                if q[0] / v[0] < 0:
                    q = -q
                e = max(e, np.abs(q - v).sum())
            err = max(err, e)
        assert err < 1e-12


def test_eigen_exact_matches_oracle_bitwise(glib, olib):
    """The non-contracted device eigenvalues equal the oracle's bit for bit
    on the golden matrices (the split decision depends on them)."""
    import ctypes as C
    import os
    import oracle
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "scherzinger_BDV.npz"))
    A = np.ascontiguousarray(g["B"])
    P = C.POINTER(C.c_double)
    D = np.empty((len(A), 3)); V = np.empty((len(A), 9))
    glib.lib.epic_gpu_test_eigen(len(A), A.ctypes.data_as(P), D.ctypes.data_as(P), V.ctypes.data_as(P), 1, 1)
    Do, _ = oracle.eigen(olib, A, values_only=True)
    # acos/cos of glibc and CUDA may differ in the last bit; allow 4 ulp
    assert np.abs(D - Do).max() <= 4 * np.spacing(np.abs(Do).max())


@pytest.mark.parametrize("shape,plane", [((64, 64, 64), 0), ((64, 64, 64), 1), ((64, 64, 64), 2),
                                         ((64, 64, 64), 3), ((128, 128, 32), 3),
                                         ((16, 16, 16), 0), ((32, 32, 24), 0), ((128, 128, 32), 0),
                                         ((48, 32, 16), 0), ((256, 256, 16), 0), ((64, 256, 16), 0),
                                         ((512, 512, 8), 0), ((128, 128, 128), 1), ((128, 128, 32), 1),
                                         ((32, 32, 24), 1), ((16, 16, 16), 1), ((256, 256, 16), 1),
                                         ((512, 512, 8), 1), ((48, 48, 48), 1), ((96, 96, 48), 1),
                                         ((96, 48, 16), 0), ((48, 48, 48), 0)])
def test_vor2vel_taylor_green_kat(glib, shape, plane):
    """test_mpi_vor2vel.f90: Taylor-Green vorticity on 64^3, max err < 1e-14; the
    same flow on other grids through the horizontal FFT paths (2-D plane
    kernel for square 16..128 grids, tiled register FFT for power-of-two axes
    up to 512 and for 48 and 96 (radix 3 x 4 and 3 x 8 in registers), Stockham
    lines otherwise, half-plane cluster kernel for square
    64 and 128)."""
    nx, ny, nz = shape
    lower = (-math.pi, -math.pi, -0.5 * math.pi)
    extent = (2 * math.pi, 2 * math.pi, 2 * math.pi)
    cfg = glib.default_config(nx, ny, nz, lower, extent)
    ctx = abi.EpicContext(glib, cfg)
    glib.lib.epic_gpu_test_set_fft_path(ctx.h, plane)
    tol = 1e-14 * max(1.0, max(shape) / 64.0)
    dx = np.array(extent) / np.array([nx, ny, nz])
    x = lower[0] + np.arange(nx) * dx[0]
    y = lower[1] + np.arange(ny) * dx[1]
    z = lower[2] + np.arange(-1, nz + 2) * dx[2]
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    AA, BB, CC = 1.0, 1.0, -2.0
    ctx.set_field(abi.VORTG[0], (CC - BB) * np.sin(X) * np.cos(Y) * np.cos(Z))
    ctx.set_field(abi.VORTG[1], (AA - CC) * np.cos(X) * np.sin(Y) * np.cos(Z))
    ctx.set_field(abi.VORTG[2], (BB - AA) * np.cos(X) * np.cos(Y) * np.sin(Z))
    ctx.vor2vel()
    ref = [AA * np.cos(X) * np.sin(Y) * np.sin(Z), BB * np.sin(X) * np.cos(Y) * np.sin(Z),
           CC * np.sin(X) * np.sin(Y) * np.cos(Z)]
    err = max(np.abs(ctx.get_field(abi.VELOG[i])[:, :, 1:-1] - ref[i][:, :, 1:-1]).max() for i in range(3))
    assert err < tol
    # velocity gradient of the same flow (cf. test_mpi_vel2vgrad.f90, 2e-14)
    dudx = -AA * np.sin(X) * np.sin(Y) * np.sin(Z)
    dvdy = -BB * np.sin(X) * np.sin(Y) * np.sin(Z)
    dwdx = CC * np.cos(X) * np.sin(Y) * np.cos(Z)
    for fid, r in ((abi.VELGRADG[0], dudx), (abi.VELGRADG[4], dvdy), (abi.VELGRADG[6], dwdx)):
        assert np.abs(ctx.get_field(fid)[:, :, 1:-1] - r[:, :, 1:-1]).max() < 2 * tol


@pytest.mark.parametrize("kind", ["thermal", "beltrami"])
def test_par2grid(olib, glib, kind):
    s = small_state(kind)
    oc, gc = pair(s, olib, glib)
    oc.par2grid(False); gc.par2grid(False)
    _cmp_fields(oc, gc, list(abi.VORTG) + [abi.TBUOYG, abi.DBUOYG, abi.HUMG, abi.VOLG], rows=slice(None))
    for fid in (abi.NPARG, abi.NSPARG):
        assert np.array_equal(gc.get_field(fid)[:, :, 1:-2], oc.get_field(fid)[:, :, 1:-2])


@pytest.mark.parametrize("kind,plane", [("thermal", 0), ("beltrami", 0), ("thermal", 1), ("thermal", 2),
                                        ("thermal", 3)])
def test_vor2vel_vtend_timestep(olib, glib, kind, plane):
    s = small_state(kind, n=64 if plane == 3 else 16)
    oc, gc = pair(s, olib, glib)
    glib.lib.epic_gpu_test_set_fft_path(gc.h, plane)
    for c in (oc, gc):
        c.par2grid(False)
        c.vor2vel()
        c.vorticity_tendency()
    _cmp_fields(oc, gc, list(abi.VELOG) + list(abi.VELGRADG) + list(abi.VORTG) + list(abi.VTEND))
    assert rel_err(gc.time_step(0.0), oc.time_step(0.0)) < TOL


@pytest.mark.parametrize("add", [False, True])
def test_grid2par(olib, glib, add):
    s = small_state("thermal")
    oc, gc = pair(s, olib, glib)
    oc.par2grid(False); oc.vor2vel(); oc.vorticity_tendency()
    ids = list(abi.VELOG) + list(abi.VELGRADG) + list(abi.VTEND)
    for i in ids:
        gc.set_field(i, oc.get_field(i))
    rng = np.random.default_rng(3)
    dp = rng.normal(size=(s.n, 3)); dv = rng.normal(size=(s.n, 3)); db = rng.normal(size=(s.n, 5))
    for c in (oc, gc):
        c.set_parcel_rk(dp, dv, db)
        c.grid2par(add)
    a, b = gc.get_parcel_rk(), oc.get_parcel_rk()
    for k in ("delta_pos", "delta_vor", "strain"):
        assert rel_err(a[k], b[k]) < TOL, k


@pytest.mark.parametrize("kind", ["thermal", "beltrami"])
def test_rk_step(olib, glib, kind):
    s = small_state(kind)
    oc, gc = pair(s, olib, glib)
    to, dto = oc.rk_step(0.0)
    tg, dtg = gc.rk_step(0.0)
    assert rel_err(dtg, dto) < TOL
    _cmp_parcels(oc, gc)


def test_merge_pairs_bit_exact(olib, glib):
    s = small_state("thermal", small_frac=0.05)
    oc, gc = pair(s, olib, glib)
    no, ng = oc.merge(), gc.merge()
    assert no == ng and no > 100
    io, co = oc.merge_pairs()
    ig, cg = gc.merge_pairs()
    assert np.array_equal(io, ig)
    assert np.array_equal(co, cg)
    assert oc.num_parcels() == gc.num_parcels()
    _cmp_parcels(oc, gc)


def test_merge_beltrami_edges(olib, glib):
    s = small_state("beltrami", small_frac=0.08, seed=11)
    oc, gc = pair(s, olib, glib)
    assert oc.merge() == gc.merge()
    assert all(np.array_equal(a, b) for a, b in zip(oc.merge_pairs(), gc.merge_pairs()))
    _cmp_parcels(oc, gc)


def test_split_bit_exact(olib, glib):
    s = small_state("thermal", stretch=True)
    oc, gc = pair(s, olib, glib)
    so, sg = oc.split(), gc.split()
    assert so == sg and so > 100
    _cmp_parcels(oc, gc)


@pytest.mark.parametrize("precision,keep_order", [(0, 1), (1, 1), (0, 0)])
def test_split_grows_full_container(olib, glib, precision, keep_order):
    """A split that overflows the container grows it (parcel_split.f90:91-94,
    grow_factor x the parcels needed) and keeps every parcel; steps go on.
    keep_order = 0: the box-sorted store, whose sort scratch (which holds the
    split's flags) is resized for the new capacity behind the split kernel."""
    s = small_state("thermal", stretch=True)
    oc = make_context(s, olib)
    gc = make_context(s, glib, capacity=s.n + 64, precision=precision, keep_order=keep_order)
    so, sg = oc.split(), gc.split()
    assert sg > 64
    po, pg = oc.get_parcels(), gc.get_parcels()
    assert len(pg["vol"]) == s.n + sg
    if precision == 0:
        assert so == sg
        assert np.array_equal(pg["vol"], po["vol"])
        _cmp_parcels(oc, gc)
    else:   # FP32 shapes: decisions may differ at the threshold, positions by rounding
        assert abs(so - sg) <= 2
        if so == sg:
            assert np.abs(pg["pos"] - po["pos"]).max() < 1e-5 * s.dx.min()
    t, _ = gc.step(0.0)
    assert t > 0


@pytest.mark.parametrize("reuse", [False, True])
def test_corrections(olib, glib, reuse):
    s = small_state("thermal", stretch=True)
    oc, gc = pair(s, olib, glib)
    for c in (oc, gc):
        c.vol2grid(False)   # fills the stored support vectors for reuse
        c.apply_laplace(reuse)
    _cmp_parcels(oc, gc)
    for c in (oc, gc):
        c.apply_gradient(True)
    _cmp_parcels(oc, gc)


def test_vortcor_and_diagnostics(olib, glib):
    s = small_state("beltrami")
    oc, gc = pair(s, olib, glib)
    for c in (oc, gc):
        c.apply_vortcor()
        c.par2grid(False); c.vor2vel(); c.vorticity_tendency(); c.grid2par(False)
    _cmp_parcels(oc, gc)
    assert rel_err(gc.parcel_diagnostics(), oc.parcel_diagnostics()) < TOL
    assert rel_err(gc.field_diagnostics(), oc.field_diagnostics()) < TOL


@pytest.mark.parametrize("kind", ["thermal", "beltrami"])
def test_full_steps(olib, glib, kind):
    """Three complete steps (vortcor, RK4, merge, split, corrections): counts
    and merge pairs bit-exact, every state at 1e-10 after every step."""
    s = small_state(kind, small_frac=0.02)
    oc, gc = pair(s, olib, glib)
    to = tg = 0.0
    for k in range(3):
        to, io = oc.step(to)
        tg, ig = gc.step(tg)
        assert io.n_parcels == ig.n_parcels
        assert io.n_splits == ig.n_splits and io.n_merges == ig.n_merges
        assert rel_err(tg, to) < TOL
        assert rel_err(np.array(ig.parcel_stats), np.array(io.parcel_stats)) < TOL
        assert rel_err(np.array(ig.field_stats), np.array(io.field_stats)) < TOL
        assert all(np.array_equal(a, b) for a, b in zip(gc.merge_pairs(), oc.merge_pairs()))
        _cmp_parcels(oc, gc)


def test_diverge(olib, glib):
    """diverge (inversion.f90:410-455) of a smooth random field."""
    import ctypes as C
    s = small_state("thermal")
    oc, gc = pair(s, olib, glib)
    rng = np.random.default_rng(5)
    shape = gc.field_shape
    phi = np.zeros(shape)
    x = np.linspace(0, 2 * np.pi, shape[0], endpoint=False)
    for _ in range(6):
        kx, ky, kz = rng.integers(0, 4, 3)
        X, Y, Z = np.meshgrid(x, x, np.linspace(0, 1, shape[2]), indexing="ij")
        phi += rng.normal() * np.cos(kx * X + rng.uniform()) * np.cos(ky * Y) * np.cos(np.pi * kz * Z)
    P = C.POINTER(C.c_double)
    go = np.empty((3,) + shape); gg = np.empty((3,) + shape)
    fo = olib.lib.epic_oracle_test_diverge
    fo.argtypes = [C.c_void_p, P, P]
    fg = glib.lib.epic_gpu_test_diverge
    fg.argtypes = [C.c_void_p, P, P]
    assert fo(oc.h, phi.ctypes.data_as(P), go.ctypes.data_as(P)) == 0
    assert fg(gc.h, phi.ctypes.data_as(P), gg.ctypes.data_as(P)) == 0
    for k in range(3):
        assert rel_err(gg[k], go[k]) < TOL, (k, rel_err(gg[k], go[k]))


@pytest.mark.parametrize("stretch", [False, True])
def test_vol2grid(olib, glib, stretch):
    s = small_state("thermal", stretch=stretch)
    oc, gc = pair(s, olib, glib)
    oc.vol2grid(False); gc.vol2grid(False)
    _cmp_fields(oc, gc, [abi.VOLG])


@pytest.mark.parametrize("case", ["p1", "p2", "p3", "p4"])
def test_nearest_constellations_gpu(olib, glib, case):
    """test_mpi_nearest_1..4 on the device: counts and pairs equal the oracle's."""
    from tests import test_oracle_cpu as T
    placement, expected = {"p1": (T._p1, 200), "p2": (T._p2, 200), "p3": (T._p3, 100), "p4": (T._p4, 100)}[case]
    oc, _ = T._nearest_case(olib, placement)
    gc, _ = T._nearest_case(glib, placement)
    assert gc.merge() == expected == oc.merge()
    assert all(np.array_equal(a, b) for a, b in zip(gc.merge_pairs(), oc.merge_pairs()))
    _cmp_parcels(oc, gc)


def _kat_params():
    from tests import test_oracle_cpu as T
    return T.NEAREST_KATS


@pytest.mark.parametrize("name,setup,expected,cell", _kat_params(),
                         ids=[f"{n[9:]}-{s}" for n, s, _, _ in _kat_params()])
def test_nearest_reference_kats_gpu(olib, glib, name, setup, expected, cell):
    """test_mpi_nearest_5.f90 .. _20.f90 on the device: the stated merge
    counts, and the oracle's pairs and merged parcels."""
    from tests import test_oracle_cpu as T
    oc, _ = T._nearest_case(olib, T.kat_placement(cell))
    gc, _ = T._nearest_case(glib, T.kat_placement(cell))
    assert gc.merge() == expected == oc.merge()
    assert all(np.array_equal(a, b) for a, b in zip(gc.merge_pairs(), oc.merge_pairs()))
    _cmp_parcels(oc, gc)


@pytest.mark.parametrize("kind", ["thermal", "beltrami"])
def test_par2grid_box_windows(olib, glib, kind):
    """par2grid and vol2grid through the box-ordered store (shared-memory
    fixed-point windows): after one step with keep_order=0 the parcel set is
    the oracle's in another order, and the gridded sums must agree."""
    s = small_state(kind, small_frac=0.02, seed=5)
    oc = make_context(s, olib)
    gc = make_context(s, glib, keep_order=0)
    oc.step(0.0)
    gc.step(0.0)
    oc.par2grid(False); gc.par2grid(False)
    _cmp_fields(oc, gc, list(abi.VORTG) + [abi.TBUOYG, abi.DBUOYG, abi.HUMG, abi.VOLG], tol=1e-9)
    oc.vol2grid(False); gc.vol2grid(False)
    _cmp_fields(oc, gc, [abi.VOLG], tol=1e-9)


@pytest.mark.parametrize("in_place", [False, True])
def test_full_steps_reordered_store(olib, glib, in_place):
    """keep_order=0: the device reorders parcels by boxes of cells each step
    (through a second store, or slot by slot in place) and carries each
    parcel's container index; merge pairs, counts and the parcels returned in
    container order equal the oracle's."""
    s = small_state("thermal", small_frac=0.02, seed=4)
    oc = make_context(s, olib)
    gc = make_context(s, glib, keep_order=0)
    if in_place:
        assert glib.lib.epic_gpu_test_drop_sort_store(gc.h) == 0
    to = tg = 0.0
    for k in range(3):
        to, io = oc.step(to)
        tg, ig = gc.step(tg)
        assert io.n_parcels == ig.n_parcels
        assert io.n_merges == ig.n_merges and io.n_splits == ig.n_splits
        assert rel_err(tg, to) < TOL
        assert rel_err(np.array(ig.parcel_stats), np.array(io.parcel_stats)) < TOL
        assert all(np.array_equal(a, b) for a, b in zip(gc.merge_pairs(), oc.merge_pairs()))
        _cmp_parcels(oc, gc)


@pytest.mark.parametrize("precision", [0, 1])
def test_autotune_keeps_results(glib, precision):
    """The autotuner only changes launch shapes: a step after tuning equals a
    step of an untuned context on the same state."""
    s = small_state("thermal", small_frac=0.02, seed=6)
    a = make_context(s, glib, keep_order=0, precision=precision)
    b = make_context(s, glib, keep_order=0, precision=precision)
    tune = a.autotune()
    assert 0 <= tune["lg_par2grid"] <= 3 and 0 <= tune["lg_vol2grid"] <= 3 and 0 <= tune["fft_path"] <= 3
    assert tune["ms_par2grid"] > 0 and tune["ms_fft"] > 0
    ta, ia = a.step(0.0)
    tb, ib = b.step(0.0)
    assert ia.n_parcels == ib.n_parcels
    assert rel_err(ta, tb) < 1e-10
    assert rel_err(np.array(ia.parcel_stats), np.array(ib.parcel_stats)) < 1e-9


def test_stage_variants_agree(glib):
    """The four variants of the stage phase (record window on / off, support
    vectors in the stage kernel or their own) give the same steps."""
    import ctypes as C
    s = small_state("thermal", small_frac=0.02, seed=8)
    L = glib.lib
    L.epic_gpu_test_set_stage_window.argtypes = [C.c_void_p, C.c_int]
    L.epic_gpu_test_set_stage_vectors.argtypes = [C.c_void_p, C.c_int]
    out = []
    for v in range(4):
        ctx = make_context(s, glib, keep_order=0)
        L.epic_gpu_test_set_stage_vectors(ctx.h, v & 1)
        L.epic_gpu_test_set_stage_window(ctx.h, (v >> 1) & 1)
        t = 0.0
        for _ in range(3):
            t, info = ctx.step(t)
        out.append((t, info.n_parcels, ctx.get_parcels()))
        ctx.close()
    for t, n, p in out[1:]:
        assert n == out[0][1] and rel_err(t, out[0][0]) < 1e-12
        for k in p:
            assert rel_err(p[k], out[0][2][k]) < 1e-11, k


@pytest.mark.parametrize("precision", [0, 1])
def test_par2grid_bitwise_reproducible(glib, precision):
    """par2grid and vol2grid sum exact integers at one fixed-point scale per
    field, so the gridded fields do not depend on the order of the adds: two
    calls on the same store, and calls with other lane mappings of the
    scatter, give bitwise the same fields.  The store is box ordered with
    split children in a tail (one step of a stretched state), so box windows,
    tail chunks and direct adds all take part."""
    import ctypes as C
    s = small_state("thermal", n=32, small_frac=0.02, seed=3, stretch=True)
    gc = make_context(s, glib, keep_order=0, precision=precision)
    _, info = gc.step(0.0)
    assert info.n_splits > 0
    ids = list(abi.VORTG) + [abi.TBUOYG, abi.DBUOYG, abi.HUMG, abi.VOLG, abi.NPARG, abi.NSPARG]
    f = glib.lib.epic_gpu_test_set_scatter_groups
    f.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
    runs = []
    for lg in (1, 1, 0, 3):
        assert f(gc.h, lg, lg, lg) == 0
        gc.par2grid(False)
        p2g = [gc.get_field(i).copy() for i in ids]
        gc.vol2grid(False)
        runs.append(p2g + [gc.get_field(abi.VOLG).copy()])
    for r in runs[1:]:
        for a, b in zip(r, runs[0]):
            assert np.array_equal(a.view(np.int64), b.view(np.int64))
