"""Parity at the benchmark configurations, through the C ABI, against the
oracle (the CPU restatement of the reference step, src/3d/epic3d.f90:135-153).

* Beltrami flow on 32^3 (262,144 parcels at the start, the configuration the
  reference runs on CPU): 10 full steps on the device, with the reference's
  container order kept (keep_order = 1) and with the box-ordered store that
  the benchmark times (keep_order = 0, container indices carried in a rank
  array), against the single-threaded oracle.  By step 10 the flow has split
  and merged several hundred thousand parcels; its symmetry makes many
  nearest-parcel distances tie exactly, so the merge pairs depend on the
  container order (parcel_nearest.f90:717-723, 1261-1311).  Every step: parcel,
  split and merge counts and the merge pairs (isma, iclo) bit-exact; dt and
  every parcel attribute within 1e-10 relative (measured at most 2e-12 after
  10 steps).
* Rising thermal on 128^3 (16,777,216 parcels): one step of the benchmarked
  path against the oracle's OpenMP build (whose sums are ordered otherwise,
  so the tolerance is 1e-10; measured 1.4e-14).
* The two store orders at size: a 64^3 thermal (2,097,152 parcels) with
  small and stretched parcels merges and splits from the first step; three
  steps with keep_order = 0 and 1 give the same counts and pairs and the same
  parcels in container order (1e-12)."""
import numpy as np
import pytest

from epic_b200 import initial, make_context
from tests.helpers import parcel_errors, small_state

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_beltrami32_ten_steps_both_store_orders(olib, glib):
    s = initial.config("beltrami-32")
    assert s.n == 262144
    oc = make_context(s, olib)
    gcs = {ko: make_context(s, glib, keep_order=ko) for ko in (1, 0)}
    to = 0.0
    tg = {ko: 0.0 for ko in gcs}
    merged = split = 0
    for step in range(10):
        to, io = oc.step(to)
        po = oc.get_parcels()
        pairs_o = oc.merge_pairs()
        merged += io.n_merges
        split += io.n_splits
        for ko, gc in gcs.items():
            tg[ko], ig = gc.step(tg[ko])
            where = f"step {step + 1}, keep_order {ko}"
            assert (ig.n_parcels, ig.n_splits, ig.n_merges) == (io.n_parcels, io.n_splits, io.n_merges), where
            assert _rel(ig.dt, io.dt) < TOL, where
            pg = gc.merge_pairs()
            assert all(np.array_equal(a, b) for a, b in zip(pg, pairs_o)), where
            err = parcel_errors(gc.get_parcels(), po, s.extent)
            assert max(err.values()) < TOL, (where, err)
    assert merged > 100000 and split > 500000


def test_thermal128_step_vs_oracle_openmp(glib):
    import oracle
    s = initial.config("thermal-128")
    assert s.n == 16777216
    oc = make_context(s, oracle.load(threads=True))
    to, io = oc.step(0.0)
    po = oc.get_parcels()
    oc.close()
    gc = make_context(s, glib, keep_order=0)
    tg, ig = gc.step(0.0)
    assert (ig.n_parcels, ig.n_splits, ig.n_merges) == (io.n_parcels, io.n_splits, io.n_merges)
    assert _rel(ig.dt, io.dt) < TOL
    assert _rel(ig.parcel_stats, io.parcel_stats) < TOL
    assert _rel(ig.field_stats, io.field_stats) < TOL
    err = parcel_errors(gc.get_parcels(), po, s.extent)
    assert max(err.values()) < TOL, err


def test_store_orders_agree_at_64cubed(glib):
    s = small_state("thermal", n=64, seed=9, small_frac=0.02, stretch=True)
    a = make_context(s, glib, keep_order=1)
    b = make_context(s, glib, keep_order=0)
    ta = tb = 0.0
    merges = splits = 0
    for step in range(3):
        ta, ia = a.step(ta)
        tb, ib = b.step(tb)
        assert (ia.n_parcels, ia.n_splits, ia.n_merges) == (ib.n_parcels, ib.n_splits, ib.n_merges), step
        assert all(np.array_equal(x, y) for x, y in zip(a.merge_pairs(), b.merge_pairs())), step
        err = parcel_errors(b.get_parcels(), a.get_parcels(), s.extent)
        assert max(err.values()) < 1e-12, (step, err)
        merges += ia.n_merges
        splits += ia.n_splits
    assert merges > 1000 and splits > 1000
