"""Labels (the reference's ENABLE_LABELS build): a 64-bit label and a log
dilution per parcel (parcel_container.f90:41-57).

* initial states: label = 1 + the regular-position index, dilution 0
  (parcel_init.f90:135-139);
* split: the child takes the parent's label and dilution (parcel_split.f90:147-150);
* merge: per small parcel, in merge order, a uniform draw keeps the target's
  label with probability vm / (vm + v_small) (dilution += log(vm / (vm + v)))
  or takes the small parcel's (dilution = its dilution + log(v / (vm + v)))
  (parcel_merge.f90:181-203); the draw comes from a counter-based generator
  (label_seed, merge call, m) instead of Fortran's random_number;
* delete and the box sort move labels with their parcels; a restart from a
  parcel file resets them to the file index (parcel_netcdf.f90:709-716).

The oracle is checked against these rules on the CPU, the device against the
oracle on the GPU."""
import numpy as np
import pytest

from epic_b200 import abi, initial, make_context
from tests.conftest import rel_err
from tests.helpers import small_state


def _labelled(lib, state, **kw):
    ctx = make_context(state, lib, labels=1, label_seed=11, **kw)
    n = ctx.num_parcels()
    ctx.set_labels(np.arange(1, n + 1), np.zeros(n))
    return ctx


def test_labels_off_is_an_error(olib):
    ctx = make_context(small_state("thermal", n=8), olib)
    with pytest.raises(abi.EpicError) as e:
        ctx.get_labels()
    assert e.value.code == 7


def test_oracle_initial_labels(olib):
    spec = initial.device_spec("thermal-16")
    cfg = olib.default_config(spec.nx, spec.ny, spec.nz, spec.lower, spec.extent, labels=1)
    ctx = abi.EpicContext(olib, cfg)
    ctx.init_state(spec.init_spec())
    lab, dil = ctx.get_labels()
    npd, nx, ny, nz = 2, spec.nx, spec.ny, spec.nz
    p = np.arange(nx * ny * nz * npd ** 3)
    i, q = p % npd + 1, p // npd
    j, q = q % npd + 1, q // npd
    k, q = q % npd + 1, q // npd
    ix, q = q % nx, q // nx
    iy, iz = q % ny, q // ny
    want = 1 + (ix * npd + i - 1) + nx * npd * ((iy * npd + j - 1) + ny * npd * (iz * npd + k - 1))
    assert np.array_equal(lab, want) and np.all(dil == 0)
    assert np.array_equal(np.sort(lab), np.arange(1, len(p) + 1))


def test_oracle_split_copies_labels(olib):
    s = small_state("thermal", n=8, stretch=True, seed=3)
    ctx = _labelled(olib, s)
    n0 = ctx.num_parcels()
    lab0, _ = ctx.get_labels()
    ctx.set_labels(lab0, np.linspace(-1.0, 0.0, n0))
    _, dil0 = ctx.get_labels()
    ns = ctx.split()
    assert ns > 0
    lab, dil = ctx.get_labels()
    assert np.array_equal(lab[:n0], lab0) and np.array_equal(dil[:n0], dil0)
    # every child carries the label and dilution of a parent that split
    assert set(lab[n0:]) <= set(lab0)
    assert np.array_equal(dil[n0:], dil0[lab[n0:] - 1])


def _merge_outcomes(ctx):
    """Merge once from labels 1..n; for every single-small-parcel group return
    (p_keep = vm / (vm + v), kept, dilution ok)."""
    p0 = ctx.get_parcels()
    vol = p0["vol"]
    nm = ctx.merge()
    assert nm > 0
    isma, iclo = ctx.merge_pairs()
    lab, dil = ctx.get_labels()
    where = {int(l): q for q, l in enumerate(lab)}
    ic_count = np.bincount(iclo, minlength=len(vol) + 1)
    out = []
    for is_, ic in zip(isma, iclo):
        if ic_count[ic] != 1:
            continue
        vm, v = vol[ic - 1], vol[is_ - 1]
        if ic in where:
            kept, d, want = True, dil[where[ic]], np.log(vm / (vm + v))
        else:
            kept, d, want = False, dil[where[is_]], np.log(v / (vm + v))
        out.append((vm / (vm + v), kept, abs(d - want) <= 1e-15 * max(1.0, abs(want))))
    return out


def test_oracle_merge_label_law(olib):
    """The target keeps its label with probability vm / (vm + v_small): over
    many single merges the count of kept labels is within 4 sigma of the sum
    of those probabilities, and every dilution follows its formula."""
    out = []
    for seed in range(4):
        ctx = _labelled(olib, small_state("thermal", n=16, small_frac=0.05, seed=seed))
        out += _merge_outcomes(ctx)
    p = np.array([o[0] for o in out])
    kept = np.array([o[1] for o in out])
    assert len(out) > 200 and all(o[2] for o in out)
    mean, sd = p.sum(), np.sqrt((p * (1 - p)).sum())
    assert abs(kept.sum() - mean) < 4 * sd
    assert 0 < (~kept).sum()   # some labels were taken from the small parcel


@pytest.mark.gpu
def test_labels_parity(olib, glib):
    """Steps with merges and splits in the reference's parcel order: the same
    labels as the oracle and the same dilutions to rounding of log."""
    s = small_state("thermal", n=16, small_frac=0.03, seed=21)
    oc = _labelled(olib, s)
    gc = _labelled(glib, s, keep_order=1)
    to = tg = 0.0
    merged = 0
    for _ in range(3):
        to, io = oc.step(to)
        tg, ig = gc.step(tg)
        merged += io.n_merges
        assert io.n_parcels == ig.n_parcels and io.n_merges == ig.n_merges
    assert merged > 0
    lo, do = oc.get_labels()
    lg, dg = gc.get_labels()
    assert np.array_equal(lg, lo)
    assert rel_err(dg, do) < 1e-13


@pytest.mark.gpu
def test_labels_follow_the_box_sort(glib):
    """With the box sort (keep_order = 0) a step without merges or splits
    permutes the stored parcels; labels, dilutions and volumes move with
    them, and the ABI returns all three in the reference's container order,
    where they are unchanged by the step."""
    s = small_state("thermal", n=16, seed=4)
    gc = _labelled(glib, s, keep_order=0)
    n = gc.num_parcels()
    gc.set_labels(np.arange(1, n + 1), -np.arange(n) / n)
    v0 = gc.get_parcels()["vol"].copy()
    _, info = gc.step(0.0)
    assert info.n_merges == 0 and info.n_splits == 0
    lab, dil = gc.get_labels()
    vol = gc.get_parcels()["vol"]
    assert np.array_equal(lab, np.arange(1, n + 1))
    assert np.array_equal(vol, v0) and np.array_equal(dil, -np.arange(n) / n)


@pytest.mark.gpu
def test_device_initial_labels_and_files(olib, glib, tmp_path):
    """init_state labels match the oracle's; a parcel file carries them as an
    NC_INT64 variable (CDF-5); a restart resets them to the file index."""
    from epic_b200.ncfiles import NcFiles
    spec = initial.device_spec("thermal-16")
    cfg_o = olib.default_config(spec.nx, spec.ny, spec.nz, spec.lower, spec.extent, labels=1)
    cfg_g = glib.default_config(spec.nx, spec.ny, spec.nz, spec.lower, spec.extent, labels=1, keep_order=0)
    oc, gc = abi.EpicContext(olib, cfg_o), abi.EpicContext(glib, cfg_g)
    oc.init_state(spec.init_spec())
    gc.init_state(spec.init_spec())
    assert np.array_equal(gc.get_labels()[0], oc.get_labels()[0])
    gc.init_correction()
    t, _ = gc.step(0.0)
    lab, dil = gc.get_labels()
    f = str(tmp_path / "lab_parcels.nc")
    gc.write_parcels_nc(f, t)
    assert open(f, "rb").read(4) == b"CDF\x05"
    nc = NcFiles(glib)
    assert np.array_equal(nc.read_variable(f, "label").astype(np.int64), lab)
    assert np.array_equal(nc.read_variable(f, "dilution"), dil)
    r = abi.EpicContext(glib, cfg_g)
    r.read_parcels_nc(f)
    l2, d2 = r.get_labels()
    assert np.array_equal(l2, np.arange(1, len(lab) + 1)) and np.all(d2 == 0)
