"""Synthetic initial states: determinism of the counter-based generator,
parcel placement of init_regular_positions, zeta boundary flags."""
import numpy as np

from epic_b200 import initial


def test_uniform_is_counter_based():
    idx = np.arange(1000, dtype=np.uint64)
    a = initial.uniform(7, idx, 2)
    b = initial.uniform(7, idx[::-1], 2)[::-1]
    assert np.array_equal(a, b)
    assert (a >= 0).all() and (a < 1).all()
    assert not np.array_equal(a, initial.uniform(8, idx, 2))
    assert abs(a.mean() - 0.5) < 0.05


def test_regular_positions_order():
    pos, vol, B = initial.regular_parcels(4, 4, 4, (0, 0, 0), (1, 1, 1), 8)
    assert len(pos) == 4 ** 3 * 8
    # first cell, parcels ordered i fastest then j then k (parcel_init.f90:125-143)
    assert np.allclose(pos[0], [0.0625, 0.0625, 0.0625])
    assert np.allclose(pos[1], [0.1875, 0.0625, 0.0625])
    assert np.allclose(pos[2], [0.0625, 0.1875, 0.0625])
    assert np.allclose(pos[4], [0.0625, 0.0625, 0.1875])
    assert np.allclose(vol, 1.0 / 4 ** 3 / 8)
    abc = 0.75 * vol[0] / np.pi
    assert np.allclose(B[0], [abc ** (2 / 3), 0, 0, abc ** (2 / 3), 0])


def test_thermal_and_beltrami_setups():
    t1 = initial.thermal(8, seed=5)
    t2 = initial.thermal(8, seed=5)
    assert np.array_equal(t1.pos, t2.pos) and np.array_equal(t1.buoy, t2.buoy)
    assert (t1.pos[:, 2] >= 0).all() and (t1.pos[:, 2] < 6.28).all()
    assert t1.n == 8 ** 3 * 8
    b = initial.beltrami(8)
    assert b.n == 8 ** 3 * 8
    assert b.options["bndry_zeta_zero"] == (1, 1)   # cos(z) vanishes at z = -pi/2, pi/2


def test_zeta_flags():
    z = np.random.default_rng(0).normal(size=(4, 4, 9))
    assert initial.zeta_boundary_flags(z) == (0, 0)
    z[:, :, 0] = 0.0
    assert initial.zeta_boundary_flags(z) == (1, 0)
