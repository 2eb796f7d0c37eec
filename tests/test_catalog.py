"""Device catalogs (fc_catalog_*), add_random_particles with device RNG and
apply_displacement_field on the GPU.

The generator is Philox4x32-10 (counter-based), so the checks are: exact
reproducibility for a seed, independence from batching, ranges, and the
first two moments against their expectations (5 sigma).  The displacement is
deterministic arithmetic and is compared bit for bit with the oracle's
restatement of fftcorr/grid/utils.pyx:21-40.
"""
import numpy as np
import pytest

from oracle import fc_oracle as O

import fftcorr_b200 as fb
from fftcorr_b200 import catalog
from fftcorr_b200.grid import apply_displacement_field

pytestmark = pytest.mark.gpu


def test_uniform_catalog_reproducible_and_in_range():
    lo, hi = [-5.0, 0.0, 100.0], [15.0, 40.0, 130.0]
    a = catalog.uniform(200000, lo, hi, seed=7, wmin=0.5, wmax=1.5).to_host()
    b = catalog.uniform(200000, lo, hi, seed=7, wmin=0.5, wmax=1.5).to_host()
    c = catalog.uniform(200000, lo, hi, seed=8, wmin=0.5, wmax=1.5).to_host()
    assert np.array_equal(a, b)
    assert not np.array_equal(a, c)
    assert np.all(a[:, :3] >= lo) and np.all(a[:, :3] < hi)
    assert np.all(a[:, 3] >= 0.5) and np.all(a[:, 3] < 1.5)
    n = a.shape[0]
    for j in range(3):
        u = (a[:, j] - lo[j]) / (hi[j] - lo[j])
        assert abs(u.mean() - 0.5) < 5 * np.sqrt(1 / 12 / n)
        assert abs(u.var() - 1 / 12) < 5 * np.sqrt(1 / 180 / n)
    # Independent coordinates: correlation near zero.
    assert abs(np.corrcoef(a[:, 0], a[:, 1])[0, 1]) < 5 / np.sqrt(n)


def test_clustered_box_in_box_and_clustered():
    L = 500.0
    a = catalog.clustered_box(100000, L, seed=3, ncentres=20, sigma=5.0).to_host()
    assert np.all(a[:, :3] >= 0) and np.all(a[:, :3] < L)
    assert np.all(a[:, 3] == 1.0)
    # 20 clumps of width 5 in a 500 box: counts in 10^3 cells are far from
    # Poisson.
    h, _ = np.histogramdd(a[:, :3], bins=10, range=[(0, L)] * 3)
    assert h.var() > 20 * h.mean()


def test_sector_catalog_geometry():
    a = catalog.sector(100000, seed=5, rmin=500, rmax=1500, ra_deg=30,
                       dec_deg=30, wmin=0.5, wmax=1.5, wsign=-1.0).to_host()
    r = np.linalg.norm(a[:, :3], axis=1)
    assert np.all(r >= 500 - 1e-9) and np.all(r < 1500 + 1e-9)
    ra = np.degrees(np.arctan2(a[:, 1], a[:, 0]))
    dec = np.degrees(np.arcsin(a[:, 2] / r))
    assert np.all(np.abs(ra) <= 30 + 1e-9) and np.all(np.abs(dec) <= 30 + 1e-9)
    assert np.all(a[:, 3] <= -0.5) and np.all(a[:, 3] > -1.5)
    # r^3 uniform: median radius.
    med = ((500 ** 3 + 1500 ** 3) / 2) ** (1 / 3)
    assert abs(np.median(r) - med) < 0.01 * med


def test_add_random_particles_independent_of_batch_size():
    grids = []
    for batch in (100000, 33333):
        g = fb.ConfigSpaceGrid.from_geometry((32, 32, 32), [10.0, -20.0, 0.0], 5.0)
        ma = catalog.add_random_particles(100000, g, fb.DistributionScheme.CLOUD_IN_CELL,
                                          total_weight=50.0, seed=11,
                                          batch_size=batch)
        assert ma.num_added == 100000 and ma.num_skipped == 0
        assert ma.totw == pytest.approx(50.0, rel=1e-12)
        grids.append(np.array(g.data))
    # Different batch splits sum the same particles in different flushes.
    assert np.max(np.abs(grids[0] - grids[1])) <= 1e-12 * np.max(np.abs(grids[0]))
    assert grids[0].sum() == pytest.approx(50.0, rel=1e-12)


def test_add_random_particles_rejects_both_weights():
    g = fb.ConfigSpaceGrid.from_geometry((8, 8, 8), [0, 0, 0], 1.0)
    with pytest.raises(ValueError):
        catalog.add_random_particles(10, g, 0, particle_weight=1.0, total_weight=2.0)


@pytest.mark.parametrize("periodic", [False, True])
def test_apply_displacement_matches_oracle(periodic):
    shape = (12, 10, 8)
    posmin = np.array([-3.0, 4.0, 10.0])
    cell = 2.5
    rng = np.random.default_rng(4)
    hi = posmin + np.array(shape) * cell
    lo = posmin - (0.2 if periodic else 0.0) * (hi - posmin)
    top = hi + (0.2 if periodic else -1e-9) * (hi - posmin)
    pos = lo + (top - lo) * rng.random((5000, 3))
    disp = rng.normal(0, 1.0, shape + (3,))
    g = fb.ConfigSpaceGrid.from_geometry(shape, posmin, cell)
    got = apply_displacement_field(g, pos, disp, periodic_wrap=periodic)
    ref = O.apply_displacement_field(pos, disp, posmin, cell, shape, periodic)
    assert np.array_equal(got, ref)


def test_apply_displacement_out_of_bounds_raises():
    g = fb.ConfigSpaceGrid.from_geometry((4, 4, 4), [0, 0, 0], 1.0)
    pos = np.array([[0.5, 0.5, 0.5], [5.0, 0.5, 0.5]])
    with pytest.raises(ValueError):
        apply_displacement_field(g, pos, np.zeros((4, 4, 4, 3)))
