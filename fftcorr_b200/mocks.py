"""Seeded synthetic catalogs for benchmarks and serving tests.

There is no public benchmark catalog for this pipeline; these stand in for
survey data (a spherical-shell sector seen from an observer at the origin,
with a clustered data catalog and a uniform random catalog) and for
periodic N-body boxes.  Generation is numpy PCG64, split over threads in
fixed chunks so the result depends only on the seed.
"""
import math
from concurrent.futures import ThreadPoolExecutor

import numpy as np

CHUNK = 1 << 22


class Sector:
    """RA in [-ra, ra], Dec in [-dec, dec] about +x, r in [r1, r2]."""

    def __init__(self, r1=500.0, r2=1500.0, ra_deg=30.0, dec_deg=30.0):
        self.r1, self.r2 = float(r1), float(r2)
        self.ra = math.radians(ra_deg)
        self.dec = math.radians(dec_deg)

    def bbox(self):
        """Analytic bounding box (posmin, posmax) of the sector."""
        cmin = math.cos(self.ra) * math.cos(self.dec)
        xmin = self.r1 * cmin
        ymax = self.r2 * math.sin(self.ra)
        zmax = self.r2 * math.sin(self.dec)
        return (np.array([xmin, -ymax, -zmax]), np.array([self.r2, ymax, zmax]))

    def contains(self, p):
        r = np.sqrt(np.sum(p * p, axis=1))
        ra = np.arctan2(p[:, 1], p[:, 0])
        sdec = p[:, 2] / np.maximum(r, 1e-300)
        return ((r >= self.r1) & (r < self.r2) & (np.abs(ra) <= self.ra) &
                (np.abs(sdec) <= math.sin(self.dec)))

    def uniform(self, rng, n, out):
        """n points uniform in volume written into out[:, :3]."""
        u = rng.random((n, 3))
        r = np.cbrt(u[:, 0] * (self.r2 ** 3 - self.r1 ** 3) + self.r1 ** 3)
        ra = (2.0 * u[:, 1] - 1.0) * self.ra
        sdec = (2.0 * u[:, 2] - 1.0) * math.sin(self.dec)
        cdec = np.sqrt(1.0 - sdec * sdec)
        out[:, 0] = r * cdec * np.cos(ra)
        out[:, 1] = r * cdec * np.sin(ra)
        out[:, 2] = r * sdec


def _fill_parallel(n, seed, fill, threads=8):
    """Allocates an (n, 4) array and fills fixed chunks from spawned seeds."""
    out = np.empty((n, 4), dtype=np.float64)
    starts = list(range(0, n, CHUNK))
    seeds = np.random.SeedSequence(seed).spawn(len(starts))

    def work(i):
        s = starts[i]
        e = min(n, s + CHUNK)
        fill(np.random.Generator(np.random.PCG64(seeds[i])), out[s:e])

    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(work, range(len(starts))))
    return out


def sector_randoms(n, seed, sector=None, threads=8):
    """Uniform randoms in the sector with weights U[0.5, 1.5]."""
    sector = sector or Sector()

    def fill(rng, block):
        sector.uniform(rng, block.shape[0], block)
        block[:, 3] = rng.uniform(0.5, 1.5, block.shape[0])

    return _fill_parallel(n, seed, fill, threads)


def sector_clustered(n, seed, ncenters=10000, sigma=5.0, sector=None,
                     threads=8):
    """Gaussian-mixture data: centres uniform in the sector, points at
    centre + N(0, sigma^2 I), redrawn until inside the sector."""
    sector = sector or Sector()
    crng = np.random.Generator(np.random.PCG64(np.random.SeedSequence(seed + 7919)))
    centers = np.empty((ncenters, 4))
    sector.uniform(crng, ncenters, centers)
    centers = centers[:, :3].copy()

    def fill(rng, block):
        m = block.shape[0]
        pts = np.empty((m, 3))
        todo = np.arange(m)
        while todo.size:
            c = centers[rng.integers(0, ncenters, todo.size)]
            p = c + rng.normal(0.0, sigma, (todo.size, 3))
            ok = sector.contains(p)
            pts[todo[ok]] = p[ok]
            todo = todo[~ok]
        block[:, :3] = pts
        block[:, 3] = rng.uniform(0.5, 1.5, m)

    return _fill_parallel(n, seed, fill, threads)


def box_clustered(n, boxsize, seed, ncenters=10000, sigma=5.0, threads=8):
    """Periodic box [0, L)^3: half clustered (wrapped), half uniform; unit
    weights."""
    crng = np.random.Generator(np.random.PCG64(np.random.SeedSequence(seed + 104729)))
    centers = crng.random((ncenters, 3)) * boxsize

    def fill(rng, block):
        m = block.shape[0]
        h = m // 2
        c = centers[rng.integers(0, ncenters, h)]
        block[:h, :3] = np.mod(c + rng.normal(0.0, sigma, (h, 3)), boxsize)
        block[h:, :3] = rng.random((m - h, 3)) * boxsize
        block[:, 3] = 1.0

    return _fill_parallel(n, seed, fill, threads)


def survey_box(sector, sep, ngrid):
    """posmin and cell size the CLI would adopt for the sector's bounding
    box padded by sep/1.5 (cc/fftcorr.cc:335-346)."""
    lo, hi = sector.bbox()
    pad = sep / 1.5
    lo = lo - pad
    hi = hi + pad
    cell = max((hi[i] - lo[i]) / ngrid[i] for i in range(3))
    return lo, cell
