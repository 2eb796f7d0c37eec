"""CPU restatement of the reference fftcorr hot path (FP64, numpy + C).

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` leg of ``bench.py`` may import this module; it is the checker,
never the thing measured or shipped.  The ``fftcorr_b200`` package does not
import it and fails loudly when its CUDA library is missing.

What it restates (reference file:line):

* ``sequence``                 cc/array/array_ops.cc:7-13
* ``grid_coords``              cc/grid/config_space_grid.h:31-46     (C)
* ``mass_assign``              cc/particle_mesh/mass_assignor.h:72-125,
                               cc/particle_mesh/distribution_functions.h:17-236,
                               cc/particle_mesh/d12.h:149-155        (C)
* ``make_ylm``                 cc/correlate/spherical_harmonics.h:32-179
* ``window_squared``           cc/correlate/window_correct.h:14-60
* ``r_subgrid``/``k_subgrid``  cc/correlate/correlator.h:109-205
* ``extract_submatrix``        cc/grid/fft_grid.cc:182-210
* ``extract_fft_submatrix_c2r`` cc/grid/fft_grid.cc:215-258
* ``Histogram``                cc/histogram/histogram_list.h:10-68   (C)
* ``periodic_correlate``       cc/correlate/correlator.h:273-357
* ``survey_correlate``         cc/correlate/correlator.h:381-497 (with the
                               grid2 FFT of correlator.h:47-77)

The 3-D FFTs use numpy's pocketfft in FP64 with FFTW's conventions (forward
sign -1, unnormalised inverse).  Parity pins: ``tests/test_oracle.py`` checks
this module against the compiled reference (``oracle/_ref``) and against the
reference's golden outputs committed under ``tests/golden/``.
"""
import ctypes
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build", "liboracle.so")
_REF = os.path.join(_HERE, "_ref")

NEAREST_CELL, TRIANGULAR_SHAPED_CLOUD, WAVELET, CLOUD_IN_CELL = 0, 1, 2, 3
NO_CORRECTION, TSC_CORRECTION, TSC_ALIASED_CORRECTION = 0, 1, 2

_lib = None


def lib():
    """The oracle's compiled C part (oracle/_build/liboracle.so)."""
    global _lib
    if _lib is None:
        if not os.path.exists(_BUILD):
            raise RuntimeError(
                f"{_BUILD} is missing; run `make -C oracle oracle` first")
        L = ctypes.CDLL(_BUILD)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.fco_grid_coords.argtypes = [dp, dp, ctypes.c_double, ip, ctypes.c_int, dp]
        L.fco_grid_coords.restype = ctypes.c_int
        L.fco_mass_assign.argtypes = [dp, ctypes.c_long, ip, dp, ctypes.c_double,
                                      ctypes.c_int, ctypes.c_int, dp, dp, dp]
        L.fco_mass_assign.restype = ctypes.c_int
        L.fco_cell_index.argtypes = [dp, ctypes.c_long, ip, dp, ctypes.c_double,
                                     ctypes.c_int, ctypes.POINTER(ctypes.c_int64)]
        L.fco_hist_accumulate.argtypes = [ctypes.c_double, ctypes.c_double,
                                          ctypes.c_int, dp, dp, ctypes.c_long,
                                          ip, dp]
        L.fco_bin_index.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                    dp, ctypes.c_long, ip]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def d12_wave():
    """The reference's transposed D12 table (8 taps x 64 sub-cell samples).

    It is read from the compiled reference harness (d12.h:149-155); the
    numbers are reference data and are not restated here.
    """
    path = os.path.join(_REF, "libfcref.so")
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing; run `make -C oracle ref`")
    L = ctypes.CDLL(path)
    out = np.zeros(512, dtype=np.float64)
    L.fcref_d12_table.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.c_int]
    if L.fcref_d12_table(_dp(out), 512) != 0:
        raise RuntimeError("fcref_d12_table failed")
    return out


# --------------------------------------------------------------------------
# Arrays, grids and mass assignment
# --------------------------------------------------------------------------

def sequence(start, step, size):
    """start + i*step for i < size (array_ops.cc:7-13)."""
    return start + np.arange(size, dtype=np.float64) * step


def grid_coords(pos, posmin, cell, shape, periodic):
    """Survey -> grid coordinates, or None when skipped (config_space_grid.h:31-46)."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    posmin = np.ascontiguousarray(posmin, dtype=np.float64)
    shape = np.ascontiguousarray(shape, dtype=np.intc)
    out = np.zeros(3)
    ok = lib().fco_grid_coords(_dp(pos), _dp(posmin), float(cell), _ip(shape),
                               int(bool(periodic)), _dp(out))
    return out if ok else None


def apply_displacement_field(pos, disp, posmin, cell, shape, periodic):
    """out = pos + disp[int(grid coords of pos)] (fftcorr/grid/utils.pyx:21-40);
    None when a position has no cell (the reference raises ValueError)."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    out = np.empty_like(pos)
    for i in range(pos.shape[0]):
        x = grid_coords(pos[i], posmin, cell, shape, periodic)
        if x is None:
            return None
        d = disp[int(x[0]), int(x[1]), int(x[2])]
        for j in range(3):
            out[i, j] = pos[i, j] + d[j]
    return out


def normalise_periodic(grid, totw):
    """The CLI's periodic normalisation (cc/fftcorr.cc:369-375): mean =
    totw / size, then add_scalar(-mean) and multiply_by(1.0 / mean)."""
    mean = totw / grid.size
    out = grid + (-mean)
    return out * (1.0 / mean)


def mass_assign(posw, shape, posmin, cell, scheme, periodic=False, grid=None,
                wave=None):
    """Grid of an (n, 4) posw catalog in input order (buffer_size 0).

    Returns (grid, stats) with stats = [num_added, num_skipped, totw, totwsq].
    ``grid`` may be passed in to accumulate several catalogs.
    """
    posw = np.ascontiguousarray(posw, dtype=np.float64)
    if posw.ndim != 2 or posw.shape[1] != 4:
        raise ValueError("posw must have shape (n, 4)")
    shape = tuple(int(s) for s in shape)
    if grid is None:
        grid = np.zeros(shape, dtype=np.float64)
    stats = np.zeros(4)
    if scheme == WAVELET and wave is None:
        wave = d12_wave()
    wave_arr = np.ascontiguousarray(wave if wave is not None else np.zeros(1))
    shp = np.array(shape, dtype=np.intc)
    pm = np.ascontiguousarray(posmin, dtype=np.float64)
    rc = lib().fco_mass_assign(_dp(posw), posw.shape[0], _ip(shp), _dp(pm),
                               float(cell), int(scheme), int(bool(periodic)),
                               _dp(wave_arr), _dp(grid), _dp(stats))
    if rc != 0:
        raise ValueError(f"fco_mass_assign failed ({rc})")
    return grid, stats


def cell_index(posw, shape, posmin, cell, periodic=False):
    posw = np.ascontiguousarray(posw, dtype=np.float64)
    out = np.zeros(posw.shape[0], dtype=np.int64)
    shp = np.array(shape, dtype=np.intc)
    pm = np.ascontiguousarray(posmin, dtype=np.float64)
    lib().fco_cell_index(_dp(posw), posw.shape[0], _ip(shp), _dp(pm), float(cell),
                         int(bool(periodic)),
                         out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
    return out


class Histogram:
    """HistogramList (histogram_list.h:10-68): n rows, floor((max-min)/bin) bins."""

    def __init__(self, n, minval, maxval, binsize):
        if n <= 0:
            raise ValueError("n must be positive.")
        if minval >= maxval:
            raise ValueError("maxval must be greater than minval.")
        if binsize <= 0:
            raise ValueError("binsize must be positive.")
        self.minval = float(minval)
        self.binsize = float(binsize)
        self.nbins = int(math.floor((maxval - minval) / binsize))
        self.bins = self.minval + (np.arange(self.nbins) + 0.5) * self.binsize
        self.counts = np.zeros((n, self.nbins), dtype=np.intc)
        self.hist = np.zeros((n, self.nbins), dtype=np.float64)

    def accumulate(self, ih, x, y):
        if ih >= self.counts.shape[0]:
            raise IndexError("ih out of range.")
        x = np.ascontiguousarray(x, dtype=np.float64).ravel()
        y = np.ascontiguousarray(y, dtype=np.float64).ravel()
        crow = np.ascontiguousarray(self.counts[ih])
        hrow = np.ascontiguousarray(self.hist[ih])
        lib().fco_hist_accumulate(self.minval, self.binsize, self.nbins, _dp(x),
                                  _dp(y), x.size, _ip(crow), _dp(hrow))
        self.counts[ih] = crow
        self.hist[ih] = hrow

    def reset(self):
        self.counts[:] = 0
        self.hist[:] = 0.0


def bin_index(x, minval, binsize, nbins):
    x = np.ascontiguousarray(x, dtype=np.float64).ravel()
    out = np.zeros(x.size, dtype=np.intc)
    lib().fco_bin_index(float(minval), float(binsize), int(nbins), _dp(x), x.size,
                        _ip(out))
    return out


# --------------------------------------------------------------------------
# Spherical harmonics and window functions
# --------------------------------------------------------------------------

def make_ylm(ell, m, xcell, ycell, zcell, coeff, mult=None):
    """Real-form Y_lm on the grid spanned by the axes, times coeff * mult.

    Follows spherical_harmonics.h:32-179 operation by operation (exponent 0,
    the only value the correlators use), so products are rounded in the
    reference's order.
    """
    if ell not in (0, 2, 4):
        raise ValueError("Unsupported ell")
    if m < -ell or m > ell:
        raise ValueError("Illegal (ell, m)")
    x = np.asarray(xcell, dtype=np.float64)[:, None, None]
    y = np.asarray(ycell, dtype=np.float64)[None, :, None]
    z = np.asarray(zcell, dtype=np.float64)[None, None, :]
    shape = (x.shape[0], y.shape[1], z.shape[2])
    D = np.ones(shape) if mult is None else np.asarray(mult, dtype=np.float64)
    if ell == 0:
        value = coeff / math.sqrt(4.0 * math.pi)
        return D * value
    z2 = z * z
    z3 = z2 * z
    z4 = z3 * z
    isqpi = math.sqrt(1.0 / math.pi)
    isqpi *= coeff
    if m != 0:
        isqpi *= math.sqrt(2.0)
    x2 = x * x
    y2 = y * y
    y3 = y2 * y
    y4 = y3 * y
    ir2 = 1.0 / (x2 + y2 + z2 + 1e-20)
    if ell == 2:
        if m == 2:
            return D * isqpi * math.sqrt(15.0 / 32.0) * (x2 - y2) * ir2
        if m == 1:
            return D * isqpi * math.sqrt(15.0 / 8.0) * x * z * ir2
        if m == 0:
            return D * isqpi * math.sqrt(5.0 / 16.0) * (2.0 * z2 - x2 - y2) * ir2
        if m == -1:
            return D * isqpi * math.sqrt(15.0 / 8.0) * y * z * ir2
        return D * isqpi * math.sqrt(15.0 / 8.0) * x * y * ir2
    if m == 4:
        return (D * isqpi * 3.0 / 16.0 * math.sqrt(35.0 / 2.0) *
                (x2 * x2 - 6.0 * x2 * y2 + y4) * ir2 * ir2)
    if m == 3:
        return (D * isqpi * 3.0 / 8.0 * math.sqrt(35.0) * (x2 - 3.0 * y2) * z * x *
                ir2 * ir2)
    if m == 2:
        return (D * isqpi * 3.0 / 8.0 * math.sqrt(5.0 / 2.0) *
                (6.0 * z2 * (x2 - y2) - x2 * x2 + y4) * ir2 * ir2)
    if m == 1:
        return (D * isqpi * 3.0 / 8.0 * math.sqrt(5.0) * 3.0 *
                (4.0 / 3.0 * z2 - x2 - y2) * x * z * ir2 * ir2)
    if m == 0:
        return (D * isqpi * 3.0 / 16.0 * 8.0 *
                (z4 - 3.0 * z2 * (x2 + y2) + 3.0 / 8.0 *
                 (x2 * x2 + 2.0 * x2 * y2 + y4)) * ir2 * ir2)
    if m == -1:
        return (D * isqpi * 3.0 / 8.0 * math.sqrt(5.0) * 3.0 *
                (4.0 / 3.0 * z2 - x2 - y2) * y * z * ir2 * ir2)
    if m == -2:
        return (D * isqpi * 3.0 / 8.0 * math.sqrt(5.0 / 2.0) *
                (2.0 * x * y * (6.0 * z2 - x2 - y2)) * ir2 * ir2)
    if m == -3:
        return (D * isqpi * 3.0 / 8.0 * math.sqrt(35.0) * (3.0 * x2 * y - y3) * z *
                ir2 * ir2)
    return (D * isqpi * 3.0 / 16.0 * math.sqrt(35.0 / 2.0) *
            (4.0 * x * (x2 * y - y3)) * ir2 * ir2)


def _sinc(x):
    return 1.0 if x == 0 else math.sin(x) / x


def window_squared(kind, k, cell):
    """|W(k)|^2 per axis value (window_correct.h:14-44)."""
    if kind == NO_CORRECTION:
        return 1.0
    if kind == TSC_CORRECTION:
        return math.pow(_sinc(k * cell / 2.0), 6)
    if kind == TSC_ALIASED_CORRECTION:
        s = math.sin(k * cell / 2.0)
        s *= s
        return 1 - s + 2.0 / 15.0 * s * s
    raise ValueError(f"unknown window correction {kind}")


# --------------------------------------------------------------------------
# Correlator geometry
# --------------------------------------------------------------------------

class Geometry:
    """r- and k-subgrid axes, norms and window (correlator.h:109-205)."""

    def __init__(self, shape, cell, window, rmax, dr, kmax, dk, maxell):
        self.shape = tuple(int(s) for s in shape)
        self.cell = float(cell)
        rmax_cells = int(math.ceil(rmax / cell))
        sizex = 2 * rmax_cells + 1
        self.rshape = (sizex,) * 3
        minsep = -cell * rmax_cells
        self.rx = sequence(minsep, cell, sizex)
        self.ry = sequence(minsep, cell, sizex)
        self.rz = sequence(minsep, cell, sizex)
        self.rnorm = np.sqrt(self.rx[:, None, None] * self.rx[:, None, None] +
                             self.ry[None, :, None] * self.ry[None, :, None] +
                             self.rz[None, None, :] * self.rz[None, None, :])
        self.rzero = (rmax_cells,) * 3
        k_nyq = math.pi / cell
        kshape = []
        for n in self.shape:
            ks = int(2 * math.ceil(kmax / (2.0 * k_nyq / n)) + 1)
            if ks > n:
                ks = 2 * (n // 2) + 1
            kshape.append(ks)
        self.kshape = tuple(kshape)
        axes = []
        for ks, n in zip(self.kshape, self.shape):
            start = (-(ks // 2)) * 2.0 * k_nyq / n
            axes.append(sequence(start, 2.0 * k_nyq / n, ks))
        self.kx, self.ky, self.kz = axes
        self.knorm = np.sqrt(self.kx[:, None, None] * self.kx[:, None, None] +
                             self.ky[None, :, None] * self.ky[None, :, None] +
                             self.kz[None, None, :] * self.kz[None, None, :])
        wx = np.array([window_squared(window, k, cell) for k in self.kx])
        wy = np.array([window_squared(window, k, cell) for k in self.ky])
        wz = np.array([window_squared(window, k, cell) for k in self.kz])
        self.inv_window = 1.0 / (wx[:, None, None] * wy[None, :, None] *
                                 wz[None, None, :])
        self.nrows = maxell // 2 + 1
        self.maxell = maxell
        self.rhist = Histogram(self.nrows, 0.0, rmax, dr)
        self.khist = Histogram(self.nrows, 0.0, kmax, dk)


def extract_submatrix(grid, oshape):
    """Centred, wrapped real subgrid of an unpadded grid (fft_grid.cc:182-210)."""
    n0, n1, n2 = grid.shape
    idx = [(n - o // 2 + np.arange(o)) % n for n, o in zip(grid.shape, oshape)]
    return grid[np.ix_(*idx)]


def extract_fft_submatrix_c2r(cgrid, oshape):
    """Centred real part of a half-complex grid (fft_grid.cc:215-258)."""
    c0, c1, _ = cgrid.shape
    ox, oy, oz = (o // 2 for o in oshape)
    ii = (c0 - ox + np.arange(oshape[0])) % c0
    jj = (c1 - oy + np.arange(oshape[1])) % c1
    iin = (c0 - ii) % c0
    jjn = (c1 - jj) % c1
    out = np.empty(oshape)
    k = np.arange(oshape[2])
    neg = k < oz
    out[:, :, neg] = cgrid[np.ix_(iin, jjn, oz - k[neg])].real
    out[:, :, ~neg] = cgrid[np.ix_(ii, jj, k[~neg] - oz)].real
    return out


def _rfftn(x):
    return np.fft.rfftn(x)


def _irfftn(c, shape):
    # FFTW's c2r is unnormalised: norm="forward" leaves the inverse unscaled.
    return np.fft.irfftn(c, s=shape, axes=(0, 1, 2), norm="forward")


def _result(geo, zerolag):
    return {
        "rbins": geo.rhist.bins.copy(),
        "rcounts": geo.rhist.counts.copy(),
        "rhist": geo.rhist.hist.copy(),
        "kbins": geo.khist.bins.copy(),
        "kcounts": geo.khist.counts.copy(),
        "khist": geo.khist.hist.copy(),
        "zerolag": zerolag,
    }


def periodic_correlate(grid, cell, window, rmax, dr, kmax, dk, maxell,
                       grid2=None):
    """PeriodicCorrelator auto/cross correlation (correlator.h:273-357)."""
    grid = np.asarray(grid, dtype=np.float64)
    geo = Geometry(grid.shape, cell, window, rmax, dr, kmax, dk, maxell)
    ncells = grid.size
    work = _rfftn(grid)
    g2 = work if grid2 is None else _rfftn(np.asarray(grid2, dtype=np.float64))
    work = work * np.conj(g2)
    k_rescale = cell * cell * cell / ncells
    for ell in range(0, maxell + 1, 2):
        coeff = math.sqrt((4.0 * math.pi) * (2 * ell + 1)) * k_rescale
        kylm = make_ylm(ell, 0, geo.kx, geo.ky, geo.kz, coeff, geo.inv_window)
        ksub = kylm * extract_fft_submatrix_c2r(work, geo.kshape)
        geo.khist.accumulate(ell // 2, geo.knorm, ksub)
    xi = _irfftn(work, grid.shape)
    r_rescale = (1.0 / ncells / ncells)
    zerolag = None
    for ell in range(0, maxell + 1, 2):
        coeff = math.sqrt((4.0 * math.pi) * (2 * ell + 1)) * r_rescale
        rylm = make_ylm(ell, 0, geo.rx, geo.ry, geo.rz, coeff)
        rsub = rylm * extract_submatrix(xi, geo.rshape)
        geo.rhist.accumulate(ell // 2, geo.rnorm, rsub)
        if ell == 0:
            zerolag = float(rsub[geo.rzero])
    return _result(geo, zerolag)


def survey_correlate(grid, cell, posmin, window, rmax, dr, kmax, dk, maxell,
                     grid2=None, terms=None):
    """Correlator (survey, Ylm about the observer) (correlator.h:381-497).

    grid2 None is autocorrelate(grid); otherwise cross_correlate(grid, grid2).
    terms, if given, is the set of (ell, m) loop indices to include (the
    others contribute nothing), for checking a term-sharded correlation.
    """
    grid = np.asarray(grid, dtype=np.float64)
    geo = Geometry(grid.shape, cell, window, rmax, dr, kmax, dk, maxell)
    ncells = grid.size
    g2 = _rfftn(grid if grid2 is None else np.asarray(grid2, dtype=np.float64))
    g2c = np.conj(g2)
    obs = [-p / cell for p in posmin]
    xc = sequence(0.5 - obs[0], 1.0, grid.shape[0])
    yc = sequence(0.5 - obs[1], 1.0, grid.shape[1])
    zc = sequence(0.5 - obs[2], 1.0, grid.shape[2])
    zerolag = None
    term = -1
    for ell in range(0, maxell + 1, 2):
        rsub = np.zeros(geo.rshape)
        ksub = np.zeros(geo.kshape)
        for m in range(-ell, ell + 1):
            term += 1
            if terms is not None and term not in terms:
                continue
            work = _rfftn(make_ylm(ell, m, xc, yc, zc, 1.0, grid))
            work *= g2c
            kylm = make_ylm(ell, m, geo.kx, geo.ky, geo.kz, 4.0 * math.pi,
                            geo.inv_window)
            ksub += kylm * extract_fft_submatrix_c2r(work, geo.kshape)
            xi = _irfftn(work, grid.shape)
            rylm = make_ylm(ell, m, geo.rx, geo.ry, geo.rz,
                            4.0 * math.pi / ncells)
            rsub += rylm * extract_submatrix(xi, geo.rshape)
        geo.rhist.accumulate(ell // 2, geo.rnorm, rsub)
        geo.khist.accumulate(ell // 2, geo.knorm, ksub)
        if ell == 0:
            zerolag = float(rsub[geo.rzero])
    return _result(geo, zerolag)


# --------------------------------------------------------------------------
# CLI-equivalent pipeline (cc/fftcorr.cc:331-448) for the golden catalogs
# --------------------------------------------------------------------------

def read_catalog(path):
    """64-byte header + (n, 4) doubles (cc/catalog_reader.h:16-71)."""
    raw = np.fromfile(path, dtype=np.float64)
    return raw[:8].copy(), raw[8:].reshape(-1, 4).copy()


def cli_box(posmin, posmax, sep, ngrid, periodic):
    """Box padding and cell size chosen by the CLI (cc/fftcorr.cc:335-346)."""
    posmin = np.array(posmin, dtype=np.float64)
    posmax = np.array(posmax, dtype=np.float64)
    if not periodic:
        pad = sep / 1.5
        posmin = posmin - pad
        posmax = posmax + pad
    cell = -123.0
    for i in range(3):
        cell = max(cell, (posmax[i] - posmin[i]) / ngrid[i])
    return posmin, cell


def cli_run(catalogs, ngrid, sep, dsep, kmax, dk, maxell, scheme, periodic,
            header):
    """What `fftcorr -in A [-in2 B] ...` computes, as result dict + grid stats."""
    ngrid = tuple(ngrid)
    posmin, cell = cli_box(header[0:3], header[3:6], sep, ngrid, periodic)
    grid = np.zeros(ngrid)
    stats = np.zeros(4)
    for cat in catalogs:
        _, st = mass_assign(cat, ngrid, posmin, cell, scheme, periodic, grid=grid)
        stats[:2] += st[:2]
        stats[2:] += st[2:]
    if periodic:
        mean = stats[2] / grid.size
        grid += -mean
        grid *= 1.0 / mean
    window = TSC_ALIASED_CORRECTION if scheme == TRIANGULAR_SHAPED_CLOUD else NO_CORRECTION
    if periodic:
        res = periodic_correlate(grid, cell, window, sep, dsep, kmax, dk, maxell)
    else:
        res = survey_correlate(grid, cell, posmin, window, sep, dsep, kmax, dk,
                               maxell)
    res["cell"] = cell
    res["posmin"] = posmin
    res["stats"] = stats
    return res


def cli_table(res, periodic):
    """Numeric rows as printed by print_hist (cc/fftcorr.cc:213-228)."""
    rows = []
    for prefix, b, c, h, norm in ((1, res["kbins"], res["kcounts"], res["khist"], True),
                                  (0, res["rbins"], res["rcounts"], res["rhist"],
                                   periodic)):
        for j in range(b.size):
            count = float(c[0, j])
            denom = count if (norm and count != 0) else 1.0
            rows.append([prefix, b[j], count] + list(h[:, j] / denom))
    return np.array(rows)
