"""Fixed small workloads for profiling the library's kernels.

    python -m fftcorr_b200.cases survey   [--ngrid 512] [--precision fp32] [--runs 1]
    python -m fftcorr_b200.cases periodic [--ngrid 384]
    python -m fftcorr_b200.cases batch
    python -m fftcorr_b200.cases assign   [--n 2e7]

survey: a survey Correlator (ell <= 4, rmax 200 / dr 5, kmax 0.3 / dk
0.005, the benchmark's geometry) autocorrelating a seeded random device
grid of the same precision (FP32 cells for fp32), once to warm up and then
--runs times.  periodic: a PeriodicCorrelator
(ell <= 2) on a seeded random grid, FP32 then FP64, two runs each.  batch:
six periodic boxes (128^3, 192^3, 256^3; 1M clustered particles each) in one
CUDA graph, run twice.  assign: TSC mass assignment of seeded uniform
sector randoms onto the benchmark's 512^3 grid (FP32 cells for fp32, the
FP32-mixed form's grids).

Each case holds a few GB of device memory at most, with inputs larger than
the 126 MB L2, so per-kernel DRAM figures are meaningful.  Everything goes
through the public API; nothing here is used by the library itself.
"""
import argparse

import numpy as np


def _survey(a):
    import fftcorr_b200 as fb
    from fftcorr_b200 import _lib, mocks
    from fftcorr_b200.correlate import TSC_ALIASED_CORRECTION
    shape = (a.ngrid,) * 3
    posmin, cell = mocks.survey_box(mocks.Sector(), 200.0, shape)
    grid = fb.ConfigSpaceGrid.from_geometry(shape, posmin, cell, precision=a.precision)
    host = np.random.default_rng(1).standard_normal(shape)
    _lib.call("fc_grid_upload", grid.handle, _lib.dptr(host))
    del host
    c = fb.Correlator(shape, cell, posmin, TSC_ALIASED_CORRECTION, 200.0, 5.0, 0.3,
                      0.005, 4, precision=a.precision)
    for _ in range(1 + a.runs):
        c.autocorrelate(grid)


def _periodic(a):
    import fftcorr_b200 as fb
    from fftcorr_b200 import _lib
    shape = (a.ngrid,) * 3
    cell = 1000.0 / a.ngrid
    grid = fb.ConfigSpaceGrid.from_geometry(shape, np.zeros(3), cell)
    host = np.random.default_rng(2).standard_normal(shape)
    _lib.call("fc_grid_upload", grid.handle, _lib.dptr(host))
    del host
    for precision in ("fp32", "fp64"):
        c = fb.PeriodicCorrelator(shape, cell, 0, 200.0, 5.0, 0.3, 0.005, 2,
                                  precision=precision)
        for _ in range(2):
            c.autocorrelate(grid)


def _batch(a):
    from fftcorr_b200 import batch, mocks
    boxes = []
    for i in range(6):
        n = (128, 192, 256)[i % 3]
        boxes.append(((n, n, n), 1000.0 / n, mocks.box_clustered(1_000_000, 1000.0, 10 + i)))
    b = batch.PeriodicBatch(boxes, rmax=200.0, dr=5.0, kmax=0.1, dk=0.005, maxell=2,
                            precision="fp32", tune=False)
    for _ in range(2):
        b.run()


def _assign(a):
    import fftcorr_b200 as fb
    from fftcorr_b200 import mocks
    sector = mocks.Sector()
    shape = (512,) * 3
    posmin, cell = mocks.survey_box(sector, 200.0, shape)
    R = mocks.sector_randoms(int(a.n), 3, sector=sector)
    grid = fb.ConfigSpaceGrid.from_geometry(shape, posmin, cell, precision=a.precision)
    ma = fb.MassAssignor(grid, fb.DistributionScheme.TRIANGULAR_SHAPED_CLOUD, False, 0)
    ma.add_particles(R)


CASES = {"survey": _survey, "periodic": _periodic, "batch": _batch, "assign": _assign}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("case", choices=sorted(CASES))
    ap.add_argument("--ngrid", type=int, default=None)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--runs", type=int, default=1)
    ap.add_argument("--n", type=float, default=2e7)
    a = ap.parse_args(argv)
    if a.ngrid is None:
        a.ngrid = 384 if a.case == "periodic" else 512
    CASES[a.case](a)
    print(f"case {a.case} done")


if __name__ == "__main__":
    main()
