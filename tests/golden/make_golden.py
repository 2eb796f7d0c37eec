"""Writes the golden fixtures under tests/golden/ from the reference's own
test data (run in a checkout where the reference tree is available).

    python tests/golden/make_golden.py [REFERENCE_ROOT]

Inputs (reference test_data, as used by test_fftcorr_aniso.py:89-134):
  test_data/{north,south}/corrDD.dat, corrRR.dat      binary catalogs
  test_data/{north,south}/nonperiodic/corr{DD,RR}.dat.out   golden P/xi tables
  test_data/{north,south}/nonperiodic/xi.txt          golden compute_xi output
Outputs:
  catalogs.npz  {hemi}_header (8 doubles), {hemi}_DD, {hemi}_RR ((n, 4) posw)
  tables.npz    {hemi}_corrDD, {hemi}_corrRR (numeric rows of the .out files),
                {hemi}_xi (xi.txt)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root):
    cats = {}
    tabs = {}
    for hemi in ("north", "south"):
        base = os.path.join(ref_root, "test_data", hemi)
        for name in ("DD", "RR"):
            raw = np.fromfile(os.path.join(base, f"corr{name}.dat"), dtype=np.float64)
            cats[f"{hemi}_header"] = raw[:8]
            cats[f"{hemi}_{name}"] = raw[8:].reshape(-1, 4)
            tabs[f"{hemi}_corr{name}"] = np.loadtxt(
                os.path.join(base, "nonperiodic", f"corr{name}.dat.out"))
        tabs[f"{hemi}_xi"] = np.loadtxt(os.path.join(base, "nonperiodic", "xi.txt"))
    np.savez_compressed(os.path.join(HERE, "catalogs.npz"), **cats)
    np.savez_compressed(os.path.join(HERE, "tables.npz"), **tabs)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FFTCORR_REFERENCE")
    if not ref:
        sys.exit("usage: make_golden.py REFERENCE_TREE (or set FFTCORR_REFERENCE)")
    main(ref)
