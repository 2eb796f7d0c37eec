"""The `fftcorr` command-line drop-in (fftcorr_b200/bin/fftcorr).

Runs the same command the reference's golden test issues
(test_fftcorr_aniso.py:89-112, fftcorr/fftcorr.py:434-443) on the golden
catalogs and compares the numeric table rows with the golden outputs at the
reference test's tolerance (rtol 1e-7, counts exact); a periodic run is
compared with the oracle.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, clustered_catalog
from oracle import fc_oracle as O

CLI = os.path.join(ROOT, "fftcorr_b200", "bin", "fftcorr")

pytestmark = pytest.mark.gpu


def _write_catalog(path, header, posw):
    with open(path, "wb") as f:
        np.asarray(header, dtype=np.float64).tofile(f)
        np.ascontiguousarray(posw, dtype=np.float64).tofile(f)


@pytest.mark.parametrize("hemi", ["north", "south"])
def test_cli_reproduces_golden_tables(hemi, tmp_path, golden_catalogs,
                                      golden_tables):
    hdr = golden_catalogs[f"{hemi}_header"]
    _write_catalog(tmp_path / "corrDD.dat", hdr, golden_catalogs[f"{hemi}_DD"])
    _write_catalog(tmp_path / "corrRR.dat", hdr, golden_catalogs[f"{hemi}_RR"])
    for name, extra in (("corrDD", ["-in2", "corrRR.dat"]), ("corrRR", [])):
        cmd = [CLI, "-in", f"{name}.dat", "-out", f"{name}.dat.out", "-dr",
               "10.000000", "-n", "256", "-ell", "2", "-r", "200.000000", *extra]
        subprocess.run(cmd, cwd=tmp_path, check=True, capture_output=True)
        tab = np.loadtxt(tmp_path / f"{name}.dat.out")
        gold = golden_tables[f"{hemi}_{name}"]
        np.testing.assert_array_equal(tab[:, 2], gold[:, 2])
        np.testing.assert_allclose(tab, gold, rtol=1e-7)


def test_cli_periodic_matches_oracle(tmp_path):
    box = 500.0
    posw = clustered_catalog(40000, [0, 0, 0], [box] * 3, 17, ncenters=30,
                             sigma=8.0)
    hdr = np.array([0, 0, 0, box, box, box, 0, 0], dtype=np.float64)
    _write_catalog(tmp_path / "box.dat", hdr, posw)
    cmd = [CLI, "-in", "box.dat", "-out", "box.out", "-n", "32", "-p", "-r",
           "60", "-dr", "5", "-kmax", "0.3", "-dk", "0.02", "-ell", "2", "-d",
           "0"]
    subprocess.run(cmd, cwd=tmp_path, check=True, capture_output=True)
    tab = np.loadtxt(tmp_path / "box.out")
    res = O.cli_run([posw], (32, 32, 32), 60.0, 5.0, 0.3, 0.02, 2, 0, True, hdr)
    ref = O.cli_table(res, True)
    np.testing.assert_array_equal(tab[:, :3], ref[:, :3])
    scale = np.max(np.abs(ref[:, 3:]), axis=0)
    assert np.all(np.abs(tab[:, 3:] - ref[:, 3:]) <= 1e-8 * scale + 1e-12)


def test_cli_rejects_bad_arguments(tmp_path):
    r = subprocess.run([CLI, "-nosuchflag"], cwd=tmp_path, capture_output=True)
    assert r.returncode == 1
