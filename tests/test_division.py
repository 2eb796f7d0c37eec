"""Division by the cell size as the device does it.

Grid coordinates are (p - posmin) / cell.  The mass-assignment kernels form
the quotient from the correctly rounded reciprocal r = 1/cell with one fused
residual correction, q = a*r, q' = fma(a - q*cell, r) + q (Markstein, IBM J.
Res. Dev. 34(1), 1990), which equals the IEEE quotient when |a| and cell lie
in [2^-400, 2^400].  This checks that claim in exact rational arithmetic on
random and near-integer quotients (the GPU-side check is
test_gpu_parity.py::test_cell_faces_match_division).
"""
from fractions import Fraction

import numpy as np


def _fma(x, y, z):
    return float(Fraction(x) * Fraction(y) + Fraction(z))


def _markstein(a, cell, r):
    q = a * r
    return _fma(_fma(-q, cell, a), r, q)


def test_reciprocal_division_equals_ieee_division():
    rng = np.random.default_rng(3)
    cells = [3.450520833333333, 10.0, 25.0, 0.1, 7.0 / 3.0] + list(
        np.exp(rng.uniform(-12, 12, 6)))
    bad = []
    for cell in cells:
        r = 1.0 / cell
        a = np.concatenate([
            rng.uniform(-200, 2000, 1500) * cell,
            rng.integers(0, 5000, 1500) * cell,  # quotients near integers
            np.ldexp(rng.uniform(0.5, 1.0, 1000), rng.integers(-300, 300, 1000)),
        ])
        a = np.concatenate([a, np.nextafter(a[1500:3000], np.inf),
                            np.nextafter(a[1500:3000], -np.inf)])
        for x in a.tolist():
            if _markstein(x, cell, r) != x / cell:
                bad.append((x, cell))
    assert not bad, bad[:5]
