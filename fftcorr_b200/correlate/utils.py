"""xi_ell from the NN and RR multipoles: the boundary correction of
Slepian & Eisenstein (2015), eqs. 8-10.

Same contract as the reference's compute_xi (fftcorr/correlate/utils.py:56-69):
inputs are [num_s, num_ell] multipole arrays (ell = 0, 2, 4, ...) of NN and RR;
f_j = RR_j / RR_0, the raw xi is NN / RR_0, and for every separation bin the
linear system (I + M) xi = xi_raw is solved with
M[k, l] = (2k' + 1) * sum_{j >= 2, even} (l' j k'; 0 0 0)^2 f_j,
k' = 2k, l' = 2l.  This is host-side numpy work of negligible cost.
"""
import math

import numpy as np


def wigner3j_000(j1, j2, j3):
    """Wigner 3j symbol (j1 j2 j3; 0 0 0) from the closed-form expression.

    Zero unless J = j1 + j2 + j3 is even and the triangle rule holds; then
    (-1)^g sqrt[(J-2j1)!(J-2j2)!(J-2j3)!/(J+1)!] g!/((g-j1)!(g-j2)!(g-j3)!)
    with g = J/2.
    """
    J = j1 + j2 + j3
    if J % 2:
        return 0.0
    if j1 + j2 < j3 or j2 + j3 < j1 or j3 + j1 < j2:
        return 0.0
    g = J // 2
    f = math.factorial
    num = f(J - 2 * j1) * f(J - 2 * j2) * f(J - 2 * j3)
    root = math.sqrt(num / f(J + 1))
    comb = f(g) // (f(g - j1) * f(g - j2) * f(g - j3))
    return (-1) ** g * root * comb


def coupling_matrix(f):
    """I + M for one separation bin, f = [f_0, f_2, f_4, ...] (f_0 unused)."""
    n = len(f)
    A = np.identity(n)
    for k in range(n):
        for l in range(n):
            s = 0.0
            for j in range(1, n):
                s += wigner3j_000(2 * l, 2 * j, 2 * k) ** 2 * f[j]
            A[k, l] += (4 * k + 1) * s
    return A


def compute_xi(hist_corrNN, hist_corrRR):
    """Anisotropic 2PCF multipoles from the NN and RR multipole moments."""
    NN = np.asarray(hist_corrNN, dtype=np.float64)
    RR = np.asarray(hist_corrRR, dtype=np.float64)
    fRR = RR / RR[:, [0]]
    xi_raw = NN / RR[:, [0]]
    xi = np.zeros_like(xi_raw)
    for s in range(xi_raw.shape[0]):
        xi[s] = np.linalg.solve(coupling_matrix(fRR[s]), xi_raw[s])
    return xi
