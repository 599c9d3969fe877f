"""CPU check of the factored translation used by the coupling kernels.

The kernels evaluate (W x)[s1, n1] = sum_{s2 != s1} sum_{p, m2} G_{12}[p, m2 - m1] V_{s2}[n1; p, m2]
with the pair factor G = P~_p^{|m2-m1|}(cos theta) h_p(k r) e^{i (m2-m1) phi} and the source factor
V = sum_{tau2, l2} A[(tau2,l2,m2), n1, p] x[s2, (tau2, l2, m2)]. This test evaluates that
factored sum in numpy and compares it with the oracle (the reference's direct four-deep loop)
and with the reference's own output.
"""

from __future__ import annotations

import numpy as np
from conftest import rel_err

from oracle import restate as R
from yasf_b200.wigner import single_index2multi


def factored_matvec(lmax, pos, k, table, x):
    nmax = 2 * lmax * (lmax + 2)
    P = 2 * lmax
    N = pos.shape[0]
    modes = [single_index2multi(n, lmax) for n in range(nmax)]
    X = x.reshape(N, nmax)
    # source factor V[s2, n1, p, m2 + lmax]
    V = np.zeros((N, nmax, P + 1, 2 * lmax + 1), dtype=complex)
    for n1 in range(nmax):
        for n2, (_, _, m2) in enumerate(modes):
            for p in range(P + 1):
                a = table[n2, n1, p]
                if a != 0:
                    V[:, n1, p, m2 + lmax] += a * X[:, n2]
    y = np.zeros((N, nmax), dtype=complex)
    for s1 in range(N):
        for s2 in range(N):
            if s1 == s2:
                continue
            d = pos[s1] - pos[s2]
            r = np.linalg.norm(d)
            ct = np.clip(d[2] / r, -1, 1)
            st = np.sqrt(1 - ct * ct)
            phi = np.arctan2(d[1], d[0])
            j, yv = R.sph_bessel(P, k * r)
            h = j + 1j * yv
            leg = R.legendre(P, ct, st)
            for n1, (_, _, m1) in enumerate(modes):
                acc = 0j
                for m2 in range(-lmax, lmax + 1):
                    dm = abs(m2 - m1)
                    ph = np.exp(1j * (m2 - m1) * phi)
                    for p in range(dm, P + 1):
                        acc += leg[p, dm] * h[p] * ph * V[s2, n1, p, m2 + lmax]
                y[s1, n1] += acc
    return y.ravel()


def test_factored_form_matches_reference(golden):
    g = golden("ref_matvec_l3.npz")
    tab = golden("ref_translation.npz")["lmax3"]
    k = 2 * np.pi / float(g["wavelength"])
    y = factored_matvec(3, g["positions"], k, tab, g["x"])
    assert rel_err(y, g["wx"]) < 1e-12
    yo = R.coupling_matvec_rows(3, g["positions"], k, tab, g["x"])
    assert rel_err(y, yo) < 1e-12
