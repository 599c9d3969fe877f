"""Exact Wigner 3j symbols and the a5/b5 VSWF translation table.

The reference obtains 3j symbols from the third-party WIGXJPF library through ``pywigxjpf``
(yasfpy/numerics.py:16, 219-275), which evaluates them exactly by prime factorisation. This module
evaluates the Racah formula in exact integer arithmetic (Python ints / ``fractions``) and rounds
once to float64, so every nonzero symbol is correctly rounded.
"""

from __future__ import annotations

import math
from fractions import Fraction
from functools import lru_cache

import numpy as np

_f = math.factorial


@lru_cache(maxsize=None)
def wigner_3j(j1: int, j2: int, j3: int, m1: int, m2: int, m3: int) -> float:
    """Wigner 3j symbol (j1 j2 j3; m1 m2 m3) for integer arguments, correctly rounded."""
    if m1 + m2 + m3 != 0:
        return 0.0
    if j3 < abs(j1 - j2) or j3 > j1 + j2:
        return 0.0
    if abs(m1) > j1 or abs(m2) > j2 or abs(m3) > j3:
        return 0.0
    if (j1 + j2 + j3) % 2 == 1 and m1 == 0 and m2 == 0 and m3 == 0:
        return 0.0
    # Racah: sum over k with all factorial arguments non-negative.
    kmin = max(0, j2 - j3 - m1, j1 - j3 + m2)
    kmax = min(j1 + j2 - j3, j1 - m1, j2 + m2)
    s = Fraction(0)
    for k in range(kmin, kmax + 1):
        den = (
            _f(k)
            * _f(j3 - j2 + k + m1)
            * _f(j3 - j1 + k - m2)
            * _f(j1 + j2 - j3 - k)
            * _f(j1 - k - m1)
            * _f(j2 - k + m2)
        )
        s += Fraction((-1) ** k, den)
    if s == 0:
        return 0.0
    pref2 = Fraction(
        _f(j1 + j2 - j3) * _f(j1 - j2 + j3) * _f(-j1 + j2 + j3),
        _f(j1 + j2 + j3 + 1),
    ) * (
        _f(j1 + m1) * _f(j1 - m1) * _f(j2 + m2) * _f(j2 - m2) * _f(j3 + m3) * _f(j3 - m3)
    )
    v2 = s * s * pref2  # exact square of the symbol
    sign = (-1) ** ((j1 - j2 - m3) % 2) * (1 if s > 0 else -1)
    return sign * _sqrt_fraction(v2)


def _sqrt_fraction(v: Fraction, bits: int = 96) -> float:
    """sqrt of a positive rational, accurate far beyond float64 before the final rounding."""
    num, den = v.numerator, v.denominator
    # sqrt(num/den) = isqrt(num * 2^(2h) / den) / 2^h, with h chosen so the integer root carries
    # at least `bits` significant bits.
    half = bits + max(0, (den.bit_length() - num.bit_length()) // 2 + 1)
    root = math.isqrt((num << (2 * half)) // den)
    return float(Fraction(root, 1 << half))


def single_index2multi(n: int, lmax: int) -> tuple[int, int, int]:
    """(tau, l, m) of a per-particle mode index (yasfpy/functions/misc.py:47-67)."""
    per_tau = lmax * (lmax + 2)
    tau = n // per_tau + 1
    q = n % per_tau
    l = math.isqrt(q + 1)
    m = q - (l * l + l - 1)
    return tau, l, m


def translation_table_ab5(lmax: int) -> np.ndarray:
    """The a5/b5 translation table of yasfpy/numerics.py:187-281, exactly evaluated.

    Returns a complex128 array (nmax, nmax, 2*lmax+1) indexed [j1, j2, p] with
    (tau1, l1, m1) = mode(j1), (tau2, l2, m2) = mode(j2):

    - tau1 == tau2 (a5): i^(|m1-m2|-|m1|-|m2|+l2-l1+p) (-1)^(m1-m2)
      sqrt((2l1+1)(2l2+1) / (2 l1(l1+1) l2(l2+1))) (l1(l1+1)+l2(l2+1)-p(p+1)) sqrt(2p+1)
      3j(l1 l2 p; m1 -m2 m2-m1) 3j(l1 l2 p; 0 0 0)
    - tau1 != tau2, p > 0 (b5): same phase and normalisation times
      sqrt((l1+l2+1+p)(l1+l2+1-p)(p+l1-l2)(p-l1+l2)(2p+1))
      3j(l1 l2 p; m1 -m2 m2-m1) 3j(l1 l2 p-1; 0 0 0)
    """
    nmax = 2 * lmax * (lmax + 2)
    P = 2 * lmax + 1
    out = np.zeros((nmax, nmax, P), dtype=np.complex128)
    modes = [single_index2multi(n, lmax) for n in range(nmax)]
    ipow = [1.0 + 0j, 1j, -1.0 + 0j, -1j]
    for j1, (tau1, l1, m1) in enumerate(modes):
        for j2, (tau2, l2, m2) in enumerate(modes):
            norm = math.sqrt((2 * l1 + 1) * (2 * l2 + 1) / (2 * l1 * (l1 + 1) * l2 * (l2 + 1)))
            sgn = -1.0 if (m1 - m2) % 2 else 1.0
            for p in range(P):
                w_m = wigner_3j(l1, l2, p, m1, -m2, -m1 + m2)
                if w_m == 0.0:
                    continue
                phase = ipow[(abs(m1 - m2) - abs(m1) - abs(m2) + l2 - l1 + p) % 4]
                if tau1 == tau2:
                    w0 = wigner_3j(l1, l2, p, 0, 0, 0)
                    if w0 == 0.0:
                        continue
                    val = (
                        sgn
                        * norm
                        * (l1 * (l1 + 1) + l2 * (l2 + 1) - p * (p + 1))
                        * math.sqrt(2 * p + 1)
                        * w_m
                        * w0
                    )
                elif p > 0:
                    w0 = wigner_3j(l1, l2, p - 1, 0, 0, 0)
                    if w0 == 0.0:
                        continue
                    rad = (l1 + l2 + 1 + p) * (l1 + l2 + 1 - p) * (p + l1 - l2) * (p - l1 + l2) * (2 * p + 1)
                    if rad <= 0:
                        continue
                    val = sgn * norm * math.sqrt(rad) * w_m * w0
                else:
                    continue
                out[j1, j2, p] = phase * val
    return out
