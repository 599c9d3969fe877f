"""Stand-in for the third-party ``pywigxjpf`` module (WIGXJPF 1.13.3), TEST ONLY.

The upstream reference calls ``wig_table_init``, ``wig_temp_init``, ``wig3jj_array``,
``wig_table_free`` and ``wig_temp_free`` (yasfpy/numerics.py:219-275). WIGXJPF
evaluates Wigner 3j symbols exactly by prime factorisation; this stand-in evaluates
them exactly with ``sympy.physics.wigner.wigner_3j`` (rational arithmetic), an
implementation independent of the product's own Racah-formula evaluator.

Arguments follow WIGXJPF's convention: every angular momentum and projection is
passed doubled (``2j1, 2j2, 2j3, 2m1, 2m2, 2m3``).
"""

from functools import lru_cache

from sympy import Rational
from sympy.physics.wigner import wigner_3j


def wig_table_init(max_two_j, wigner_type):  # noqa: D103 - API stand-in
    return None


def wig_temp_init(max_two_j):  # noqa: D103
    return None


def wig_table_free():  # noqa: D103
    return None


def wig_temp_free():  # noqa: D103
    return None


@lru_cache(maxsize=None)
def _w3j(tj1, tj2, tj3, tm1, tm2, tm3):
    return float(
        wigner_3j(
            Rational(tj1, 2),
            Rational(tj2, 2),
            Rational(tj3, 2),
            Rational(tm1, 2),
            Rational(tm2, 2),
            Rational(tm3, 2),
        )
    )


def wig3jj_array(args):
    """Wigner 3j symbol from six doubled quantum numbers."""
    a = [int(round(float(v))) for v in args]
    return _w3j(*a)


def wig3jj(tj1, tj2, tj3, tm1, tm2, tm3):
    return _w3j(int(tj1), int(tj2), int(tj3), int(tm1), int(tm2), int(tm3))
