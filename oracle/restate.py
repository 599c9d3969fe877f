"""ORACLE — TEST INFRASTRUCTURE ONLY. numpy restatements + ctypes access to ``cpu_ref.c``.

Used by ``tests/`` and ``__graft_entry__.smoke()`` (as the parity reference) and the CPU
baseline leg of ``bench.py`` (timed). Nothing here is imported by the product package.

Functions and the reference code they restate:
  coupling_matvec_rows      yasfpy/functions/cpu_numba.py:22-95 via cpu_ref.c (and the near-field
                            pair selection of yasfpy/coupling/backends.py:259-459)
  scattering_bilinear_rows  yasfpy/functions/cpu_numba.py:410-457 via cpu_ref.c
  sph_bessel                yasfpy/functions/misc.py:183-193 (SciPy spherical_jn / spherical_yn)
  legendre                  yasfpy/functions/legendre_normalized_trigon.py:12-95
  master_matvec             yasfpy/matrix_apply.py:66-120
  scipy_gmres_solve         yasfpy/scattered_field_coefficients.py:95-144 + yasfpy/solver.py:108-121
  block_matrix              (I - T W)[B, B] column by column from master_matvec, the preconditioner
                            pin (yasfpy/preconditioner.py:92-175 cannot build multi-sphere blocks)
  reference_translation_table  the reference's own Numerics.translation_ab5 (yasfpy/numerics.py:187-281)
                            for lmax 1-8, as generated by tests/golden/make_golden.py
"""

from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from oracle.build import build

_lib = None

GOLDEN = Path(__file__).resolve().parents[1] / "tests" / "golden"


def reference_translation_table(lmax: int) -> np.ndarray:
    """The a5/b5 table computed by the reference itself (committed fixtures), indexed
    [n_source, n_receiver, p] as particle_interaction_scalar reads it."""
    name = "ref_translation.npz" if lmax <= 6 else "ref_translation_l78.npz"
    with np.load(GOLDEN / name) as z:
        return np.ascontiguousarray(z[f"lmax{lmax}"], dtype=np.complex128)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        path = build()
        L = ctypes.CDLL(str(path))
        dp = ctypes.POINTER(ctypes.c_double)
        L.oracle_sph_bessel.argtypes = [ctypes.c_int, ctypes.c_double, dp, dp]
        L.oracle_legendre.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, dp]
        L.oracle_coupling_matvec.argtypes = [ctypes.c_int, ctypes.c_int, dp, ctypes.c_double, dp, dp,
                                             ctypes.c_int, ctypes.c_int, dp, ctypes.c_int]
        L.oracle_coupling_matvec_cutoff.argtypes = [ctypes.c_int, ctypes.c_int, dp, ctypes.c_double, dp, dp,
                                                    ctypes.c_int, ctypes.c_int, dp, ctypes.c_int,
                                                    ctypes.c_double]
        L.oracle_scattering_bilinear.argtypes = [ctypes.c_int, ctypes.c_int, dp, ctypes.c_double, dp,
                                                 dp, ctypes.c_int, ctypes.c_int, dp, ctypes.c_int]
        L.oracle_max_threads.argtypes = []
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def max_threads() -> int:
    return int(lib().oracle_max_threads())


def sph_bessel(pmax: int, x: float):
    j = np.zeros(pmax + 1)
    y = np.zeros(pmax + 1)
    lib().oracle_sph_bessel(pmax, float(x), _dp(j), _dp(y))
    return j, y


def legendre(lmax: int, ct: float, st: float) -> np.ndarray:
    out = np.zeros((lmax + 1) * (lmax + 1))
    lib().oracle_legendre(lmax, float(ct), float(st), _dp(out))
    return out.reshape(lmax + 1, lmax + 1)


def coupling_matvec_rows(lmax: int, positions: np.ndarray, k: float, table: np.ndarray, x: np.ndarray,
                         s1_begin: int = 0, s1_end: int | None = None, threads: int = 0,
                         near_field_radius: float | None = None) -> np.ndarray:
    """(W x) for receiving particles [s1_begin, s1_end), flattened particle-major. With
    near_field_radius, only pairs at most that far apart contribute (the near-field pairs of
    yasfpy/coupling/backends.py:259-459)."""
    pos = np.ascontiguousarray(positions, dtype=np.float64)
    N = pos.shape[0]
    s1_end = N if s1_end is None else s1_end
    nmax = 2 * lmax * (lmax + 2)
    tab = np.ascontiguousarray(table, dtype=np.complex128)
    xv = np.ascontiguousarray(x, dtype=np.complex128).reshape(-1)
    out = np.zeros((s1_end - s1_begin) * nmax, dtype=np.complex128)
    cutoff2 = -1.0 if near_field_radius is None else float(near_field_radius) ** 2
    lib().oracle_coupling_matvec_cutoff(lmax, N, _dp(pos), float(k), _dp(tab.view(np.float64)),
                                        _dp(xv.view(np.float64)), s1_begin, s1_end,
                                        _dp(out.view(np.float64)), threads, cutoff2)
    return out


def scattering_bilinear_rows(lmax: int, positions: np.ndarray, k: float, table: np.ndarray,
                             b: np.ndarray, s1_begin: int = 0, s1_end: int | None = None,
                             threads: int = 0) -> complex:
    pos = np.ascontiguousarray(positions, dtype=np.float64)
    N = pos.shape[0]
    s1_end = N if s1_end is None else s1_end
    tab = np.ascontiguousarray(table, dtype=np.complex128)
    bv = np.ascontiguousarray(b, dtype=np.complex128).reshape(-1)
    out = np.zeros(2)
    lib().oracle_scattering_bilinear(lmax, N, _dp(pos), float(k), _dp(tab.view(np.float64)),
                                     _dp(bv.view(np.float64)), s1_begin, s1_end, _dp(out), threads)
    return complex(out[0], out[1])


def master_matvec(lmax, positions, k, table, tmat_flat, x, threads: int = 0) -> np.ndarray:
    wx = coupling_matvec_rows(lmax, positions, k, table, x, threads=threads)
    return np.asarray(x).reshape(-1) - np.asarray(tmat_flat).reshape(-1) * wx


def scipy_gmres_solve(lmax, positions, k, table, tmat_flat, rhs, rtol=1e-8, restart=100,
                      maxiter=1000, x0=None):
    """The reference solve path: SciPy GMRES on (I - T W), x0 = rhs, atol = 0."""
    from scipy.sparse.linalg import LinearOperator, gmres

    n = rhs.size
    op = LinearOperator((n, n), matvec=lambda v: master_matvec(lmax, positions, k, table, tmat_flat, v),
                        dtype=complex)
    x0 = rhs.copy() if x0 is None else x0
    x, info = gmres(op, rhs, x0, rtol=rtol, atol=0, restart=restart, maxiter=maxiter)
    return x, info


def block_matrix(lmax, positions, k, table, tmat_flat, block: np.ndarray) -> np.ndarray:
    """(I - T W)[B, B] in the block's particle order, particle-major, from master_matvec."""
    nmax = 2 * lmax * (lmax + 2)
    N = positions.shape[0]
    idx = (np.asarray(block)[:, None] * nmax + np.arange(nmax)[None, :]).ravel()
    M = np.zeros((idx.size, idx.size), dtype=complex)
    for c, gi in enumerate(idx):
        e = np.zeros(N * nmax, dtype=complex)
        e[gi] = 1.0
        M[:, c] = master_matvec(lmax, positions, k, table, tmat_flat, e)[idx]
    return M
