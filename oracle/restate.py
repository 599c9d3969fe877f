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
  angular_functions         yasfpy/functions/spherical_functions_trigon.py:11-96 (pi_lm, tau_lm)
  far_field                 yasfpy/functions/cpu_numba.py:536-601 evaluated serially (the reference's
                            parallel loop adds into shared elements), one wavelength
  polarization_components   yasfpy/functions/cpu_numba.py:604-660
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


def angular_functions(lmax: int, theta: np.ndarray):
    """pi_lm(theta), tau_lm(theta), each (lmax+1, lmax+1, n): the normalised angular functions of
    yasfpy/functions/spherical_functions_trigon.py:11-96, by the same recurrences."""
    from math import factorial

    ct = np.cos(np.asarray(theta, dtype=float).ravel())
    st = np.sin(np.asarray(theta, dtype=float).ravel())
    K = ct.size
    plm = np.zeros((lmax + 1, lmax + 1, K))
    pilm = np.zeros_like(plm)
    taulm = np.zeros_like(plm)
    dp0 = np.zeros((lmax + 1, K))  # d/dct of P_l0
    plm[0, 0] = np.sqrt(0.5)
    plm[1, 0] = np.sqrt(1.5) * ct
    dp0[1] = np.sqrt(3.0) * plm[0, 0]
    taulm[1, 0] = -st * dp0[1]
    for l in range(1, lmax):
        plm[l + 1, 0] = (np.sqrt((2 * l + 1) * (2 * l + 3)) * ct * plm[l, 0]
                         - l * np.sqrt((2 * l + 3) / (2 * l - 1)) * plm[l - 1, 0]) / (l + 1)
        dp0[l + 1] = np.sqrt((2 * l + 3) / (2 * l + 1)) * ((l + 1) * plm[l, 0] + ct * dp0[l])
        taulm[l + 1, 0] = -st * dp0[l + 1]
    for m in range(1, lmax + 1):
        c = np.sqrt((2 * m + 1) / 2 / factorial(2 * m)) * np.prod(np.arange(1, 2 * m, 2, dtype=float))
        plm[m, m] = c * st**m
        pilm[m, m] = c * st ** (m - 1)
        taulm[m, m] = m * ct * pilm[m, m]
        for l in range(m, lmax):
            a1 = np.sqrt((2 * l + 1) * (2 * l + 3) / (l + 1 - m) / (l + 1 + m)) * ct
            a2 = np.sqrt((2 * l + 3) * (l - m) * (l + m) / (2 * l - 1) / (l + 1 - m) / (l + 1 + m))
            prev_p = plm[l - 1, m] if l - 1 >= m else 0.0
            prev_pi = pilm[l - 1, m] if l - 1 >= m else 0.0
            plm[l + 1, m] = a1 * plm[l, m] - a2 * prev_p
            pilm[l + 1, m] = a1 * pilm[l, m] - a2 * prev_pi
            taulm[l + 1, m] = ((l + 1) * ct * pilm[l + 1, m]
                               - (l + 1 + m) * np.sqrt((2 * l + 3) * (l + 1 - m) / (2 * l + 1) / (l + 1 + m))
                               * pilm[l, m])
    return pilm, taulm


def far_field(lmax: int, positions: np.ndarray, k: float, coef: np.ndarray, polar: np.ndarray,
              azimuthal: np.ndarray):
    """(E_theta, E_phi) on the sampling directions, each (n,) complex: the sum over every particle s
    and mode n = (tau, l, m) of yasfpy/functions/cpu_numba.py:536-601 for one wavelength, with
    coef (N, nmax) the scattered-field coefficients."""
    polar = np.asarray(polar, dtype=float).ravel()
    azimuthal = np.asarray(azimuthal, dtype=float).ravel()
    pilm, taulm = angular_functions(lmax, polar)
    e_r = np.stack((np.sin(polar) * np.cos(azimuthal), np.sin(polar) * np.sin(azimuthal), np.cos(polar)), axis=1)
    phase = np.exp(-1j * k * (np.asarray(positions) @ e_r.T))  # (N, A)
    nmax = 2 * lmax * (lmax + 2)
    e_theta = np.zeros(polar.size, dtype=complex)
    e_phi = np.zeros_like(e_theta)
    for n in range(nmax):
        tau = 1 if n < nmax // 2 else 2
        rem = n - (tau - 1) * (nmax // 2)
        l = int(np.floor(np.sqrt(rem + 1)))
        m = rem + 1 - l * l - l
        t = (1j ** (tau - l - 2)) / np.sqrt(2 * l * (l + 1)) * np.exp(1j * m * azimuthal) \
            * (coef[:, n] @ phase)
        pi_, ta_ = pilm[l, abs(m)], taulm[l, abs(m)]
        if tau == 1:
            e_theta += t * pi_ * 1j * m
            e_phi -= t * ta_
        else:
            e_theta += t * ta_
            e_phi += t * pi_ * 1j * m
    return e_theta, e_phi


def polarization_components(e_theta: np.ndarray, e_phi: np.ndarray):
    """I and the degrees of polarisation (dop, dolp, dolp_q, dolp_u, docp) of the far field
    (yasfpy/functions/cpu_numba.py:604-660)."""
    at, ap = np.abs(e_theta) ** 2, np.abs(e_phi) ** 2
    x = e_theta * np.conj(e_phi)
    I, Q, U, V = at + ap, at - ap, -2 * x.real, 2 * x.imag
    return I, np.sqrt(Q**2 + U**2 + V**2) / I, np.sqrt(Q**2 + U**2) / I, -Q / I, U / I, V / I
