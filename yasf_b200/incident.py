"""Plane-wave incident-field VSWF coefficients (yasfpy/initial_field_coefficients.py:79-142).

``spherical_functions_trigon`` restates yasfpy/functions/spherical_functions_trigon.py:11-96 and
``transformation_coefficients`` restates yasfpy/functions/misc.py:70-114 (one mode, one incidence;
kept for the host tests). ``plane_wave_mode_factors`` evaluates the same coefficients for R
incidences at once (vectorised over incidences); ``plane_wave_block`` forms the host block from them,
and ``CouplingDevice.plane_wave_rhs`` the same block and the right-hand sides on the device.
"""

from __future__ import annotations

import math

import numpy as np


def spherical_functions_trigon(lmax: int, ct, st):
    ct = np.atleast_1d(np.asarray(ct, dtype=float)).ravel()
    st = np.atleast_1d(np.asarray(st, dtype=float)).ravel()
    K = ct.shape[0]
    plm = np.zeros((lmax + 1, lmax + 1, K))
    pilm = np.zeros_like(plm)
    taulm = np.zeros_like(plm)
    pp0 = np.zeros((lmax + 1, K))
    plm[0, 0] = np.sqrt(1 / 2)
    if lmax >= 1:
        plm[1, 0] = np.sqrt(3 / 2) * ct
        pp0[1] = np.sqrt(3) * plm[0, 0]
        taulm[1, 0] = -st * pp0[1]
    for l in range(1, lmax):
        plm[l + 1, 0] = (1 / (l + 1) * np.sqrt((2 * l + 1) * (2 * l + 3)) * ct * plm[l, 0]
                         - l / (l + 1) * np.sqrt((2 * l + 3) / (2 * l - 1)) * plm[l - 1, 0])
        pp0[l + 1] = np.sqrt((2 * l + 3) / (2 * l + 1)) * ((l + 1) * plm[l, 0] + ct * pp0[l])
        taulm[l + 1, 0] = -st * pp0[l + 1]
    for m in range(1, lmax + 1):
        coeff = np.sqrt((2 * m + 1) / 2 / math.factorial(2 * m)) * np.prod(np.arange(1, 2 * m, 2))
        plm[m, m] = coeff * np.power(st, m)
        pilm[m, m] = coeff * np.power(st, m - 1)
        taulm[m, m] = m * ct * pilm[m, m]
        for l in range(m, lmax):
            c1 = np.sqrt((2 * l + 1) * (2 * l + 3) / (l + 1 - m) / (l + 1 + m)) * ct
            c2 = np.sqrt((2 * l + 3) * (l - m) * (l + m) / (2 * l - 1) / (l + 1 - m) / (l + 1 + m))
            plm[l + 1, m] = c1 * plm[l, m] - c2 * plm[l - 1, m]
            pilm[l + 1, m] = c1 * pilm[l, m] - c2 * pilm[l - 1, m]
            taulm[l + 1, m] = (l + 1) * ct * pilm[l + 1, m] - (l + 1 + m) * np.sqrt(
                (2 * l + 3) * (l + 1 - m) / (2 * l + 1) / (l + 1 + m)) * pilm[l, m]
    return pilm, taulm


def transformation_coefficients(pilm, taulm, tau, l, m, pol, dagger: bool = False):
    ifac = -1j if dagger else 1j
    if pol in (1, 2):
        spher = taulm[l, abs(m)] if tau == pol else m * pilm[l, abs(m)]
        return (-1 / np.power(ifac, l + 1) / np.sqrt(2 * l * (l + 1))
                * (ifac * (pol == 1) + (pol == 2)) * spher)
    return (-1 / np.power(ifac, l + 1) / np.sqrt(2 * l * (l + 1)) * (ifac + 1)
            * (taulm[l, abs(m)] + m * pilm[l, abs(m)]) / 2)


def mode_index(lmax: int, tau: int, l: int, m: int) -> int:
    return (tau - 1) * lmax * (lmax + 2) + (l - 1) * (l + 1) + l + m


def plane_wave_mode_factors(lmax: int, polar, azimuthal, pol, amplitude: float = 1.0) -> np.ndarray:
    """coef[r, n] = 4 E0 e^{-i m alpha_r} B^dagger_{tau l m}(beta_r): the sphere-independent factor
    of the plane-wave coefficients of incidence r (yasfpy/initial_field_coefficients.py:79-142),
    (R, nmax) complex128. Vectorised over incidences: one pass over the nmax modes."""
    polar = np.atleast_1d(np.asarray(polar, dtype=float))
    azimuthal = np.atleast_1d(np.asarray(azimuthal, dtype=float))
    pol = np.atleast_1d(np.asarray(pol, dtype=int))
    R = polar.size
    nmax = 2 * lmax * (lmax + 2)
    pilm, taulm = spherical_functions_trigon(lmax, np.cos(polar), np.sin(polar))  # (L+1, L+1, R)
    coef = np.zeros((R, nmax), dtype=complex)
    ifac = -1j  # B^dagger
    for m in range(-lmax, lmax + 1):
        phase = 4.0 * amplitude * np.exp(-1j * m * azimuthal)  # (R,)
        for l in range(max(1, abs(m)), lmax + 1):
            pre = -1.0 / np.power(ifac, l + 1) / np.sqrt(2 * l * (l + 1))
            tau_l, pi_l = taulm[l, abs(m)], m * pilm[l, abs(m)]  # (R,)
            for tau in (1, 2):
                # TE (pol 1) / TM (pol 2): tau == pol selects tau_lm, else m pi_lm; unpolarised: mean
                spher = np.where(pol == tau, tau_l, pi_l)
                pfac = np.where(pol == 1, ifac, 1.0)
                tc = pre * pfac * spher
                unp = pre * (ifac + 1) * (tau_l + pi_l) / 2
                tc = np.where((pol == 1) | (pol == 2), tc, unp)
                coef[:, mode_index(lmax, tau, l, m)] = phase * tc
    return coef


def wave_vectors(polar, azimuthal, k: float) -> np.ndarray:
    """(R, 3) wave vectors of the incidences (direction from the polar / azimuthal angles)."""
    polar = np.atleast_1d(np.asarray(polar, dtype=float))
    azimuthal = np.atleast_1d(np.asarray(azimuthal, dtype=float))
    return np.ascontiguousarray(np.stack((np.sin(polar) * np.cos(azimuthal), np.sin(polar) * np.sin(azimuthal),
                                          np.cos(polar)), axis=1) * float(np.real(k)))


def plane_wave_block(lmax: int, positions: np.ndarray, k: complex, polar: np.ndarray,
                     azimuthal: np.ndarray, pol: np.ndarray, amplitude: float = 1.0,
                     focal_point=(0.0, 0.0, 0.0)) -> np.ndarray:
    """Plane-wave coefficients a[s, n, r] for R incidences (complex128, (N, nmax, R)), host."""
    coef = plane_wave_mode_factors(lmax, polar, azimuthal, pol, amplitude)  # (R, nmax)
    kvec = np.stack((np.sin(np.atleast_1d(polar)) * np.cos(np.atleast_1d(azimuthal)),
                     np.sin(np.atleast_1d(polar)) * np.sin(np.atleast_1d(azimuthal)),
                     np.cos(np.atleast_1d(polar))), axis=0) * k  # (3, R)
    rel = positions - np.asarray(focal_point, dtype=float)
    eikr = np.exp(1j * (rel @ kvec))  # (N, R)
    return eikr[:, None, :] * coef.T[None, :, :]


def compute_initial_field_coefficients(lmax: int, positions: np.ndarray, k_medium: np.ndarray,
                                       initial_field) -> np.ndarray:
    """(N, nmax, channels) plane-wave coefficients of ``initial_field`` (one incidence)."""
    bw = initial_field.beam_width
    if np.isfinite(bw) and bw > 0:
        raise NotImplementedError("Gaussian wavebundles are out of scope for the b200 backend")
    k_medium = np.atleast_1d(k_medium)
    cols = []
    for k in k_medium:
        a = plane_wave_block(lmax, positions, k, np.array([initial_field.polar_angle]),
                             np.array([initial_field.azimuthal_angle]), np.array([initial_field.pol]),
                             initial_field.amplitude, initial_field.focal_point)
        cols.append(a[:, :, 0])
    return np.stack(cols, axis=-1)
