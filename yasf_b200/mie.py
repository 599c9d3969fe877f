"""Mie coefficients: the diagonal sphere T-matrix (yasfpy/mie_coefficients.py:29-161).

Same formulas as the reference: for every unique (radius, refractive index) pair and channel,
tau=1 -> -(j(mx) [x j(x)]' - j(x) [mx j(mx)]') / (j(mx) [x h(x)]' - h(x) [mx j(mx)]'),
tau=2 the corresponding m^2-weighted ratio, replicated over m = -l..l.
"""

from __future__ import annotations

import numpy as np
from scipy.special import spherical_jn, spherical_yn


def compute_mie_coefficients(lmax: int, omega: np.ndarray, k_medium: np.ndarray,
                             unique_radius_index_pairs: np.ndarray):
    """Mie coefficients per unique (radius, refractive index) pair and wavelength channel,
    complex (U, nmax, channels), the layout of yasfpy's ``Simulation.mie_coefficients``
    (yasfpy/mie_coefficients.py:29-161). The channel's refractive index is omega * n_particle / k.
    Returned with None in place of the reference's internal-field ratio (scatter_to_internal),
    which only the near-field consumers read."""
    pairs = np.asarray(unique_radius_index_pairs)
    k_medium = np.atleast_1d(k_medium)
    omega = np.atleast_1d(omega)
    radii = np.real(pairs[:, 0]).astype(float)
    U = radii.size
    nmax = 2 * lmax * (lmax + 2)
    mie = np.zeros((U, nmax, k_medium.size), dtype=complex)
    for w, k in enumerate(k_medium):
        m = omega[w] * pairs[:, 1 + w] / k
        mie[:, :, w] = mie_tmatrix_per_sphere(lmax, k, radii, m, k_is_complex=True).reshape(U, nmax)
    return mie, None


def mie_tmatrix_per_sphere(lmax: int, k_medium: float, radii: np.ndarray,
                           refractive_index: complex | np.ndarray, k_is_complex: bool = False) -> np.ndarray:
    """Diagonal T for every sphere at once, (N*nmax,) complex128 in the unknowns' order, from
    the Mie coefficients of a homogeneous sphere (the definition of T the reference uses,
    yasfpy/mie_coefficients.py:87-161), vectorised over spheres and orders l.
    """
    if not k_is_complex:
        k_medium = float(np.real(k_medium))
    radii = np.asarray(radii, dtype=float)
    N = radii.size
    m = np.broadcast_to(np.asarray(refractive_index, dtype=complex), (N,))
    nmax = 2 * lmax * (lmax + 2)
    lg = np.arange(1, lmax + 1)[:, None]
    x = (k_medium * radii)[None, :]
    mx = (k_medium * m * radii)[None, :]
    jx = spherical_jn(lg, x)
    jxp = spherical_jn(lg, x, derivative=True)
    yx = spherical_yn(lg, x)
    yxp = spherical_yn(lg, x, derivative=True)
    jmx = spherical_jn(lg, mx)
    jmxp = spherical_jn(lg, mx, derivative=True)
    hx = jx + 1j * yx
    hxp = jxp + 1j * yxp
    djx = jx + x * jxp
    djmx = jmx + mx * jmxp
    dhx = hx + x * hxp
    mm = m[None, :]
    t1 = -(jmx * djx - jx * djmx) / (jmx * dhx - hx * djmx)
    t2 = -(mm**2 * jmx * djx - jx * djmx) / (mm**2 * jmx * dhx - hx * djmx)
    out = np.zeros((N, nmax), dtype=complex)
    for li, l in enumerate(range(1, lmax + 1)):
        w = 2 * l + 1
        s1 = l * l - 1
        s2 = lmax * (lmax + 2) + l * l - 1
        out[:, s1:s1 + w] = t1[li, :, None]
        out[:, s2:s2 + w] = t2[li, :, None]
    return out.ravel()
