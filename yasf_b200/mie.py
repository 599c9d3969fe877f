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
    """Return (mie, scatter_to_internal), each complex (U, nmax, channels)."""
    nmax = 2 * lmax * (lmax + 2)
    k_medium = np.atleast_1d(k_medium)
    channels = k_medium.shape[0]
    U = unique_radius_index_pairs.shape[0]
    mie = np.zeros((U, nmax, channels), dtype=complex)
    ratio = np.zeros_like(mie)
    l_orders = np.arange(1, lmax + 1)
    for u in range(U):
        k_sphere = np.atleast_1d(omega) * unique_radius_index_pairs[u, 1:]
        radius = float(np.real(unique_radius_index_pairs[u, 0]))
        m = k_sphere / k_medium
        x = np.atleast_1d(k_medium) * radius
        mx = np.atleast_1d(k_sphere) * radius
        lg = l_orders[:, None]
        jx = spherical_jn(lg, x[None, :])
        jxp = spherical_jn(lg, x[None, :], derivative=True)
        yx = spherical_yn(lg, x[None, :])
        yxp = spherical_yn(lg, x[None, :], derivative=True)
        jmx = spherical_jn(lg, mx[None, :])
        jmxp = spherical_jn(lg, mx[None, :], derivative=True)
        hx = jx + 1j * yx
        hxp = jxp + 1j * yxp
        djx = jx + x * jxp
        djmx = jmx + mx * jmxp
        dhx = hx + x * hxp
        num = jmx * djx - jx * djmx
        den = jmx * dhx - hx * djmx
        t1 = -num / den
        t2 = -(m**2 * jmx * djx - jx * djmx) / (m**2 * jmx * dhx - hx * djmx)
        r1 = (jx * dhx - hx * djx) / (-num)
        r2 = (m * jx * dhx - m * hx * djx) / (-(m**2 * jmx * djx - jx * djmx))
        for li, l in enumerate(l_orders):
            w = 2 * int(l) + 1
            s1 = int(l) * int(l) - 1
            s2 = lmax * (lmax + 2) + int(l) * int(l) - 1
            mie[u, s1:s1 + w, :] = t1[li, :]
            ratio[u, s1:s1 + w, :] = r1[li, :]
            mie[u, s2:s2 + w, :] = t2[li, :]
            ratio[u, s2:s2 + w, :] = r2[li, :]
    return mie, ratio


def mie_tmatrix_per_sphere(lmax: int, k_medium: float, radii: np.ndarray,
                           refractive_index: complex | np.ndarray) -> np.ndarray:
    """Diagonal T for every sphere at once, (N*nmax,) complex128 in the unknowns' order.

    The same formulas as ``compute_mie_coefficients`` (yasfpy/mie_coefficients.py:87-161),
    vectorised over spheres instead of looping over unique (radius, index) pairs.
    """
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
