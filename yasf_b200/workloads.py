"""Seeded synthetic sphere aggregates and incidence sets for tests and benchmarks.

No dataset is involved: every aggregate is built by random sequential addition (RSA) of
non-overlapping spheres with ``numpy.random.default_rng(seed)``. Lengths are in micrometres, the
medium is vacuum (k = 2 pi / wavelength).

Named workloads:

- ``aggregate_c1``: 100 spheres, radii U[0.05, 0.15], RSA in a cube at volume fraction 0.10,
  m = 1.5+0.01i, wavelength 0.55, lmax 4.
- ``aggregate_c2``: 2000 spheres, radii lognormal (median 0.1, sigma_ln 0.2) clipped to
  [0.04, 0.25], RSA in a ball at volume fraction 0.20, m = 1.6+0.005i, wavelength 0.6, lmax 6.
- ``aggregate_c5``: 20000 spheres, radii U[0.08, 0.12], RSA in a cube at volume fraction 0.30,
  m = 1.5+0.01i, wavelength 0.55, lmax 4.
- ``incidences``: Fibonacci-sphere directions x (TE, TM).
- ``serving_requests``: the mixed request stream (Poisson arrivals, per-request N, lmax, volume
  fraction, radii, wavelength, refractive index and incidence count drawn per request).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Aggregate:
    name: str
    positions: np.ndarray          # (N, 3)
    radii: np.ndarray              # (N,)
    refractive_index: complex
    wavelength: float
    lmax: int
    seed: int
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return self.positions.shape[0]

    @property
    def k(self) -> float:
        return 2 * math.pi / self.wavelength


def _rsa(radii: np.ndarray, sampler, rng: np.random.Generator, max_attempts: int,
         largest_first: bool = False) -> np.ndarray:
    """Random sequential addition with a uniform-grid neighbour search.

    Spheres are inserted in index order, or largest first (the usual way to reach dense
    polydisperse packings: small spheres still fit in the gaps the large ones leave); sphere i
    keeps radius radii[i] either way.
    """
    N = radii.size
    rmax = float(radii.max())
    cell = 2.0 * rmax
    grid: dict[tuple[int, int, int], list[int]] = {}
    pos = np.zeros((N, 3))
    attempts = 0
    batch = 256
    order = np.argsort(-radii, kind="stable") if largest_first else range(N)
    for i in order:
        placed = False
        while not placed:
            cand = sampler(radii[i], batch)
            for c in cand:
                attempts += 1
                if attempts > max_attempts:
                    raise RuntimeError(f"RSA failed to place {N} spheres within {max_attempts} attempts")
                key = tuple(np.floor(c / cell).astype(int))
                ok = True
                for dx in (-1, 0, 1):
                    for dy in (-1, 0, 1):
                        for dz in (-1, 0, 1):
                            for j in grid.get((key[0] + dx, key[1] + dy, key[2] + dz), ()):
                                d = c - pos[j]
                                if d @ d < (radii[i] + radii[j]) ** 2:
                                    ok = False
                                    break
                            if not ok:
                                break
                        if not ok:
                            break
                    if not ok:
                        break
                if ok:
                    pos[i] = c
                    grid.setdefault(key, []).append(i)
                    placed = True
                    break
    return pos


def rsa_cube(radii: np.ndarray, volume_fraction: float, rng: np.random.Generator,
             max_attempts: int = 50_000_000, largest_first: bool = False) -> np.ndarray:
    """Centres in a cube of side L = (sum 4/3 pi r^3 / phi)^(1/3), each sphere inside the cube."""
    side = (np.sum(4.0 / 3.0 * np.pi * radii**3) / volume_fraction) ** (1.0 / 3.0)

    def sampler(r, n):
        return rng.uniform(r, side - r, size=(n, 3))

    return _rsa(radii, sampler, rng, max_attempts, largest_first)


def rsa_ball(radii: np.ndarray, volume_fraction: float, rng: np.random.Generator,
             max_attempts: int = 50_000_000, largest_first: bool = False) -> np.ndarray:
    """Centres in a ball of radius R = (sum r^3 / phi)^(1/3), each sphere inside the ball."""
    R = (np.sum(radii**3) / volume_fraction) ** (1.0 / 3.0)

    def sampler(r, n):
        v = rng.normal(size=(n, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        rad = (R - r) * rng.uniform(0.0, 1.0, size=(n, 1)) ** (1.0 / 3.0)
        return v * rad

    return _rsa(radii, sampler, rng, max_attempts, largest_first)


def aggregate_c1(seed: int = 0, n: int = 100) -> Aggregate:
    rng = np.random.default_rng(seed)
    radii = rng.uniform(0.05, 0.15, size=n)
    pos = rsa_cube(radii, 0.10, rng)
    return Aggregate("rsa-cube-phi0.10-N%d-lmax4" % n, pos, radii, 1.5 + 0.01j, 0.55, 4, seed)


def aggregate_c2(seed: int = 0, n: int = 2000, lmax: int = 6) -> Aggregate:
    rng = np.random.default_rng(seed)
    radii = np.clip(rng.lognormal(mean=math.log(0.1), sigma=0.2, size=n), 0.04, 0.25)
    pos = rsa_ball(radii, 0.20, rng)
    return Aggregate("rsa-ball-phi0.20-N%d-lmax%d" % (n, lmax), pos, radii, 1.6 + 0.005j, 0.6, lmax, seed)


def aggregate_c5(seed: int = 0, n: int = 20000) -> Aggregate:
    rng = np.random.default_rng(seed)
    radii = rng.uniform(0.08, 0.12, size=n)
    pos = rsa_cube(radii, 0.30, rng)
    return Aggregate("rsa-cube-phi0.30-N%d-lmax4" % n, pos, radii, 1.5 + 0.01j, 0.55, 4, seed)


def incidences(n_directions: int, rotation_seed: int | None = None):
    """(polar, azimuthal, pol) arrays for n_directions Fibonacci directions x (TE, TM)."""
    i = np.arange(n_directions)
    golden = (1 + 5**0.5) / 2
    phi = 2 * np.pi * (i / golden % 1)
    theta = np.arccos(1 - 2 * i / n_directions)
    if rotation_seed is not None:
        rng = np.random.default_rng(rotation_seed)
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        a, b, c, d = q
        Rm = np.array([[a*a+b*b-c*c-d*d, 2*(b*c-a*d), 2*(b*d+a*c)],
                       [2*(b*c+a*d), a*a-b*b+c*c-d*d, 2*(c*d-a*b)],
                       [2*(b*d-a*c), 2*(c*d+a*b), a*a-b*b-c*c+d*d]])
        v = np.stack((np.sin(theta) * np.cos(phi), np.sin(theta) * np.sin(phi), np.cos(theta)), 1) @ Rm.T
        theta = np.arccos(np.clip(v[:, 2], -1, 1))
        phi = np.arctan2(v[:, 1], v[:, 0])
    polar = np.repeat(theta, 2)
    azim = np.repeat(phi, 2)
    pol = np.tile(np.array([1, 2]), n_directions)
    return polar, azim, pol


@dataclass
class Request:
    rid: int
    arrival: float
    aggregate: Aggregate
    polar: np.ndarray
    azimuthal: np.ndarray
    pol: np.ndarray


def serving_requests(n_requests: int = 512, rate: float = 20.0, seed: int = 0,
                     n_range=(50, 3000), lmax_choices=(3, 4, 5, 6, 7, 8),
                     rhs_choices=(1, 2, 16, 64), param_seed: int = 1000) -> list[Request]:
    """The serving stream: Poisson arrivals; per-request parameters from seed param_seed + i.

    Request i of a shorter stream is request i of the 512-request stream (same arrival, same
    parameters), so a prefix is served by asking for fewer requests."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=n_requests)
    arrivals = np.cumsum(gaps) - gaps[0]
    reqs = []
    for i in range(n_requests):
        r = np.random.default_rng(param_seed + i)
        n = int(r.integers(n_range[0], n_range[1] + 1))
        lmax = int(r.choice(lmax_choices))
        phi = float(r.uniform(0.05, 0.30))
        radii = r.uniform(0.05, 0.2, size=n)
        wl = float(r.uniform(0.4, 0.8))
        m = complex(r.uniform(1.3, 1.8), 10 ** r.uniform(-4, -1))
        R = int(r.choice(rhs_choices))
        pos = rsa_cube(radii, phi, r, largest_first=True)
        agg = Aggregate(f"req{i}", pos, radii, m, wl, lmax, param_seed + i, {"phi": phi})
        ndir = max(1, R // 2) if R > 1 else 1
        polar, azim, pol = incidences(ndir)
        if R == 1:
            polar, azim, pol = polar[:1], azim[:1], pol[:1]
        reqs.append(Request(i, float(arrivals[i]), agg, polar[:R], azim[:R], pol[:R]))
    return reqs
