"""``Numerics``: numerical settings of a run (mirror of yasfpy/numerics.py:23-344).

Keeps the reference's constructor keywords (``lmax``, ``sampling_points_number``, ``gpu``,
``particle_distance_resolution``, ``solver``, ``coupling_backend``, ``coupling_tile_size``,
``coupling_near_field_radius``) and adds ``coupling_backend="b200"`` (the default here) and
``b200_precision`` ("c128" plain float64 solve, "c64" complex64 inner solves in float64 iterative
refinement). The translation table is computed exactly (``yasf_b200.wigner``) and cached in memory
per lmax; set ``YASF_B200_CACHE`` to a directory to also cache it on disk.
"""

from __future__ import annotations

import logging
import os
from pathlib import Path
from typing import Callable, Union

import numpy as np

from yasf_b200.wigner import translation_table_ab5

_TABLE_CACHE: dict[int, np.ndarray] = {}


def cached_translation_table(lmax: int) -> np.ndarray:
    """a5/b5 table for lmax (memory cache, optional disk cache in $YASF_B200_CACHE)."""
    if lmax in _TABLE_CACHE:
        return _TABLE_CACHE[lmax]
    cache_dir = os.environ.get("YASF_B200_CACHE")
    path = Path(cache_dir) / f"ab5_lmax{lmax}.npy" if cache_dir else None
    if path is not None and path.exists():
        table = np.load(path)
    else:
        table = translation_table_ab5(lmax)
        if path is not None:
            path.parent.mkdir(parents=True, exist_ok=True)
            np.save(path, table)
    _TABLE_CACHE[lmax] = table
    return table


class Numerics:
    """Numerical configuration: truncation order, sampling grid, coupling backend, solver."""

    def __init__(
        self,
        lmax: int,
        sampling_points_number: Union[int, np.ndarray] = np.array([100]),
        polar_angles: np.ndarray | None = None,
        polar_weight_func: Callable = lambda x: x,
        azimuthal_angles: np.ndarray | None = None,
        gpu: bool = True,
        particle_distance_resolution: float = 10.0,
        solver=None,
        coupling_backend: str = "b200",
        coupling_tile_size: int = 64,
        coupling_near_field_radius: float | None = None,
        b200_precision: str = "c128",
    ):
        self.log = logging.getLogger(self.__class__.__module__)
        self.lmax = int(lmax)
        self.sampling_points_number = np.squeeze(sampling_points_number)
        if (polar_angles is None) or (azimuthal_angles is None):
            spn = np.atleast_1d(self.sampling_points_number)
            if spn.size == 0:
                spn = np.array([100])
            if spn.size == 1:
                _, polar_angles, azimuthal_angles = Numerics.compute_fibonacci_sphere_points(int(spn[0]))
            else:
                pol = np.pi * polar_weight_func(np.linspace(0, 1, int(spn[1])))
                azi = 2 * np.pi * np.linspace(0, 1, int(spn[0]) + 1)[:-1]
                polar_angles, azimuthal_angles = np.meshgrid(pol, azi, indexing="xy")
                polar_angles = polar_angles.ravel()
                azimuthal_angles = azimuthal_angles.ravel()
        self.polar_angles = polar_angles
        self.azimuthal_angles = azimuthal_angles
        self.gpu = gpu
        self.particle_distance_resolution = particle_distance_resolution
        self.solver = solver
        self.coupling_backend = coupling_backend
        self.coupling_tile_size = int(coupling_tile_size)
        self.coupling_near_field_radius = coupling_near_field_radius
        if b200_precision not in ("c128", "c64"):
            raise ValueError("b200_precision must be 'c128' or 'c64'")
        self.b200_precision = b200_precision
        self.nmax = 2 * self.lmax * (self.lmax + 2)
        self.translation_ab5: np.ndarray | None = None

    def compute_translation_table(self, force_compute: bool = False) -> None:
        """Fill ``translation_ab5`` (nmax, nmax, 2*lmax+1) as yasfpy/numerics.py:187-281 does."""
        if force_compute:
            _TABLE_CACHE.pop(self.lmax, None)
        self.translation_ab5 = cached_translation_table(self.lmax)

    @staticmethod
    def compute_fibonacci_sphere_points(n: int = 100):
        """Fibonacci-sphere points (yasfpy/numerics.py:283-312): (points, theta, phi)."""
        golden_ratio = (1 + 5**0.5) / 2
        i = np.arange(0, n)
        phi = 2 * np.pi * (i / golden_ratio % 1)
        theta = np.arccos(1 - 2 * i / n)
        pts = np.stack(
            (np.sin(theta) * np.cos(phi), np.sin(theta) * np.sin(phi), np.cos(theta)), axis=1
        )
        return pts, theta, phi
