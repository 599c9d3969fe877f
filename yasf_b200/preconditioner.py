"""Block-diagonal (block-Jacobi) preconditioner on the device (yasfpy/preconditioner.py:58-519).

``make_particle_partition`` keeps the reference's cell assignment exactly (bin edges from
``min - 1`` to ``max + 1`` by the edge size, ``np.digitize`` per axis, blocks in first-seen order,
yasfpy/preconditioner.py:222-265). ``prepare(simulation)`` assembles M_B = (I - T W)[B, B] for
every block on the device with the matvec's pair generator, in particle-major order with the
receiver's Mie factor, and inverts each block (complex128). ``apply(rhs)`` returns M^{-1} rhs
block by block (host arrays in and out, for API parity); the device solver uses the same factors
without leaving the GPU. Singleton blocks give M_B = I, as in the reference.
"""

from __future__ import annotations

import logging
from typing import List

import numpy as np
import torch

from yasf_b200.device import PRECISIONS, DevicePreconditioner


def make_particle_partition(positions: np.ndarray, edge_sizes: np.ndarray) -> List[np.ndarray]:
    x_min, y_min, z_min = positions.min(axis=0) - 1.0
    x_max, y_max, z_max = positions.max(axis=0) + 1.0
    x_edges = np.arange(x_min, x_max + edge_sizes[0], edge_sizes[0])
    y_edges = np.arange(y_min, y_max + edge_sizes[1], edge_sizes[1])
    z_edges = np.arange(z_min, z_max + edge_sizes[2], edge_sizes[2])
    xb = np.digitize(positions[:, 0], x_edges)
    yb = np.digitize(positions[:, 1], y_edges)
    zb = np.digitize(positions[:, 2], z_edges)
    groups: dict = {}
    for i in range(len(positions)):
        groups.setdefault((xb[i], yb[i], zb[i]), []).append(i)
    return [np.array(v, dtype=int) for v in groups.values()]


class BlockDiagonalPreconditioner:
    def __init__(self, partition_edge_sizes: np.ndarray):
        self.partition_edge_sizes = np.asarray(partition_edge_sizes, dtype=float)
        if self.partition_edge_sizes.shape != (3,):
            raise ValueError("partition_edge_sizes must be array of shape (3,)")
        self.partitioning: List[np.ndarray] | None = None
        self.partitioning_idcs: List[np.ndarray] | None = None
        self._dev: DevicePreconditioner | None = None
        self._sim = None
        self.log = logging.getLogger(self.__class__.__module__)

    def prepare(self, simulation, channel: int = 0):
        """Partition, assemble and invert every block for wavelength channel ``channel``."""
        positions = simulation.parameters.particles.position
        nmax = simulation.numerics.nmax
        self.partitioning = make_particle_partition(positions, self.partition_edge_sizes)
        self.partitioning_idcs = [
            (blk[:, None] * nmax + np.arange(nmax)[None, :]).ravel() for blk in self.partitioning
        ]
        dev = simulation.device_state(channel)
        tmat = simulation.device_tmat(channel)
        self._dev = DevicePreconditioner(dev, self.partitioning)
        self._dev.prepare(tmat)
        self._sim = simulation
        return simulation

    def device_handle(self, dev=None) -> DevicePreconditioner:
        if self._dev is None:
            raise RuntimeError("Preconditioner not prepared. Call prepare() first.")
        return self._dev

    def apply(self, rhs: np.ndarray, precision: str = "c128") -> np.ndarray:
        if self._dev is None:
            raise RuntimeError("Preconditioner not prepared. Call prepare() first.")
        x = torch.from_numpy(np.ascontiguousarray(np.asarray(rhs, dtype=np.complex128).ravel()))
        y = self._dev.apply(x.to(self._dev.dev.device), PRECISIONS[precision])
        return y.cpu().numpy()
