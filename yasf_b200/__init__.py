"""yasf_b200: B200-native coupling backend for the T-matrix multiple-sphere solve of yasfpy.

The public objects mirror yasfpy's (``Particles``, ``InitialField``, ``Parameters``, ``Numerics``,
``Solver``, ``Simulation``, ``Optics``, ``BlockDiagonalPreconditioner``) with
``Numerics(coupling_backend="b200")`` selecting the device path. The arithmetic on the hot path
(coupling matvec, master operator, GMRES, preconditioner apply, cross sections) runs in the CUDA
library ``yasf_b200/_build/libyasf_b200.so`` through the C ABI of ``include/yasf_b200.h``.
"""

from yasf_b200.initial_field import InitialField
from yasf_b200.numerics import Numerics
from yasf_b200.parameters import Parameters
from yasf_b200.particles import Particles

__version__ = "0.1.0"

__all__ = [
    "InitialField",
    "Numerics",
    "Parameters",
    "Particles",
    "Simulation",
    "Solver",
    "Optics",
    "BlockDiagonalPreconditioner",
]


def __getattr__(name):
    # Device-backed objects import torch and the CUDA library lazily.
    if name == "Simulation":
        from yasf_b200.simulation import Simulation

        return Simulation
    if name == "Solver":
        from yasf_b200.solver import Solver

        return Solver
    if name == "Optics":
        from yasf_b200.optics import Optics

        return Optics
    if name == "BlockDiagonalPreconditioner":
        from yasf_b200.preconditioner import BlockDiagonalPreconditioner

        return BlockDiagonalPreconditioner
    raise AttributeError(name)
