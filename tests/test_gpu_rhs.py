"""Right-hand sides of R plane-wave incidences formed on the device (yasf_plane_wave_rhs), against
the reference's own incident coefficients and right-hand side (yasfpy/initial_field_coefficients.py:
79-142, yasfpy/simulation.py:189-205; fixture ref_solve_c1_tol1e-8.npz) and against the host block
for several incidences and polarisations (TE, TM, unpolarised). Tolerance 1e-12 relative (max-norm)."""

from __future__ import annotations

import numpy as np
import pytest
import torch
from conftest import rel_err

from yasf_b200.device import CouplingDevice
from yasf_b200.incident import plane_wave_block
from yasf_b200.wigner import translation_table_ab5

pytestmark = pytest.mark.gpu


def test_device_rhs_matches_reference(golden, cuda_device):
    g = golden("ref_solve_c1_tol1e-8.npz")
    lmax = int(g["lmax"])
    k = 2 * np.pi / float(g["wavelength"])
    dev = CouplingDevice(lmax, translation_table_ab5(lmax), g["positions"], k, cuda_device)
    tmat = torch.from_numpy(np.ascontiguousarray(g["mie"][g["sidx"]].ravel())).to(cuda_device)
    A, B = dev.plane_wave_rhs(tmat, [0.0], [0.0], [1])  # +z, TE: the fixture's incidence
    assert rel_err(A.cpu().numpy()[0], g["initial"].ravel()) < 1e-12
    assert rel_err(B.cpu().numpy()[0], g["rhs"].ravel()) < 1e-12


def test_device_rhs_matches_host_block_for_many_incidences(cuda_device):
    rng = np.random.default_rng(8)
    lmax, N = 5, 23
    pos = rng.uniform(-1, 1, size=(N, 3))
    k = 2 * np.pi / 0.7
    dev = CouplingDevice(lmax, translation_table_ab5(lmax), pos, k, cuda_device)
    R = 6
    polar, azim = rng.uniform(0, np.pi, R), rng.uniform(0, 2 * np.pi, R)
    pol = np.array([1, 2, 0, 2, 1, 0])
    tm = rng.normal(size=dev.n) + 1j * rng.normal(size=dev.n)
    A, B = dev.plane_wave_rhs(torch.from_numpy(tm).to(cuda_device), polar, azim, pol, amplitude=0.7,
                              focal_point=(0.1, -0.2, 0.3))
    host = plane_wave_block(lmax, pos, k, polar, azim, pol, 0.7, (0.1, -0.2, 0.3))  # (N, nmax, R)
    Ah = np.moveaxis(host, 2, 0).reshape(R, -1)
    assert rel_err(A.cpu().numpy(), Ah) < 1e-12
    assert rel_err(B.cpu().numpy(), Ah * tm[None, :]) < 1e-12
