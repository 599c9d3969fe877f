"""GPU parity of the float64 dense multi-column coupling (yasf_dpanel_matvec) against the
single-column float64 coupling kernel: equal to rounding (relative 1e-12), every lmax it supports,
column counts that are and are not multiples of the 32- and 64-column tiles, the master form
x - T (.) W x, and a single sphere (W = 0)."""

from __future__ import annotations

import numpy as np
import pytest
import torch
from conftest import rel_err

from yasf_b200.device import CouplingDevice
from yasf_b200.wigner import translation_table_ab5
from yasf_b200.workloads import rsa_cube

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _setup(lmax, n, seed, device):
    rng = np.random.default_rng(seed)
    radii = rng.uniform(0.05, 0.12, size=n)
    pos = rsa_cube(radii, 0.15, rng)
    dev = CouplingDevice(lmax, translation_table_ab5(lmax), pos, 2 * np.pi / 0.55, device)
    return dev, rng


@pytest.mark.parametrize("lmax,n,R", [(1, 6, 3), (2, 9, 1), (3, 17, 33), (4, 30, 64), (5, 12, 7), (6, 25, 40),
                                      (6, 21, 130), (3, 10, 64), (2, 7, 65), (1, 5, 64), (5, 14, 70)])
def test_dpanel_matches_float64_coupling(cuda_device, lmax, n, R):
    dev, rng = _setup(lmax, n, 300 + lmax, cuda_device)
    X = torch.from_numpy(rng.normal(size=(R, dev.n)) + 1j * rng.normal(size=(R, dev.n))).to(cuda_device)
    Y = dev.dpanel(X).cpu().numpy()
    ref = dev.coupling(X).cpu().numpy()
    for c in range(R):
        assert rel_err(Y[c], ref[c]) < TOL, c


def test_dpanel_master_form(cuda_device):
    dev, rng = _setup(6, 20, 11, cuda_device)
    R = 5
    X = torch.from_numpy(rng.normal(size=(R, dev.n)) + 1j * rng.normal(size=(R, dev.n))).to(cuda_device)
    T = torch.from_numpy(0.3 * (rng.normal(size=dev.n) + 1j * rng.normal(size=dev.n))).to(cuda_device)
    Y = dev.dpanel(X, T).cpu().numpy()
    ref = dev.master(X, T).cpu().numpy()
    assert rel_err(Y, ref) < TOL


def test_dpanel_single_sphere_is_zero(cuda_device):
    dev, _ = _setup(4, 1, 5, cuda_device)
    X = torch.ones((3, dev.n), dtype=torch.complex128, device=cuda_device)
    assert np.all(dev.dpanel(X).cpu().numpy() == 0)
