"""GPU parity of the tensor-core panel (yasf_panel_matvec, tcgen05 kind::tf32) against the
complex128 coupling matvec. TF32 inputs carry 11 significant bits, so the panel is checked at a
relative tolerance of 5e-3 (max-norm) and column by column against the float64 result."""

from __future__ import annotations

import numpy as np
import pytest
import torch
from conftest import rel_err

from yasf_b200.device import CouplingDevice
from yasf_b200.wigner import translation_table_ab5
from yasf_b200.workloads import rsa_cube

pytestmark = pytest.mark.gpu

TOL = 5e-3


def _setup(lmax, n, seed, device):
    rng = np.random.default_rng(seed)
    radii = rng.uniform(0.05, 0.12, size=n)
    pos = rsa_cube(radii, 0.15, rng)
    dev = CouplingDevice(lmax, translation_table_ab5(lmax), pos, 2 * np.pi / 0.55, device)
    return dev, rng


@pytest.mark.parametrize("lmax,n,R", [(1, 5, 3), (2, 9, 1), (3, 17, 7), (4, 33, 64), (5, 12, 65), (6, 20, 16),
                                      (6, 41, 128), (3, 2, 2), (4, 23, 130), (5, 9, 200), (7, 19, 5),
                                      (7, 27, 100), (8, 7, 3), (8, 16, 70)])
def test_panel_matches_float64_matvec(cuda_device, lmax, n, R):
    dev, rng = _setup(lmax, n, 100 + lmax, cuda_device)
    X = torch.from_numpy(rng.normal(size=(R, dev.n)) + 1j * rng.normal(size=(R, dev.n))).to(cuda_device)
    Y = dev.panel(X).cpu().numpy()
    ref = dev.coupling(X).cpu().numpy()
    assert np.isfinite(Y).all()
    for c in range(R):
        assert rel_err(Y[c], ref[c]) < TOL, c


def test_panel_master_epilogue(cuda_device):
    dev, rng = _setup(4, 25, 7, cuda_device)
    R = 4
    X = torch.from_numpy(rng.normal(size=(R, dev.n)) + 1j * rng.normal(size=(R, dev.n))).to(cuda_device)
    T = torch.from_numpy(0.2 * (rng.normal(size=dev.n) + 1j * rng.normal(size=dev.n))).to(cuda_device)
    Y = dev.panel(X, T).cpu().numpy()
    ref = dev.master(X, T).cpu().numpy()
    xnp = X.cpu().numpy()
    # compare the coupling part x - y against T W x
    assert rel_err(xnp - Y, xnp - ref) < TOL


def test_panel_single_sphere_is_zero(cuda_device):
    dev, rng = _setup(3, 1, 3, cuda_device)
    X = torch.ones((2, dev.n), dtype=torch.complex128, device=cuda_device)
    Y = dev.panel(X).cpu().numpy()
    assert np.all(Y == 0)


@pytest.mark.parametrize("fixture,lmax", [("ref_matvec_l7.npz", 7), ("ref_matvec_l8.npz", 8)])
def test_panel_high_orders_match_reference(golden, cuda_device, fixture, lmax):
    # lmax 7-8 pack the generation coefficients as FP16 pairs: checked against the reference's own
    # coupling matvec and master operator at those orders
    g = golden(fixture)
    k = 2 * np.pi / float(g["wavelength"])
    dev = CouplingDevice(lmax, translation_table_ab5(lmax), g["positions"], k, cuda_device)
    X = torch.from_numpy(np.ascontiguousarray(g["x"][None, :])).to(cuda_device)
    T = torch.from_numpy(np.ascontiguousarray(g["tmat"])).to(cuda_device)
    assert rel_err(dev.panel(X).cpu().numpy()[0], g["wx"]) < TOL
    mx = dev.panel(X, T).cpu().numpy()[0]
    assert rel_err(g["x"] - mx, g["x"] - g["mx"]) < TOL
