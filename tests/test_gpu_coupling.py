"""GPU parity of the coupling matvec and master operator (C ABI) against the oracle and the
reference fixtures. Tolerances: 1e-12 relative (max-norm) for complex128, 2e-5 for complex64."""

from __future__ import annotations

import numpy as np
import pytest
import torch
from conftest import rel_err

from oracle import restate as R
from yasf_b200._lib import YASF_C64
from yasf_b200.device import CouplingDevice
from yasf_b200.wigner import translation_table_ab5
from yasf_b200.workloads import aggregate_c2, rsa_cube

pytestmark = pytest.mark.gpu


def _dev(lmax, pos, k, device, table=None):
    table = translation_table_ab5(lmax) if table is None else table
    return CouplingDevice(lmax, table, pos, k, device), table


def _t(a, device):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.complex128)).to(device)


@pytest.mark.parametrize("fixture,lmax", [("ref_matvec_c1.npz", 4), ("ref_matvec_l6.npz", 6),
                                          ("ref_matvec_l3.npz", 3), ("ref_matvec_l7.npz", 7),
                                          ("ref_matvec_l8.npz", 8)])
def test_matvec_matches_reference(golden, cuda_device, fixture, lmax):
    g = golden(fixture)
    k = 2 * np.pi / float(g["wavelength"])
    dev, _ = _dev(lmax, g["positions"], k, cuda_device)
    wx = dev.coupling(_t(g["x"], cuda_device)).cpu().numpy()
    assert rel_err(wx, g["wx"]) < 1e-12
    mx = dev.master(_t(g["x"], cuda_device), _t(g["tmat"], cuda_device)).cpu().numpy()
    assert rel_err(mx, g["mx"]) < 1e-12


def test_matvec_matches_celes_golden(golden, cuda_device):
    g = golden("celes_coupling.npz")
    lmax = int(g["lmax"])
    k = 2 * np.pi / float(g["wavelength"]) * float(g["medium_index"])
    dev, _ = _dev(lmax, g["positions"], k, cuda_device)
    wx = dev.coupling(_t(g["x"], cuda_device)).cpu().numpy()
    np.testing.assert_allclose(wx, g["wx"], rtol=2e-4, atol=1e-5)


@pytest.mark.parametrize("lmax", [1, 2, 3, 4, 5, 6, 7, 8])
def test_matvec_every_lmax_matches_oracle(cuda_device, lmax):
    rng = np.random.default_rng(100 + lmax)
    n = 7
    radii = rng.uniform(0.05, 0.12, size=n)
    pos = rsa_cube(radii, 0.2, rng)
    k = 2 * np.pi / 0.5
    nmax = 2 * lmax * (lmax + 2)
    x = rng.normal(size=n * nmax) + 1j * rng.normal(size=n * nmax)
    dev, table = _dev(lmax, pos, k, cuda_device)
    wx = dev.coupling(_t(x, cuda_device)).cpu().numpy()
    ref = R.coupling_matvec_rows(lmax, pos, k, table, x)
    assert rel_err(wx, ref) < 1e-12


@pytest.mark.parametrize("n", [1, 2, 31, 33, 129, 300])
def test_matvec_ragged_sizes(cuda_device, n):
    """Lane tails (N not a multiple of 32/128), the single-sphere case (W x = 0), chunking."""
    lmax = 3
    rng = np.random.default_rng(n)
    radii = rng.uniform(0.05, 0.1, size=n)
    pos = rsa_cube(radii, 0.15, rng)
    k = 2 * np.pi / 0.6
    nmax = 30
    x = rng.normal(size=n * nmax) + 1j * rng.normal(size=n * nmax)
    dev, table = _dev(lmax, pos, k, cuda_device)
    wx = dev.coupling(_t(x, cuda_device)).cpu().numpy()
    if n == 1:
        assert np.all(wx == 0)
        return
    rows = min(n, 12)
    ref = R.coupling_matvec_rows(lmax, pos, k, table, x, 0, rows)
    assert rel_err(wx[: rows * nmax], ref) < 1e-12
    t0 = max(0, n - 3)
    ref_tail = R.coupling_matvec_rows(lmax, pos, k, table, x, t0, n)
    assert rel_err(wx[t0 * nmax:], ref_tail) < 1e-12


def test_complex64_matvec_within_single_precision(golden, cuda_device):
    g = golden("ref_matvec_c1.npz")
    k = 2 * np.pi / float(g["wavelength"])
    dev, _ = _dev(4, g["positions"], k, cuda_device)
    wx = dev.coupling(_t(g["x"], cuda_device), YASF_C64).cpu().numpy()
    assert rel_err(wx, g["wx"]) < 2e-5


def test_multi_column_matches_single(golden, cuda_device):
    g = golden("ref_matvec_l3.npz")
    k = 2 * np.pi / float(g["wavelength"])
    dev, _ = _dev(3, g["positions"], k, cuda_device)
    rng = np.random.default_rng(1)
    X = rng.normal(size=(3, dev.n)) + 1j * rng.normal(size=(3, dev.n))
    Y = dev.coupling(_t(X, cuda_device)).cpu().numpy()
    for c in range(3):
        y = dev.coupling(_t(X[c], cuda_device)).cpu().numpy()
        assert np.array_equal(Y[c], y)


def test_full_size_properties(cuda_device):
    """2000 spheres, lmax 6: linearity, determinism and a row-sampled oracle check."""
    agg = aggregate_c2(seed=0)
    dev, table = _dev(agg.lmax, agg.positions, agg.k, cuda_device)
    rng = np.random.default_rng(2)
    x1 = rng.normal(size=dev.n) + 1j * rng.normal(size=dev.n)
    x2 = rng.normal(size=dev.n) + 1j * rng.normal(size=dev.n)
    a = 0.3 - 1.7j
    y1 = dev.coupling(_t(x1, cuda_device))
    y2 = dev.coupling(_t(x2, cuda_device))
    y12 = dev.coupling(_t(x1 + a * x2, cuda_device))
    assert rel_err((y12).cpu().numpy(), (y1 + a * y2).cpu().numpy()) < 1e-12
    y1b = dev.coupling(_t(x1, cuda_device))
    assert torch.equal(y1, y1b)
    nmax = dev.nmax
    for s in (0, 977, 1999):
        ref = R.coupling_matvec_rows(agg.lmax, agg.positions, agg.k, table, x1, s, s + 1)
        assert rel_err(y1.cpu().numpy()[s * nmax:(s + 1) * nmax], ref) < 1e-11


def test_near_field_matvec_matches_reference_nearfar(golden, cuda_device):
    """yasf_coupling_matvec_nearfield against the reference's NearFarCouplingBackend (the pairs
    within the radius only, yasfpy/coupling/backends.py:259-459), at 1e-12; complex64 at 2e-5."""
    g = golden("ref_matvec_nearfar.npz")
    lmax = int(g["lmax"])
    k = 2 * np.pi / float(g["wavelength"])
    dev, _ = _dev(lmax, g["positions"], k, cuda_device)
    x = _t(g["x"], cuda_device)
    radius = float(g["near_field_radius"])
    assert rel_err(dev.coupling_nearfield(x, radius).cpu().numpy(), g["wx_near"]) < 1e-12
    assert rel_err(dev.coupling_nearfield(x, radius, YASF_C64).cpu().numpy(), g["wx_near"]) < 2e-5


@pytest.mark.parametrize("n,radius", [(300, 0.35), (129, 0.8)])
def test_near_field_matvec_matches_oracle_and_limits(cuda_device, n, radius):
    """Spatially scattered receivers, so many thread blocks skip whole sources; a radius beyond
    every distance gives the dense product, one below every distance gives zero."""
    rng = np.random.default_rng(n)
    radii = rng.uniform(0.05, 0.1, size=n)
    pos = rsa_cube(radii, 0.1, rng)
    k = 2 * np.pi / 0.6
    lmax = 3
    dev, table = _dev(lmax, pos, k, cuda_device)
    nmax = 2 * lmax * (lmax + 2)
    x = rng.normal(size=n * nmax) + 1j * rng.normal(size=n * nmax)
    xt = _t(x, cuda_device)
    ref = R.coupling_matvec_rows(lmax, pos, k, table, x, near_field_radius=radius)
    assert rel_err(dev.coupling_nearfield(xt, radius).cpu().numpy(), ref) < 1e-12
    far = 10.0 * float(np.ptp(pos, axis=0).max() + 1.0)
    assert rel_err(dev.coupling_nearfield(xt, far).cpu().numpy(), dev.coupling(xt).cpu().numpy()) < 1e-14
    assert np.all(dev.coupling_nearfield(xt, 0.0).cpu().numpy() == 0)
