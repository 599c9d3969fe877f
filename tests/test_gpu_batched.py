"""Batched right-hand sides (yasf_batched_solve): float64-refined lockstep GMRES with the
tensor-core TF32 panel (and the complex64 / complex128 kernels) as the inner operator, against
independent float64 solves of every column (yasf_gmres_solve, rtol 1e-12)."""

from __future__ import annotations

import numpy as np
import pytest
import torch
from conftest import rel_err

from yasf_b200.device import CouplingDevice, DevicePreconditioner
from yasf_b200.incident import plane_wave_block
from yasf_b200.mie import compute_mie_coefficients
from yasf_b200.preconditioner import make_particle_partition
from yasf_b200.wigner import translation_table_ab5
from yasf_b200.workloads import aggregate_c1, aggregate_c2, incidences

pytestmark = pytest.mark.gpu


def _problem(device, n=30, ndir=3, agg=None):
    agg = aggregate_c1(seed=4, n=n) if agg is None else agg
    dev = CouplingDevice(agg.lmax, translation_table_ab5(agg.lmax), agg.positions, agg.k, device)
    pairs = np.array([[r, agg.refractive_index] for r in agg.radii])
    mie, _ = compute_mie_coefficients(agg.lmax, np.array([agg.k]), np.array([agg.k]), pairs)
    tm = np.ascontiguousarray(mie[:, :, 0].ravel())
    polar, azim, pol = incidences(ndir)
    a = plane_wave_block(agg.lmax, agg.positions, agg.k, polar, azim, pol)  # (N, nmax, R)
    A = np.ascontiguousarray(np.moveaxis(a, 2, 0).reshape(len(pol), -1))
    B = A * tm[None, :]
    return agg, dev, torch.from_numpy(tm).to(device), torch.from_numpy(B).to(device), A


def _reference(dev, tmat, B):
    X = []
    for c in range(B.shape[0]):
        x = B[c].clone()
        st = dev.gmres(tmat, B[c].contiguous(), x, 1e-12, 100, 50)
        assert st["info"] == 0
        X.append(x.cpu().numpy())
    return np.stack(X)


@pytest.mark.parametrize("inner", ["tf32", "c64", "c128"])
def test_batched_solve_matches_per_column_solves(cuda_device, inner):
    agg, dev, tmat, B, A = _problem(cuda_device)
    Xref = _reference(dev, tmat, B)
    X, st = dev.batched_solve(tmat, B, rtol=1e-10, restart=40, inner=inner, inner_rtol=1e-3)
    assert st["unconverged"] == 0 and st["worst_relative_residual"] <= 1e-10, st
    Xn = X.cpu().numpy()
    for c in range(B.shape[0]):
        assert rel_err(Xn[c], Xref[c]) < 1e-8, (inner, c)
        # extinction: C_ext = -pi/k^2 Re(a^H b)
        ce = -np.real(np.vdot(A[c], Xn[c]))
        cr = -np.real(np.vdot(A[c], Xref[c]))
        assert abs(ce - cr) <= 1e-9 * abs(cr)
    if inner == "tf32":
        assert st["panel_matvecs"] > 0 and st["refinement_steps"] >= 2


def test_batched_solve_with_block_jacobi(cuda_device):
    agg, dev, tmat, B, A = _problem(cuda_device, n=40, ndir=4)
    ext = agg.positions.max(axis=0) - agg.positions.min(axis=0)
    blocks = make_particle_partition(agg.positions, (ext + 2.0) / 2)
    pc = DevicePreconditioner(dev, blocks)
    pc.prepare(tmat)
    Xref = _reference(dev, tmat, B)
    X, st = dev.batched_solve(tmat, B, rtol=1e-10, restart=30, inner="tf32", precond=pc)
    assert st["unconverged"] == 0, st
    Xn = X.cpu().numpy()
    for c in range(B.shape[0]):
        assert rel_err(Xn[c], Xref[c]) < 1e-8


def test_batched_zero_column(cuda_device):
    agg, dev, tmat, B, A = _problem(cuda_device, n=12, ndir=1)
    B2 = torch.stack([B[0], torch.zeros_like(B[0]), B[1]])
    X, st = dev.batched_solve(tmat, B2, rtol=1e-9, restart=20, inner="tf32")
    assert st["unconverged"] == 0
    assert torch.count_nonzero(X[1]) == 0


@pytest.mark.parametrize("lmax", [7, 8])
def test_batched_tf32_high_lmax(cuda_device, lmax):
    # the packed panel variant (FP16 coefficients, implicit pair-table addresses) as inner operator
    agg, dev, tmat, B, A = _problem(cuda_device, ndir=2, agg=aggregate_c2(seed=5, n=10, lmax=lmax))
    Xref = _reference(dev, tmat, B)
    X, st = dev.batched_solve(tmat, B, rtol=1e-10, restart=40, inner="tf32", inner_rtol=1e-3)
    assert st["unconverged"] == 0 and st["panel_matvecs"] > 0, st
    Xn = X.cpu().numpy()
    for c in range(B.shape[0]):
        assert rel_err(Xn[c], Xref[c]) < 1e-8, c
        ce = -np.real(np.vdot(A[c], Xn[c]))
        cr = -np.real(np.vdot(A[c], Xref[c]))
        assert abs(ce - cr) <= 1e-9 * abs(cr)
