"""The grouped solve (yasf_grouped_solve): right-hand sides of several aggregates of one lmax
(different sphere counts, positions, wavenumbers, refractive indices, incidence counts) solved
together, every operator application one persistent work-queue contraction for all of them.

Each aggregate's solution must equal its own float64 batched solve: with the complex128 inner
operator to 1e-9 relative (max-norm; both are float64 GMRES to rtol 1e-11), with the complex64
inner operator (float64 refinement to rtol 1e-9) to 1e-7. Extinction cross sections of the mixed
form within 1e-6 of float64."""

from __future__ import annotations

import numpy as np
import pytest
import torch
from conftest import rel_err

from yasf_b200.device import CouplingDevice, grouped_solve
from yasf_b200.mie import mie_tmatrix_per_sphere
from yasf_b200.numerics import cached_translation_table
from yasf_b200.workloads import incidences, rsa_cube

pytestmark = pytest.mark.gpu


def _aggregates(device, lmax, specs):
    out = []
    for i, (n, R, wl, m) in enumerate(specs):
        rng = np.random.default_rng(900 + i)
        radii = rng.uniform(0.05, 0.12, size=n)
        pos = rsa_cube(radii, 0.15, rng)
        k = 2 * np.pi / wl
        dev = CouplingDevice(lmax, cached_translation_table(lmax), pos, k, device)
        tmat = torch.from_numpy(mie_tmatrix_per_sphere(lmax, k, radii, m)).to(device)
        polar, azim, pol = incidences((R + 1) // 2)  # R columns: ceil(R / 2) directions x TE/TM
        A, B = dev.plane_wave_rhs(tmat, polar[:R], azim[:R], pol[:R])
        out.append((dev, tmat, B, A))
    return out


@pytest.mark.parametrize("lmax", [3, 6])
def test_grouped_solve_equals_each_aggregate_alone(cuda_device, lmax):
    specs = [(40, 1, 0.5, 1.5 + 0.01j), (170, 2, 0.6, 1.4 + 0.05j), (7, 3, 0.45, 1.7 + 0.001j),
             (95, 1, 0.55, 1.33 + 0.1j)]
    aggs = _aggregates(cuda_device, lmax, specs)
    items = [(d, t, B) for d, t, B, _ in aggs]
    X64, st64 = grouped_solve(items, rtol=1e-11, restart=60, inner_rtol=1e-11, inner="c128")
    assert st64["unconverged"] == 0 and st64["columns"] == sum(R for _, R, _, _ in specs)
    for (dev, tmat, B, A), X in zip(aggs, X64):
        alone, sa = dev.batched_solve(tmat, B, rtol=1e-11, restart=60, inner_rtol=1e-11, inner="c128")
        assert sa["unconverged"] == 0
        assert rel_err(X.cpu().numpy(), alone.cpu().numpy()) < 1e-9
    Xm, stm = grouped_solve(items, rtol=1e-9, restart=40, inner_rtol=1e-4, inner="c64")
    assert stm["unconverged"] == 0 and stm["worst_relative_residual"] <= 1e-9
    for (dev, tmat, B, A), X, X_ref in zip(aggs, Xm, X64):
        assert rel_err(X.cpu().numpy(), X_ref.cpu().numpy()) < 1e-7
        k = dev.k
        ce = -torch.real((A.conj() * X).sum(dim=1)).cpu().numpy()
        ce64 = -torch.real((A.conj() * X_ref).sum(dim=1)).cpu().numpy()
        assert np.all(np.abs(ce - ce64) <= 1e-6 * np.abs(ce64)), k


def test_grouped_solve_single_sphere_and_validation(cuda_device):
    aggs = _aggregates(cuda_device, 4, [(1, 1, 0.5, 1.5 + 0.01j), (30, 2, 0.5, 1.5 + 0.01j)])
    items = [(d, t, B) for d, t, B, _ in aggs]
    X, st = grouped_solve(items, rtol=1e-10, inner="c128", inner_rtol=1e-10)
    # one sphere: no coupling, so (I - T W) x = b gives x = b
    assert rel_err(X[0].cpu().numpy(), aggs[0][2].cpu().numpy()) < 1e-14
    assert st["unconverged"] == 0
    other = _aggregates(cuda_device, 3, [(10, 1, 0.5, 1.5 + 0.01j)])[0]
    with pytest.raises(ValueError):
        grouped_solve(items + [(other[0], other[1], other[2])], rtol=1e-8)
