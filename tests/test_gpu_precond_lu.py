"""The batched block LU of the block-Jacobi preconditioner (yasf_precond_factor) and its
triangular-sweep apply, against dense solves of the same assembled blocks.

Block orders are multiples of nmax (48 at lmax 4, 96 at lmax 6), so most are not multiples of the
64-row tiles: the ragged last tile, several tiles per block and blocks of very different orders in
one factorisation are all exercised. Tolerances: forward error 1e-10 relative (max-norm) with the
complex128 factors kept; with the complex64 factors the solves stream, the residual of the block
system below 1e-5 of the right-hand side (backward error; the forward error is bounded by it times
the blocks' condition number).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch
from conftest import rel_err

from yasf_b200._lib import YASF_C64, YASF_C128
from yasf_b200.device import CouplingDevice, DevicePreconditioner
from yasf_b200.mie import mie_tmatrix_per_sphere
from yasf_b200.preconditioner import make_particle_partition
from yasf_b200.wigner import translation_table_ab5
from yasf_b200.workloads import rsa_cube

pytestmark = pytest.mark.gpu


def _setup(device, lmax, n, phi, cells, seed):
    rng = np.random.default_rng(seed)
    radii = rng.uniform(0.06, 0.12, size=n)
    pos = rsa_cube(radii, phi, rng, largest_first=True)
    k = 2 * np.pi / 0.55
    dev = CouplingDevice(lmax, translation_table_ab5(lmax), pos, k, device)
    tm = mie_tmatrix_per_sphere(lmax, k, radii, 1.55 + 0.01j)
    tmat = torch.from_numpy(tm).to(device)
    extent = pos.max(axis=0) - pos.min(axis=0)
    blocks = make_particle_partition(pos, (extent + 2.0) / cells)
    return dev, tmat, blocks, rng


def _block_product(dev, mats, blocks, y):
    out = np.zeros_like(y)
    nmax = dev.nmax
    for M, blk in zip(mats, blocks):
        idx = (blk[:, None] * nmax + np.arange(nmax)[None, :]).ravel()
        out[idx] = M @ y[idx]
    return out


@pytest.mark.parametrize("lmax,n,phi,cells", [(4, 160, 0.25, 3), (6, 40, 0.2, 2), (3, 90, 0.3, 1)])
def test_block_lu_apply_inverts_the_blocks(cuda_device, lmax, n, phi, cells):
    dev, tmat, blocks, rng = _setup(cuda_device, lmax, n, phi, cells, 10 + lmax)
    assert max(len(b) for b in blocks) * dev.nmax > 128  # several tiles in the largest block
    pc = DevicePreconditioner(dev, blocks)
    pc.assemble(tmat)
    mats = [pc.block_matrix(b).cpu().numpy() for b in range(len(blocks))]
    pc.prepare(tmat, keep_float64=True)
    y = rng.normal(size=dev.n) + 1j * rng.normal(size=dev.n)
    My = torch.from_numpy(_block_product(dev, mats, blocks, y)).to(cuda_device)
    out = pc.apply(My, YASF_C128).cpu().numpy()
    assert rel_err(out, y) < 1e-10
    # complex64 factors: a backward-stable solve with them leaves a small residual of the block
    # system (its forward error grows with the blocks' condition number, ~1e5 at lmax 6)
    out64 = pc.apply(My, YASF_C64).cpu().numpy()
    resid = _block_product(dev, mats, blocks, out64) - My.cpu().numpy()
    assert np.linalg.norm(resid) < 1e-5 * np.linalg.norm(My.cpu().numpy())
    # several right-hand sides in one apply (one launch per tile row and sweep) agree with the
    # one-column applies (one launch, rows ordered by tickets) up to the order of the float64 sums
    X = torch.from_numpy(rng.normal(size=(3, dev.n)) + 1j * rng.normal(size=(3, dev.n))).to(cuda_device)
    Y = pc.apply(X, YASF_C64).cpu().numpy()
    for c in range(3):
        yc = pc.apply(X[c].contiguous(), YASF_C64).cpu().numpy()
        assert rel_err(Y[c], yc) < 1e-10
        # the one-column solve sums every row in a fixed order: repeated applies are bitwise equal
        assert np.array_equal(pc.apply(X[c].contiguous(), YASF_C64).cpu().numpy(), yc)
    Y64 = pc.apply(X, YASF_C128).cpu().numpy()
    assert rel_err(Y64[0], pc.apply(X[0].contiguous(), YASF_C128).cpu().numpy()) < 1e-12


def test_finalize_releases_the_float64_factors(cuda_device):
    dev, tmat, blocks, rng = _setup(cuda_device, 4, 60, 0.2, 2, 3)
    pc = DevicePreconditioner(dev, blocks)
    pc.prepare(tmat)  # complex64 factors only
    held = pc.nbytes()
    elems = sum((len(b) * dev.nmax) ** 2 for b in blocks)
    assert held < elems * 16  # below the complex128 matrices alone
    with pytest.raises(Exception):
        pc.block_matrix(0)  # released
    pc.assemble(tmat)  # a new assembly reallocates the blocks
    M0 = pc.block_matrix(0).cpu().numpy()
    assert M0.shape[0] == len(blocks[0]) * dev.nmax


@pytest.mark.parametrize("lmax,n,phi,cells", [(4, 160, 0.25, 3), (6, 40, 0.2, 2)])
def test_complex64_factorisation_matches_the_references_precision(cuda_device, lmax, n, phi, cells):
    """The default factorisation runs in complex64, as the reference's prepare does (scipy.linalg.lu
    on complex64 blocks, yasfpy/preconditioner.py:391, 445-468). The residual of the block system
    solved with our factors stays within a small factor of the residual left by scipy's complex64
    LU of the same blocks (the reference's own operation, run here on the host)."""
    import scipy.linalg as sla

    dev, tmat, blocks, rng = _setup(cuda_device, lmax, n, phi, cells, 40 + lmax)
    pc = DevicePreconditioner(dev, blocks)
    pc.assemble(tmat)
    mats = [pc.block_matrix(b).cpu().numpy() for b in range(len(blocks))]
    phases = pc.prepare(tmat)  # complex64 factorisation, complex128 blocks released
    assert set(phases) == {"assemble_s", "factor_s", "finalize_s"}
    with pytest.raises(Exception):
        pc.block_matrix(0)
    y = rng.normal(size=dev.n) + 1j * rng.normal(size=dev.n)
    My = _block_product(dev, mats, blocks, y)
    out = pc.apply(torch.from_numpy(My).to(cuda_device), YASF_C64).cpu().numpy()
    ours = np.linalg.norm(_block_product(dev, mats, blocks, out) - My)
    # the reference's complex64 LU of every block, applied in complex64
    ref = np.zeros_like(My)
    nmax = dev.nmax
    for M, blk in zip(mats, blocks):
        idx = (blk[:, None] * nmax + np.arange(nmax)[None, :]).ravel()
        lu = sla.lu_factor(M.astype(np.complex64))
        ref[idx] = sla.lu_solve(lu, My[idx].astype(np.complex64))
    theirs = np.linalg.norm(_block_product(dev, mats, blocks, ref) - My)
    assert ours <= 10 * theirs + 1e-12 * np.linalg.norm(My), (ours, theirs)
    assert ours < 1e-4 * np.linalg.norm(My)
