"""Failure detection on the device: bounded waits that run out.

Every wait inside the library's kernels is bounded (the coupling contraction by a poll count, the
tensor-core and float64 dense panels and the preconditioner's one-launch sweeps by %globaltimer). When a wait runs out the kernel sets the
call's error word, writes NaN outputs, frees what it holds and returns, so the CUDA context stays
usable. The test hook ``yasf_test_stall`` keeps one producer role from ever delivering (a flag that
nothing sets) and shortens the bound, so each wait below runs out in milliseconds; nothing faults,
traps or spins without a bound. Each test then checks the error word, the NaN output, the status a
solve reports, and that the next normal call on the same context is correct.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch
from conftest import rel_err

from oracle import restate as R
from yasf_b200 import _lib
from yasf_b200._lib import (YASF_C64, YASF_STALL_CONTRACT, YASF_STALL_DPANEL, YASF_STALL_NONE, YASF_STALL_PANEL,
                            YASF_STALL_PRECOND, YasfError)
from yasf_b200.device import CouplingDevice
from yasf_b200.wigner import translation_table_ab5

pytestmark = pytest.mark.gpu

YASF_ERR_NOT_FINITE = 7


def _pair(device, lmax=3):
    pos = np.array([[0.0, 0.0, 0.0], [0.31, -0.12, 0.22]])
    table = translation_table_ab5(lmax)
    return CouplingDevice(lmax, table, pos, 2 * np.pi / 0.55, device), table, pos


def _error_word(dev: CouplingDevice, need: int) -> int:
    """The int at byte offset (required workspace bytes - 256) of the call's workspace."""
    return int(dev.ws.buf[need - 256:need - 252].view(torch.int32).item())


def _cols(rng, dev, R_, device):
    x = rng.normal(size=(R_, dev.n)) + 1j * rng.normal(size=(R_, dev.n))
    return torch.from_numpy(x).to(device)


def test_contraction_wait_runs_out(cuda_device):
    dev, table, pos = _pair(cuda_device)
    rng = np.random.default_rng(3)
    x = rng.normal(size=dev.n) + 1j * rng.normal(size=dev.n)
    xt = torch.from_numpy(x).to(cuda_device)
    tmat = torch.from_numpy(0.1 * (rng.normal(size=dev.n) + 1j * rng.normal(size=dev.n))).to(cuda_device)
    need = dev.coupling_ws_bytes()
    try:
        _lib.test_stall(YASF_STALL_CONTRACT, 4096, 0.0)
        y = dev.coupling(xt)
        torch.cuda.synchronize()
        err = _error_word(dev, need)
        b = xt.clone()
        x0 = xt.clone()
        with pytest.raises(YasfError) as info:
            dev.gmres(tmat, b, x0, 1e-8, 10, 3)
    finally:
        _lib.test_stall(YASF_STALL_NONE)
    assert err == 1
    assert torch.isnan(y.real).all() and torch.isnan(y.imag).all()
    assert info.value.status == YASF_ERR_NOT_FINITE
    # the context is still usable and the next call is correct
    y2 = dev.coupling(xt).cpu().numpy()
    assert _error_word(dev, need) == 0
    ref = R.coupling_matvec_rows(3, pos, dev.k, table, x)
    assert rel_err(y2, ref) < 1e-12


def test_panel_wait_runs_out(cuda_device):
    dev, table, pos = _pair(cuda_device)
    rng = np.random.default_rng(4)
    X = _cols(rng, dev, 64, cuda_device)
    nb = dev_panel_bytes(dev, 64)
    try:
        _lib.test_stall(YASF_STALL_PANEL, 0, 0.05)
        y = dev.panel(X)
        torch.cuda.synchronize()
        err = _error_word(dev, nb)
    finally:
        _lib.test_stall(YASF_STALL_NONE)
    assert err == 1
    assert torch.isnan(y.real).all()
    y2 = dev.panel(X)
    torch.cuda.synchronize()
    assert _error_word(dev, nb) == 0
    ref = dev.coupling(X)
    assert rel_err(y2.cpu().numpy(), ref.cpu().numpy()) < 5e-3


def test_dense_panel_wait_runs_out(cuda_device):
    dev, table, pos = _pair(cuda_device)
    rng = np.random.default_rng(5)
    X = _cols(rng, dev, 32, cuda_device)
    nb = dev_dpanel_bytes(dev, 32)
    try:
        _lib.test_stall(YASF_STALL_DPANEL, 0, 0.05)
        y = dev.dpanel(X)
        torch.cuda.synchronize()
        err = _error_word(dev, nb)
    finally:
        _lib.test_stall(YASF_STALL_NONE)
    assert err == 1
    assert torch.isnan(y.real).all()
    y2 = dev.dpanel(X)
    torch.cuda.synchronize()
    assert _error_word(dev, nb) == 0
    ref = dev.coupling(X)
    assert rel_err(y2.cpu().numpy(), ref.cpu().numpy()) < 1e-12


def test_preconditioner_sweep_wait_runs_out(cuda_device):
    from yasf_b200.device import DevicePreconditioner
    from yasf_b200.mie import mie_tmatrix_per_sphere
    from yasf_b200.workloads import rsa_cube

    rng = np.random.default_rng(6)
    lmax = 4
    radii = rng.uniform(0.06, 0.1, size=60)
    pos = rsa_cube(radii, 0.2, rng, largest_first=True)
    dev = CouplingDevice(lmax, translation_table_ab5(lmax), pos, 2 * np.pi / 0.55, cuda_device)
    tmat = torch.from_numpy(mie_tmatrix_per_sphere(lmax, dev.k, radii, 1.5 + 0.01j)).to(cuda_device)
    ext = pos.max(axis=0) - pos.min(axis=0)
    from yasf_b200.preconditioner import make_particle_partition

    pc = DevicePreconditioner(dev, make_particle_partition(pos, (ext + 2.0) / 2))
    pc.prepare(tmat)
    x = torch.from_numpy(rng.normal(size=dev.n) + 1j * rng.normal(size=dev.n)).to(cuda_device)
    good = pc.apply(x, YASF_C64)
    try:
        # the first tile row never delivers: the rows that wait on it give up after 50 ms
        _lib.test_stall(YASF_STALL_PRECOND, 0, 0.05)
        y = pc.apply(x, YASF_C64)
        torch.cuda.synchronize()
    finally:
        _lib.test_stall(YASF_STALL_NONE)
    assert torch.isnan(y.real).any()
    # the context is still usable and the next apply equals the one before the stall
    assert torch.equal(pc.apply(x, YASF_C64), good)


def dev_panel_bytes(dev, R_):
    import ctypes

    nb = ctypes.c_size_t()
    _lib.call("yasf_panel_workspace_size", dev.plan.handle, dev.n_particles, R_, ctypes.byref(nb))
    return nb.value


def dev_dpanel_bytes(dev, R_):
    import ctypes

    nb = ctypes.c_size_t()
    _lib.call("yasf_dpanel_workspace_size", dev.plan.handle, dev.n_particles, R_, ctypes.byref(nb))
    return nb.value
