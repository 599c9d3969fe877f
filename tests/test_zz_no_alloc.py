"""The no-allocation coupling matvec (yasf_coupling_matvec_noalloc) against the regular one.

It exists for callers that cannot allocate device memory when they call (memory reserved once at
start-up, an embedding runtime that owns the allocator, fixed buffers only): its scratch is one
static device array. This file is collected last on purpose, so a run that stops at the first
failure has already run every other test; it also passes alone in a fresh process.
"""

from __future__ import annotations


import numpy as np
import pytest
import torch
from conftest import rel_err

from yasf_b200 import _lib
from yasf_b200._lib import YASF_C64, YASF_C128
from yasf_b200.device import CouplingDevice, _ptr, _stream_ptr
from yasf_b200.wigner import translation_table_ab5
from yasf_b200.workloads import rsa_cube

pytestmark = pytest.mark.gpu


def _noalloc(dev: CouplingDevice, x: torch.Tensor, precision: int = YASF_C128) -> tuple[int, torch.Tensor]:
    y = torch.full_like(x, complex("nan"))
    st = _lib.load().yasf_coupling_matvec_noalloc(dev.plan.handle, dev.n_particles, _ptr(dev.pos),
                                                  dev.k, _ptr(x), _ptr(y), precision, _stream_ptr())
    return st, y


def test_noalloc_matches_regular_entry_point_twice(cuda_device):
    lmax, n = 4, 40
    rng = np.random.default_rng(21)
    radii = rng.uniform(0.05, 0.12, size=n)
    pos = rsa_cube(radii, 0.15, rng)
    dev = CouplingDevice(lmax, translation_table_ab5(lmax), pos, 2 * np.pi / 0.55, cuda_device)
    need = dev.coupling_ws_bytes(YASF_C128)
    assert need <= 64 * 1024 * 1024
    for call in range(2):  # two calls in a row: the shared scratch keeps the previous contents
        x = torch.from_numpy(rng.normal(size=dev.n) + 1j * rng.normal(size=dev.n)).to(cuda_device)
        st, y = _noalloc(dev, x)
        assert st == 0, _lib.load().yasf_status_string(st)
        ref = dev.coupling(x)  # regular entry point, caller-provided workspace
        torch.cuda.synchronize()
        assert rel_err(y.cpu().numpy(), ref.cpu().numpy()) < 1e-12, f"call {call}"


def _aggregate(device, lmax, n, seed):
    rng = np.random.default_rng(seed)
    radii = rng.uniform(0.05, 0.12, size=n)
    pos = rsa_cube(radii, 0.15, rng)
    return CouplingDevice(lmax, translation_table_ab5(lmax), pos, 2 * np.pi / 0.55, device), rng


def test_noalloc_smaller_problem_after_larger_one(cuda_device):
    # The shared scratch keeps what the larger call left; the smaller call must not read any of it
    # (its stream and partial sums are written in full before they are read).
    big, rng = _aggregate(cuda_device, 5, 120, 31)
    small, _ = _aggregate(cuda_device, 3, 17, 32)
    assert big.coupling_ws_bytes(YASF_C128) > small.coupling_ws_bytes(YASF_C128)
    assert big.coupling_ws_bytes(YASF_C128) <= 64 * 1024 * 1024
    for dev in (big, small, big, small):  # all on the current stream, in order
        x = torch.from_numpy(rng.normal(size=dev.n) + 1j * rng.normal(size=dev.n)).to(cuda_device)
        st, y = _noalloc(dev, x)
        assert st == 0, _lib.load().yasf_status_string(st)
        ref = dev.coupling(x)
        torch.cuda.synchronize()
        assert rel_err(y.cpu().numpy(), ref.cpu().numpy()) < 1e-12


def test_noalloc_complex64_matches_regular_complex64(cuda_device):
    dev, rng = _aggregate(cuda_device, 4, 60, 33)
    for call in range(2):
        x = torch.from_numpy(rng.normal(size=dev.n) + 1j * rng.normal(size=dev.n)).to(cuda_device)
        st, y = _noalloc(dev, x, YASF_C64)
        assert st == 0, _lib.load().yasf_status_string(st)
        ref = dev.coupling(x, YASF_C64)  # regular complex64 call, caller-provided workspace
        torch.cuda.synchronize()
        assert rel_err(y.cpu().numpy(), ref.cpu().numpy()) < 2e-5, f"call {call}"


def test_noalloc_rejects_problems_beyond_the_static_scratch(cuda_device):
    lmax, n = 6, 600  # needs ~ 90 MB of scratch
    rng = np.random.default_rng(5)
    radii = rng.uniform(0.05, 0.1, size=n)
    pos = rsa_cube(radii, 0.1, rng)
    dev = CouplingDevice(lmax, translation_table_ab5(lmax), pos, 2 * np.pi / 0.6, cuda_device)
    assert dev.coupling_ws_bytes(YASF_C128) > 64 * 1024 * 1024
    x = torch.zeros(dev.n, dtype=torch.complex128, device=cuda_device)
    st, y = _noalloc(dev, x)
    assert st == 9  # YASF_ERR_SCRATCH_LIMIT, nothing launched
    assert torch.isnan(y.real).all()  # output untouched (sentinel real parts are NaN)
