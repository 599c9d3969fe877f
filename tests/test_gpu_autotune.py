"""The autotuner on the GPU: it times the real inner operators of a problem, picks the cheaper one
(the TF32 panel wins at many columns, the complex64 column kernel at one column), and a serving
request solved with the tuned choice matches the fixed-rule solve to the serving tolerance."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from yasf_b200.autotune import Autotuner
from yasf_b200.device import CouplingDevice
from yasf_b200.serve import ServeConfig, solve_request
from yasf_b200.wigner import translation_table_ab5
from yasf_b200.workloads import Aggregate, Request, incidences, rsa_cube

pytestmark = pytest.mark.gpu


def test_tuned_choice_by_columns(cuda_device):
    rng = np.random.default_rng(21)
    radii = rng.uniform(0.05, 0.12, size=300)
    pos = rsa_cube(radii, 0.15, rng)
    dev = CouplingDevice(5, translation_table_ab5(5), pos, 2 * np.pi / 0.55, cuda_device)
    tmat = torch.from_numpy(0.2 * (rng.normal(size=dev.n) + 1j * rng.normal(size=dev.n))).to(cuda_device)
    t = Autotuner()
    d1, d64 = t.decide(dev, tmat, 1), t.decide(dev, tmat, 64)
    # every candidate (inner operator x tile shape) timed: contraction waves, panel, dense-panel tiles
    assert {"c64/w1", "c64/w2", "c64/w4", "tf32/g0", "f64/c32", "f64/c64"} == set(d64.ms_per_step)
    assert all(v > 0 for v in d64.ms_per_step.values())
    assert d64.inner == "tf32" and d1.inner == "c64"
    assert d1.tiles.get("contract_waves") in (1, 2, 4) and d64.tiles.get("dpanel_cols") in (32, 64)


def test_tile_shapes_give_the_same_products(cuda_device):
    """Tile shapes change only how the work is split: every shape gives the same coupling product
    (float64: identical partial-sum layout per chunk count, so agreement to rounding), the same
    dense-panel result and the same tensor-core panel result."""
    from conftest import rel_err

    from yasf_b200._lib import set_tiles

    rng = np.random.default_rng(3)
    radii = rng.uniform(0.05, 0.12, size=150)
    pos = rsa_cube(radii, 0.15, rng)
    dev = CouplingDevice(4, translation_table_ab5(4), pos, 2 * np.pi / 0.55, cuda_device)
    x = torch.from_numpy(rng.normal(size=(130, dev.n)) + 1j * rng.normal(size=(130, dev.n))).to(cuda_device)
    ref = dev.coupling(x[0]).cpu().numpy()
    refd = dev.dpanel(x[:40]).cpu().numpy()
    refp = dev.panel(x).cpu().numpy()
    try:
        for w in (1, 2, 4, 8):
            set_tiles(w, 0, 0)
            assert rel_err(dev.coupling(x[0]).cpu().numpy(), ref) < 1e-13
        for c in (32, 64):
            set_tiles(0, c, 0)
            assert rel_err(dev.dpanel(x[:40]).cpu().numpy(), refd) < 1e-13
        for g in (1, 2):
            set_tiles(0, 0, g)
            assert rel_err(dev.panel(x).cpu().numpy(), refp) < 1e-6
    finally:
        set_tiles(0, 0, 0)


def test_tuned_request_matches_rule(cuda_device):
    rng = np.random.default_rng(5)
    radii = rng.uniform(0.05, 0.12, size=40)
    agg = Aggregate("t", rsa_cube(radii, 0.15, rng), radii, 1.5 + 0.01j, 0.55, 4, 5)
    polar, azim, pol = incidences(8)
    req = Request(0, 0.0, agg, polar, azim, pol)
    a = solve_request(req, ServeConfig(rtol=1e-8), cuda_device)
    b = solve_request(req, ServeConfig(rtol=1e-8, tuner=Autotuner()), cuda_device)
    assert b.stats["inner"] in ("tf32", "c64")
    assert np.allclose(a.c_ext, b.c_ext, rtol=1e-6, atol=0)
