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
    assert set(d64.ms_per_step) == {"c64", "tf32"} and all(v > 0 for v in d64.ms_per_step.values())
    assert d64.inner == "tf32" and d1.inner == "c64"


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
