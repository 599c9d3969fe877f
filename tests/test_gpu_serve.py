"""Serving on the GPU: requests of different sizes solved concurrently (one stream each, kernels
interleaving on the device) give the same results as each request solved alone, and the
mixed-precision extinction cross sections stay within 1e-6 of a float64 solve."""

from __future__ import annotations

import numpy as np
import pytest
import torch
from conftest import rel_err

from yasf_b200.device import CouplingDevice
from yasf_b200.incident import plane_wave_block
from yasf_b200.mie import mie_tmatrix_per_sphere
from yasf_b200.serve import ServeConfig, Server, groupable, solve_group, solve_request, summarize
from yasf_b200.wigner import translation_table_ab5
from yasf_b200.workloads import Aggregate, Request, incidences, rsa_cube

pytestmark = pytest.mark.gpu


def _requests():
    out = []
    specs = [(40, 3, 1), (25, 5, 4), (60, 4, 2), (33, 6, 2), (18, 7, 1), (50, 3, 8)]
    for i, (n, lmax, R) in enumerate(specs):
        rng = np.random.default_rng(500 + i)
        radii = rng.uniform(0.05, 0.12, size=n)
        pos = rsa_cube(radii, 0.15, rng)
        agg = Aggregate(f"t{i}", pos, radii, complex(1.4 + 0.05 * i, 0.01), 0.5 + 0.03 * i, lmax, i)
        if R == 1:
            polar, azim, pol = np.array([0.3]), np.array([0.1]), np.array([1])
        else:
            polar, azim, pol = incidences(R // 2)
        out.append(Request(i, 0.0, agg, polar, azim, pol))
    return out


def test_results_same_alone_and_in_the_mix(cuda_device):
    cfg = ServeConfig(max_slots=4, rtol=1e-8, keep_solutions=True)
    reqs = _requests()
    mixed = Server(cfg, device=cuda_device).run(reqs, realtime=False)
    for r in mixed:
        assert r.error is None, r.error
    # a small complex64-inner request is solved by a grouped solve in the mix: alone it is a group
    # of one; every column's trajectory is its own, so the results agree bit for bit
    alone = [solve_group([q], cfg, cuda_device)[0] if groupable(q, cfg) else solve_request(q, cfg, cuda_device)
             for q in reqs]
    for m, a in zip(mixed, alone):
        assert m.rid == a.rid
        assert rel_err(m.x, a.x) <= 1e-12
        assert np.allclose(m.c_ext, a.c_ext, rtol=1e-12, atol=0)
    s = summarize(mixed)
    assert s["completed"] == len(reqs) and s["failed"] == 0


def test_mixed_precision_extinction_within_target(cuda_device):
    cfg = ServeConfig(max_slots=1, rtol=1e-6, keep_solutions=True)
    req = _requests()[1]
    res = solve_request(req, cfg, cuda_device)
    agg = req.aggregate
    dev = CouplingDevice(agg.lmax, translation_table_ab5(agg.lmax), agg.positions, agg.k, cuda_device)
    tm = mie_tmatrix_per_sphere(agg.lmax, agg.k, agg.radii, agg.refractive_index)
    a = plane_wave_block(agg.lmax, agg.positions, agg.k, req.polar, req.azimuthal, req.pol)
    tmat = torch.from_numpy(tm).to(cuda_device)
    for c in range(len(req.pol)):
        b = torch.from_numpy(np.ascontiguousarray(tm * a[:, :, c].ravel())).to(cuda_device)
        x = b.clone()
        st = dev.gmres(tmat, b, x, 1e-12, 100, 50)
        assert st["info"] == 0
        c64 = -np.real(np.vdot(a[:, :, c].ravel(), x.cpu().numpy())) / agg.k**2 * np.pi
        assert abs(res.c_ext[c] - c64) <= 1e-6 * abs(c64)


def test_admission_footprint_covers_the_device_memory_of_a_request(cuda_device):
    """The admission footprint (the library's workspace query plus the request's vectors) is at
    least the device memory a request's solve allocates, and not grossly more."""
    from yasf_b200.serve import footprint_bytes

    cfg = ServeConfig(max_slots=1, rtol=1e-6)
    for req in _requests()[:4]:
        fp = footprint_bytes(req, cfg, cuda_device)
        solve_request(req, cfg, cuda_device)  # plans, kernels and caches set up
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        base = torch.cuda.memory_allocated(cuda_device)
        torch.cuda.reset_peak_memory_stats(cuda_device)
        solve_request(req, cfg, cuda_device)
        torch.cuda.synchronize()
        peak = torch.cuda.max_memory_allocated(cuda_device) - base
        assert peak <= fp, (req.rid, peak, fp)
        assert fp <= 2 * peak + (16 << 20), (req.rid, peak, fp)


def _small_requests():
    reqs = []
    for i, (n, R) in enumerate([(30, 1), (80, 2), (12, 1), (55, 2), (41, 1)]):
        rng = np.random.default_rng(700 + i)
        radii = rng.uniform(0.05, 0.12, size=n)
        pos = rsa_cube(radii, 0.15, rng)
        agg = Aggregate(f"g{i}", pos, radii, complex(1.45 + 0.02 * i, 0.01), 0.5 + 0.02 * i, 4, i)
        polar, azim, pol = incidences(1)
        reqs.append(Request(i, 0.0, agg, polar[:R], azim[:R], pol[:R]))
    return reqs


def test_group_footprint_covers_the_device_memory_of_a_group(cuda_device):
    """A group is admitted by the grouped solve's own size query plus its requests' vectors: at
    least the device memory the grouped solve allocates."""
    from yasf_b200.serve import group_footprint_bytes

    reqs = _small_requests()
    cfg = ServeConfig(max_slots=1, rtol=1e-6)
    fp = group_footprint_bytes(reqs, cfg, cuda_device)
    solve_group(reqs, cfg, cuda_device)  # plans and caches set up
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    base = torch.cuda.memory_allocated(cuda_device)
    torch.cuda.reset_peak_memory_stats(cuda_device)
    out = solve_group(reqs, cfg, cuda_device)
    torch.cuda.synchronize()
    peak = torch.cuda.max_memory_allocated(cuda_device) - base
    assert all(r.error is None for r in out)
    assert peak <= fp, (peak, fp)


def test_small_requests_grouped_equal_alone(cuda_device):
    """Five small requests of one lmax arriving together are served by one grouped solve; each
    result equals that request solved alone (a group of one), and the float64 solve within 1e-6."""
    reqs = _small_requests()
    cfg = ServeConfig(max_slots=2, rtol=1e-8, keep_solutions=True)
    assert all(groupable(q, cfg) for q in reqs)
    mixed = Server(cfg, device=cuda_device).run(reqs, realtime=False)
    sizes = {r.stats.get("group_size") for r in mixed}
    assert max(sizes) > 1  # at least one group of several requests
    for r, q in zip(mixed, reqs):
        assert r.error is None, r.error
        alone = solve_group([q], cfg, cuda_device)[0]
        assert rel_err(r.x, alone.x) <= 1e-12
        assert np.allclose(r.c_ext, alone.c_ext, rtol=1e-12, atol=0)
