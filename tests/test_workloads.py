"""The seeded synthetic inputs that stand in for the reference's benchmark data (no dataset):
random-sequential-addition packings, the named aggregates, Fibonacci incidence sets and the
serving request stream (CPU only)."""

from __future__ import annotations

import numpy as np
import pytest

from yasf_b200.workloads import aggregate_c1, incidences, rsa_ball, rsa_cube, serving_requests


def _no_overlap(pos, radii):
    d = np.linalg.norm(pos[:, None, :] - pos[None, :, :], axis=-1)
    gap = d - (radii[:, None] + radii[None, :])
    np.fill_diagonal(gap, np.inf)
    return gap.min()


@pytest.mark.parametrize("shape", ["cube", "ball"])
def test_rsa_packing_is_valid_and_seeded(shape):
    rng = np.random.default_rng(7)
    radii = rng.uniform(0.05, 0.15, size=300)
    phi = 0.15
    fn = rsa_cube if shape == "cube" else rsa_ball
    pos = fn(radii, phi, np.random.default_rng(1))
    assert pos.shape == (300, 3)
    assert _no_overlap(pos, radii) >= -1e-12
    vol = np.sum(4.0 / 3.0 * np.pi * radii**3)
    if shape == "cube":
        side = (vol / phi) ** (1.0 / 3.0)
        assert np.all(pos - radii[:, None] >= -1e-12) and np.all(pos + radii[:, None] <= side + 1e-12)
    else:
        R = (np.sum(radii**3) / phi) ** (1.0 / 3.0)
        assert np.all(np.linalg.norm(pos, axis=1) + radii <= R + 1e-12)
        assert abs(vol / (4.0 / 3.0 * np.pi * R**3) - phi) < 1e-12
    np.testing.assert_array_equal(pos, fn(radii, phi, np.random.default_rng(1)))


def test_aggregate_c1_matches_its_specification():
    a = aggregate_c1(seed=0)
    assert a.n == 100 and a.lmax == 4 and a.wavelength == 0.55 and a.refractive_index == 1.5 + 0.01j
    assert a.radii.min() >= 0.05 and a.radii.max() <= 0.15
    assert _no_overlap(a.positions, a.radii) >= -1e-12
    assert abs(a.k - 2 * np.pi / 0.55) < 1e-15
    np.testing.assert_array_equal(a.positions, aggregate_c1(seed=0).positions)


def test_incidences_are_fibonacci_directions_times_te_tm():
    polar, azim, pol = incidences(64)
    assert polar.shape == azim.shape == pol.shape == (128,)
    np.testing.assert_array_equal(pol, np.tile([1, 2], 64))
    np.testing.assert_array_equal(polar[0::2], polar[1::2])
    assert np.all((polar >= 0) & (polar <= np.pi))
    v = np.stack((np.sin(polar) * np.cos(azim), np.sin(polar) * np.sin(azim), np.cos(polar)), 1)[0::2]
    d = np.linalg.norm(v[:, None] - v[None, :], axis=-1) + 10 * np.eye(64)
    assert d.min() > 0.1  # 64 well-separated directions
    pr, ar, _ = incidences(64, rotation_seed=3)
    vr = np.stack((np.sin(pr) * np.cos(ar), np.sin(pr) * np.sin(ar), np.cos(pr)), 1)[0::2]
    np.testing.assert_allclose(np.sort(np.linalg.norm(vr[:, None] - vr[None, :], axis=-1).ravel()),
                               np.sort((d - 10 * np.eye(64)).ravel()), atol=1e-12)  # a rotation


def test_serving_stream_prefix_and_ranges():
    short = serving_requests(6)
    long = serving_requests(12)
    for a, b in zip(short, long):
        assert a.arrival == b.arrival and a.aggregate.n == b.aggregate.n
        np.testing.assert_array_equal(a.aggregate.positions, b.aggregate.positions)
    arr = [r.arrival for r in long]
    assert arr[0] == 0.0 and all(x < y for x, y in zip(arr, arr[1:]))
    for r in long:
        agg = r.aggregate
        assert 50 <= agg.n <= 3000 and agg.lmax in (3, 4, 5, 6, 7, 8)
        assert len(r.pol) in (1, 2, 16, 64) and len(r.polar) == len(r.pol)
        assert 0.4 <= agg.wavelength <= 0.8 and 1.3 <= agg.refractive_index.real <= 1.8
        assert 1e-4 <= agg.refractive_index.imag <= 1e-1
        assert _no_overlap(agg.positions, agg.radii) >= -1e-12
