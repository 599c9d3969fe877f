"""The (lmax, N, R) autotuner's host logic: keys and buckets, the cheapest-candidate rule, caching
(no second measurement for a key, thread-safe), and JSON persistence. The measurement itself is
replaced by a stand-in; tests/test_gpu_autotune.py times real operators."""

from __future__ import annotations

import threading

from yasf_b200.autotune import Autotuner, choose, n_bucket


class FakeDev:
    def __init__(self, lmax, n):
        self.lmax, self.n_particles = lmax, n


def test_choose_and_buckets():
    assert choose({"c64/w2": 30.0, "tf32/g0": 12.0}) == "tf32/g0"
    assert choose({"c64/w2": 3.0, "tf32/g0": 12.0, "f64/c32": 1.0}) == "c64/w2"  # residual tiles apart
    assert n_bucket(2000) == n_bucket(2050)
    assert n_bucket(2000) != n_bucket(2600)


def test_cache_and_persistence(tmp_path):
    calls = []

    def measure(dev, tmat, nrhs):
        calls.append((dev.lmax, dev.n_particles, nrhs))
        # a shape without a panel candidate (fake: lmax 9) decides among what was measured
        c = {"c64/w1": 6.0 * nrhs, "c64/w2": 5.0 * nrhs, "c64/w4": 5.5 * nrhs}
        if dev.lmax <= 8:
            c.update({"tf32/g1": 41.0, "tf32/g2": 40.0, "f64/c32": 9.0, "f64/c64": 7.0})
        return c

    path = tmp_path / "tune.json"
    t = Autotuner(path=path, measure=measure)
    assert t.decide(FakeDev(6, 2000), None, 1).inner == "c64"
    assert t.decide(FakeDev(6, 2000), None, 64).inner == "tf32"
    assert t.decide(FakeDev(6, 2030), None, 64).inner == "tf32"   # same bucket: cached
    assert t.decide(FakeDev(9, 2000), None, 64).inner == "c64"    # no panel candidate
    assert len(calls) == 3
    t2 = Autotuner(path=path, measure=measure)
    assert t2.decide(FakeDev(6, 2000), None, 64).inner == "tf32"
    assert len(calls) == 3                                          # loaded, not re-measured
    assert {tuple(d.key) for d in t2.decisions()} == {tuple(d.key) for d in t.decisions()}


def test_concurrent_decisions_agree():
    def measure(dev, tmat, nrhs):
        return {"c64": 1.0, "tf32": 2.0}

    t = Autotuner(measure=measure)
    out = []
    th = [threading.Thread(target=lambda: out.append(t.decide(FakeDev(5, 900), None, 16).inner)) for _ in range(8)]
    for x in th:
        x.start()
    for x in th:
        x.join()
    assert out == ["c64"] * 8 and len(t.decisions()) == 1


def test_decision_carries_tile_shapes(tmp_path):
    from yasf_b200.autotune import decision_from

    d = decision_from({"c64/w1": 3.0, "c64/w4": 2.0, "tf32/g0": 9.0, "f64/c32": 4.0, "f64/c64": 5.0}, (6, 1, 2))
    assert d.inner == "c64" and d.tiles == {"contract_waves": 4, "dpanel_cols": 32}
    d = decision_from({"c64/w2": 30.0, "tf32/g1": 9.0, "tf32/g2": 8.0}, (6, 1, 128))
    assert d.inner == "tf32" and d.tiles == {"panel_groups": 2}
    path = tmp_path / "t.json"
    t = Autotuner(path=path, measure=lambda dev, tm, r: {"c64/w1": 1.0, "tf32/g0": 2.0})
    assert t.decide(FakeDev(4, 500), None, 2).tiles == {"contract_waves": 1}
    assert Autotuner(path=path).decide(FakeDev(4, 500), None, 2).tiles == {"contract_waves": 1}
