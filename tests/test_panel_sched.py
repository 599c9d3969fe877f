"""The build-time W-generation schedule of the tensor-core panel, checked on the host.

- structure: every entry of both W blocks is produced, and every warp's stores of a step hit 32
  different banks (primary entries; mirrors up to a few lanes that recompute padding),
- arithmetic: emulating the kernel's generation in float64 from the schedule (items of an entry
  and its mirror, the A[p][|d|] table, phases e^{i d phi}, P = Wa + Wb, Q = Wa - Wb) and its
  tau-symmetric product (S = X1 + X2, D = X1 - X2, Y1 = (U + V) / 2, Y2 = (U - V) / 2) reproduces
  the oracle's two-sphere coupling W_ij x_j to rounding. The emulation reads the pair table the
  way the kernel does: up to lmax 6 slot by slot from the schedule's slot table, for lmax 7 and 8
  slot q of a step at row p0 + 2q of the lane's term window (zero coefficients outside the item's
  terms); every read stays inside the written, finite part of the table,
- slot tables: a half-warp's loads of one slot are bank-conflict-free, and lanes that recompute
  one item add its terms in the same order.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import restate as R
from yasf_b200.panel_sched import PAD, WARPS, _lm, _wavefronts, mirror, schedule, slot_tables, window_starts
from yasf_b200.wigner import translation_table_ab5


@pytest.mark.parametrize("L", [1, 2, 3, 4, 5, 6, 7, 8])
def test_schedule_structure(L):
    steps, table = schedule(L)
    H = L * (L + 2)
    covered = set()
    collisions = 0
    for w in range(WARPS):
        for k in range(len(steps)):
            row = table[w][k]
            assert len({(q1 & 7, q2 & 3) for q1, q2 in row}) == 32
            mcls = [((mirror(q1) & 7, mirror(q2) & 3) if q1 < H and q2 < H else (q1 & 7, q2 & 3))
                    for q1, q2 in row]
            collisions += 32 - len(set(mcls))
            for q1, q2 in row:
                if q1 < H and q2 < H:
                    covered.add((q1, q2))
                    covered.add((mirror(q1), mirror(q2)))
    assert len(covered) == H * H
    assert collisions <= 4 * WARPS * len(steps)  # a few lanes per step, padding recomputation only


def _emulate_wx(L, table_ab5, ri, rj, k, xj, packed=False, blocks=False):
    H = L * (L + 2)
    P = 2 * L + 1
    d = np.asarray(ri) - np.asarray(rj)
    r = np.linalg.norm(d)
    ct, st = d[2] / r, np.hypot(d[0], d[1]) / r
    phi = np.arctan2(d[1], d[0])
    j, y = R.sph_bessel(P - 1, k * r)
    h = j + 1j * y
    leg = R.legendre(P - 1, ct, st)
    A = np.array([[leg[p, dd] * h[p] if dd <= p else 0 for dd in range(P)] for p in range(P)])
    # the kernel's pair table: A[p][d] at p P + d (zero for p < d), phases at P P + 2L + delta
    g = np.zeros(P * P + 4 * L + 1, dtype=complex)
    g[:P * P] = A.reshape(-1)
    g[P * P:] = np.exp(1j * np.arange(-2 * L, 2 * L + 1) * phi)
    steps, sched = schedule(L)
    win = window_starts(L, steps, sched)
    slots = None if packed else slot_tables(L, steps, sched)
    bases = np.cumsum([0] + [a + b for a, b in steps])
    Pm = np.full((H, H), np.nan, dtype=complex)
    Qm = np.full((H, H), np.nan, dtype=complex)
    tab = np.asarray(table_ab5)
    for w in range(WARPS):
        for kk in range(len(steps)):
            for q1, q2 in sched[w][kk]:
                if q1 >= H or q2 >= H:
                    continue
                l1, m1 = _lm(q1)
                l2, m2 = _lm(q2)
                dl = m2 - m1
                pmin = max(abs(l1 - l2), abs(dl))
                Sa = Sb = 0j
                if packed:
                    pa0, pb0 = win[w][kk][sched[w][kk].index((q1, q2))]
                    for which, (p0, T) in enumerate(((pa0, steps[kk][0]), (pb0, steps[kk][1]))):
                        for q in range(T):
                            p = p0 + 2 * q
                            idx = p * P + abs(dl)
                            assert 0 <= idx < g.size and np.isfinite(g[idx])
                            real = pmin <= p <= l1 + l2 and ((l1 + l2 + p) % 2 == 0) == (which == 0)
                            if which == 0:
                                Sa += (tab[q2, q1, p].real if real else 0.0) * g[idx]
                            else:
                                Sb += (tab[H + q2, q1, p].imag if real else 0.0) * g[idx]
                else:
                    # the kernel's reads: slot by slot from the schedule's slot table
                    lane = sched[w][kk].index((q1, q2))
                    seen = []
                    for s in range(bases[kk], bases[kk + 1]):
                        v = slots[w][lane][s]
                        idx = v & 0xFF
                        assert 0 <= idx < g.size and np.isfinite(g[idx])
                        if v & PAD:
                            continue
                        p, dd = divmod(idx, P)
                        assert dd == abs(dl) and pmin <= p <= l1 + l2
                        wa = (l1 + l2 + p) % 2 == 0
                        assert (s < bases[kk] + steps[kk][0]) == wa  # Wa terms in the Wa slots
                        seen.append(p)
                        if wa:
                            Sa += tab[q2, q1, p].real * g[idx]
                        else:
                            Sb += tab[H + q2, q1, p].imag * g[idx]
                    assert sorted(seen) == list(range(pmin, l1 + l2 + 1))
                E = np.exp(1j * dl * phi)
                Wa, Wb = E * Sa, 1j * E * Sb
                Pm[q1, q2], Qm[q1, q2] = Wa + Wb, Wa - Wb
                Wa2, Wb2 = np.conj(E) * Sa, -1j * np.conj(E) * Sb
                Pm[mirror(q1), mirror(q2)], Qm[mirror(q1), mirror(q2)] = Wa2 + Wb2, Wa2 - Wb2
    assert not np.isnan(Pm).any() and not np.isnan(Qm).any()
    if blocks:
        return Pm, Qm
    x1, x2 = xj[:H], xj[H:]
    U, V = Pm @ (x1 + x2), Qm @ (x1 - x2)
    return np.concatenate([(U + V) / 2, (U - V) / 2])


@pytest.mark.parametrize("L, packed", [(1, False), (2, False), (3, False), (4, False), (5, False), (6, False),
                                       (7, True), (8, True)])
def test_generation_algebra_matches_oracle(L, packed):
    rng = np.random.default_rng(L)
    tab = translation_table_ab5(L)
    k = 2 * np.pi / 0.55
    pos = np.array([[0.0, 0.0, 0.0], rng.normal(size=3) * 0.4])
    nmax = 2 * L * (L + 2)
    x = np.zeros(2 * nmax, dtype=complex)
    x[nmax:] = rng.normal(size=nmax) + 1j * rng.normal(size=nmax)
    ref = R.coupling_matvec_rows(L, pos, k, tab, x, 0, 1)
    got = _emulate_wx(L, tab, pos[0], pos[1], k, x[nmax:], packed=packed)
    assert np.max(np.abs(got - ref)) <= 1e-11 * np.max(np.abs(ref))


@pytest.mark.parametrize("L", [4, 5, 6])
def test_slot_tables_are_conflict_free(L):
    """A half-warp's 8-byte pair-table loads of one slot hit different banks (or one address), and
    lanes that recompute one item add its terms in one order (identical stores)."""
    steps, sched = schedule(L)
    st = slot_tables(L, steps, sched)
    S = sum(a + b for a, b in steps)
    extra = sum(_wavefronts([st[w][l][q] & 0xFF for l in range(16 * h, 16 * h + 16)]) - 1
                for w in range(WARPS) for h in range(2) for q in range(S))
    assert extra <= 0.02 * 2 * WARPS * S
    bases = np.cumsum([0] + [a + b for a, b in steps])
    order = {}
    for k in range(len(steps)):
        for w in range(WARPS):
            for lane, e in enumerate(sched[w][k]):
                seq = tuple(v for v in st[w][lane][bases[k]:bases[k + 1]] if not v & PAD)
                assert order.setdefault(e, seq) == seq


def test_slot_tables_are_deterministic():
    """The generated header (and with it the plan's coefficient layout) does not change between
    builds: the slot search is seeded."""
    steps, sched = schedule(5)
    assert slot_tables(5, steps, sched) == slot_tables(5, steps, sched)


@pytest.mark.parametrize("L", [3, 6])
def test_reverse_pair_blocks_are_sign_flipped_swaps(L):
    """With r_ji = -r_ij, A_ji[p][d] = (-1)^(p+d) A_ij[p][d] and the phase gains (-1)^d, so every
    term picks up (-1)^p: (-1)^(l1+l2) on Wa terms and -(-1)^(l1+l2) on Wb terms. Hence
    P_ji = s Q_ij and Q_ji = s P_ij entrywise with s = (-1)^(l1+l2): one generation per unordered
    pair could serve both directions."""
    rng = np.random.default_rng(11)
    tab = translation_table_ab5(L)
    k = 2 * np.pi / 0.55
    ri, rj = np.zeros(3), rng.normal(size=3) * 0.4
    H = L * (L + 2)
    Pij, Qij = _emulate_wx(L, tab, ri, rj, k, None, blocks=True)
    Pji, Qji = _emulate_wx(L, tab, rj, ri, k, None, blocks=True)
    ls = np.array([_lm(q)[0] for q in range(H)])
    sgn = (-1.0) ** (ls[:, None] + ls[None, :])
    scale = max(np.abs(Pij).max(), np.abs(Qij).max())
    assert np.max(np.abs(Pji - sgn * Qij)) <= 1e-12 * scale
    assert np.max(np.abs(Qji - sgn * Pij)) <= 1e-12 * scale
