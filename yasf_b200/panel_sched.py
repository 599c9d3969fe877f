"""Build step: the W-generation schedule of the tensor-core panel kernel (lmax 1..8).

The panel kernel forms, for every ordered sphere pair (i, j), the two translation blocks of the
tau-symmetric coupling, Wa (tau1 = tau2) and Wb (tau1 != tau2), and stores P = Wa + Wb and
Q = Wa - Wb in shared memory as TF32 tensor-core operands. With the pair table
G[p][d] = A[p][|d|] e^{i d phi}, A[p][d] = Pn_p^d(cos theta) h_p(k r), entry (q1, q2) of both
blocks is a short sum over the orders p (d = m2 - m1):

    Wa[q1][q2] = e^{i d phi} sum_p a_p A[p][|d|],   p in [pmin, l1 + l2], l1 + l2 + p even
    Wb[q1][q2] = i e^{i d phi} sum_p b_p A[p][|d|], p in [pmin, l1 + l2], l1 + l2 + p odd

with a_p, b_p real and pmin = max(|l1 - l2|, |d|) (3j selection rules; the coefficients are the
a5/b5 table of the plan). The mirror entry (l1, -m1), (l2, -m2) has the same a_p, the negated
b_p and the conjugate phase, so one generator thread computes an item (an entry and its mirror)
from one set of pair-table loads. This module fixes, at build time, which item each of the 512
generator threads computes in which step so that

- the 32 lanes of a warp always store to 32 different shared-memory banks: the primary entries of
  one step cover all 32 classes (q1 mod 8, q2 mod 4) of the K-major operand layout, and the mirror
  class (c - q1, 2 - q2) (mod 8, mod 4) is a bijection of the primary class for the items of a
  step, which share c (c depends on l1 only),
- the number of Wa and Wb terms of a step is the same for all lanes and all 16 warps (a step's
  lanes are padded with zero terms to the step's maximum), so the kernel's generation code is
  straight-line code with compile-time register indices and no per-term branches.

Lanes without an item of their class in a step write zeros to a padding entry (row or column
beyond the lmax(lmax+2) modes) of that class, or recompute an item that another lane also
computes (same values, same addresses). The output header holds, per lmax, the step table as a
macro list, the (warp, step, lane) -> primary entry table used by the plan to lay out
coefficients, the term windows of the packed variant (``window_starts``) and, up to lmax 6, the
pair-table entry each thread reads in each slot (``slot_tables``).
"""

from __future__ import annotations

import random
from collections import defaultdict
from pathlib import Path

WARPS = 16  # generator warps of the panel kernel


def _lm(q: int) -> tuple[int, int]:
    l = 1
    while (l + 1) * (l + 1) - 1 <= q:
        l += 1
    return l, q + 1 - l * l - l


def term_counts(L: int, q1: int, q2: int) -> tuple[int, int]:
    """(Wa terms, Wb terms) of entry (q1, q2) under the selection rules."""
    l1, m1 = _lm(q1)
    l2, m2 = _lm(q2)
    pmin = max(abs(l1 - l2), abs(m2 - m1))
    ps = range(pmin, l1 + l2 + 1)
    na = sum(1 for p in ps if (l1 + l2 + p) % 2 == 0)
    return na, len(ps) - na


def mirror(q: int) -> int:
    """Mode index of (l, -m) for the mode (l, m) at index q."""
    l, m = _lm(q)
    return l * l + l - 1 - m


def _mirror_shift(q1: int) -> int:
    """c with mirror(q1) = c - q1 (mod 8); mirror(q2) = 2 - q2 (mod 4) for every q2."""
    l, _ = _lm(q1)
    return (2 * (l * l + l - 1)) % 8


def schedule(L: int):
    """(steps, table): steps = [(Wa slots, Wb slots)], table[warp][step][lane] = (q1, q2).

    One lane computes an item: an entry (q1, q2) and its mirror (mirror(q1), mirror(q2)), whose Wa
    coefficients are equal and whose Wb coefficients are negated; the lane stores both. The
    primary entries of a group cover the 32 bank classes once, and because the mirror class is
    (c - a, 2 - b) for the primary class (a, b), groups whose items share c store their mirrors to
    32 different banks as well.
    """
    H = L * (L + 2)
    HP = (H + 7) // 8 * 8
    items, seen = [], set()
    for q1 in range(H):
        for q2 in range(H):
            if (q1, q2) in seen:
                continue
            e, m = (q1, q2), (mirror(q1), mirror(q2))
            seen.add(e)
            seen.add(m)
            na, nb = term_counts(L, q1, q2)
            items.append({"e": e, "m": m, "na": na, "nb": nb, "c": _mirror_shift(q1)})
    # orientation: balance the primary-class counts within each c-set, heavy items first
    count = defaultdict(int)
    for it in sorted(items, key=lambda x: (-(x["na"] + x["nb"]), x["e"])):
        ce = (it["c"], it["e"][0] & 7, it["e"][1] & 3)
        cm = (it["c"], it["m"][0] & 7, it["m"][1] & 3)
        if it["e"] != it["m"] and count[cm] < count[ce]:
            it["e"], it["m"] = it["m"], it["e"]
            ce = cm
        count[ce] += 1
    groups = []
    for c in sorted({it["c"] for it in items}):
        classes = defaultdict(list)
        for it in items:
            if it["c"] == c:
                classes[(it["e"][0] & 7, it["e"][1] & 3)].append(it)
        for v in classes.values():
            v.sort(key=lambda x: (-(x["na"] + x["nb"]), -x["na"], x["e"]))
        n_groups = max(len(v) for v in classes.values())
        for g in range(n_groups):
            lanes = []
            for lane in range(32):
                cls = classes[(lane >> 2, lane & 3)]
                lanes.append(cls[g] if g < len(cls) else None)
            ta = max(x["na"] for x in lanes if x)
            tb = max(x["nb"] for x in lanes if x)
            groups.append((ta, tb, lanes, c))
    groups.sort(key=lambda x: (-(x[0] + x[1]), -x[0]))
    by_class = defaultdict(list)
    for it in items:
        by_class[(it["e"][0] & 7, it["e"][1] & 3)].append(it)
    padding = defaultdict(list)
    for q1 in range(HP):
        for q2 in range(HP):
            if q1 >= H or q2 >= H:
                padding[(q1 & 7, q2 & 3)].append((q1, q2))
    n_steps = (len(groups) + WARPS - 1) // WARPS
    steps, table = [], [[None] * n_steps for _ in range(WARPS)]
    for k in range(n_steps):
        block = groups[k * WARPS:(k + 1) * WARPS]
        ta = max(g[0] for g in block)
        tb = max(g[1] for g in block)
        steps.append((ta, tb))
        for w in range(WARPS):
            grp = block[w] if w < len(block) else block[0]  # idle warps recompute a step's group
            row = []
            for lane in range(32):
                it = grp[2][lane]
                if it is not None:
                    row.append(it["e"])
                    continue
                cls = (lane >> 2, lane & 3)
                if padding[cls]:  # zero entry of this class (its mirror is a padding entry too)
                    row.append(padding[cls][0])
                    continue
                # recompute an item of this class that another lane also computes (same values)
                cand = [x for x in by_class[cls] if x["na"] <= ta and x["nb"] <= tb]
                cand.sort(key=lambda x: x["c"] != grp[3])
                if not cand:
                    raise RuntimeError(f"lmax {L}: no store target for lane class {cls}")
                row.append(cand[0]["e"])
            table[w][k] = row
    return steps, table


def window_start(L: int, q1: int, q2: int, which: int, T: int) -> int:
    """First order p0 of a lane's window of T slots for the Wa (which=0) or Wb terms of (q1, q2).

    The packed generation reads slot q at table row p0 + 2q (column |d|), so the window must cover
    the item's own terms (same parity, stride 2) and stay inside rows 0 .. 2L + 1: rows p < |d|
    hold zeros and row 2L + 1 is the phase row of the pair table, both finite. The window starts
    at the item's first term and moves down by 2 until it fits. Padding entries (q1 or q2 beyond
    the modes) start at 0.
    """
    H = L * (L + 2)
    first = last = -1
    if q1 < H and q2 < H:
        l1, m1 = _lm(q1)
        l2, m2 = _lm(q2)
        pmin = max(abs(l1 - l2), abs(m2 - m1))
        ps = [p for p in range(pmin, l1 + l2 + 1) if ((l1 + l2 + p) % 2 == 0) == (which == 0)]
        if ps:
            first, last = ps[0], ps[-1]
    p0 = max(first, 0)
    while p0 >= 0 and p0 + 2 * (T - 1) > 2 * L + 1:
        p0 -= 2
    if p0 < 0 or (first >= 0 and p0 + 2 * (T - 1) < last):
        raise RuntimeError(f"lmax {L}: no term window for entry ({q1}, {q2})")
    return p0


def window_starts(L: int, steps, table):
    """[warp][step][lane] -> (p0 of the Wa window, p0 of the Wb window)."""
    return [[[(window_start(L, q1, q2, 0, steps[k][0]), window_start(L, q1, q2, 1, steps[k][1]))
              for (q1, q2) in table[w][k]] for k in range(len(steps))] for w in range(WARPS)]


def _terms(L: int, q1: int, q2: int):
    """Pair-table entries (p P + |d|) of the Wa and Wb terms of entry (q1, q2), in order of p."""
    H, P = L * (L + 2), 2 * L + 1
    if q1 >= H or q2 >= H:
        return [], []
    l1, m1 = _lm(q1)
    l2, m2 = _lm(q2)
    ad = abs(m2 - m1)
    ps = range(max(abs(l1 - l2), ad), l1 + l2 + 1)
    return ([p * P + ad for p in ps if (l1 + l2 + p) % 2 == 0],
            [p * P + ad for p in ps if (l1 + l2 + p) % 2 == 1])


def _wavefronts(addrs) -> int:
    """Shared-memory wavefronts of one half-warp's 8-byte loads (16 banks of 8 bytes)."""
    by_bank = {}
    for a in addrs:
        by_bank.setdefault(a % 16, set()).add(a)
    return max((len(v) for v in by_bank.values()), default=1)


def _place_half(lists, fixed, T, rng, tries):
    """Slots of one half-warp's terms for one part (Wa or Wb) of one step.

    lists[i]: the lane's terms; fixed[i]: True if their order is already fixed (the lane recomputes
    an item placed before: the terms keep that order, so both lanes add them in the same order and
    store the same values). A free lane may put its terms in any slots. Returns (wavefronts,
    rows) with rows[i][s] the entry read by lane i in slot s (None: zero coefficient)."""
    n = len(lists)
    best = None
    for _ in range(tries):
        rows = [[None] * T for _ in range(n)]
        order = sorted(range(n), key=lambda i: (not fixed[i], -len(lists[i]), rng.random()))

        def clash(s, t):
            return sum(1 for a in {rows[o][s] for o in range(n)} - {None, t} if a % 16 == t % 16)

        for i in order:
            ts = lists[i]
            if fixed[i]:
                # monotone placement of the fixed order: slots s_0 < s_1 < ... (small DP)
                m = len(ts)
                INF = 1 << 30
                cost = [[INF] * (T + 1) for _ in range(m + 1)]
                cost[0] = [0] * (T + 1)
                for j in range(1, m + 1):
                    for s in range(j, T + 1):
                        cost[j][s] = min(cost[j][s - 1], cost[j - 1][s - 1] + clash(s - 1, ts[j - 1]))
                s = T
                for j in range(m, 0, -1):
                    while cost[j][s] == cost[j][s - 1] and s - 1 >= j:
                        s -= 1
                    rows[i][s - 1] = ts[j - 1]
                    s -= 1
            else:
                free = list(range(T))
                for t in sorted(ts, key=lambda _: rng.random()):
                    sl = min(free, key=lambda s: (clash(s, t), rng.random()))
                    rows[i][sl] = t
                    free.remove(sl)
        total = sum(_wavefronts([r[s] for r in rows if r[s] is not None] or [0]) for s in range(T))
        if best is None or total < best[0]:
            best = (total, rows)
    return best


PAD = 0x100  # flag of a slot without a term of the lane (its entry is read with a zero coefficient)


def slot_tables(L: int, steps, table, tries: int = 24):
    """[warp][lane] -> the pair-table entry read in each of the S slots (lmax <= 6), | PAD on slots
    without a term of the lane.

    Up to lmax 6 every slot carries its own table offset, so a lane's terms may sit in any of the
    step's slots. The slots are chosen per half-warp so that the 16 lanes' 8-byte loads of a slot
    hit different banks (one wavefront); a slot without a term of the lane reads an entry another
    lane of the half-warp reads in that slot (a broadcast, zero coefficient). Items that occur in
    more than one lane (recomputed duplicates) keep the term order of their first placement.
    Deterministic (seeded)."""
    S = sum(a + b for a, b in steps)
    out = [[[0] * S for _ in range(32)] for _ in range(WARPS)]
    canon = {}
    base = 0
    for k, (ta, tb) in enumerate(steps):
        for w in range(WARPS):
            row = table[w][k]
            for part, T, off in ((0, ta, base), (1, tb, base + ta)):
                for h in range(2):
                    lanes = list(range(16 * h, 16 * h + 16))
                    keys = [(row[l], part) for l in lanes]
                    lists = [list(canon.get(key, _terms(L, *row[l])[part])) for key, l in zip(keys, lanes)]
                    fixed = [key in canon for key in keys]
                    # a lane repeated inside this half-warp takes the first lane's placement
                    first = {}
                    for i, key in enumerate(keys):
                        first.setdefault(key, i)
                    uniq = [i for i, key in enumerate(keys) if first[key] == i]
                    rng = random.Random((((L * 64 + k) * WARPS + w) * 2 + part) * 2 + h)
                    _, rows = _place_half([lists[i] for i in uniq], [fixed[i] for i in uniq], T, rng, tries)
                    placed = {keys[i]: rows[j] for j, i in enumerate(uniq)}
                    for s in range(T):
                        used = [r[s] for r in placed.values() if r[s] is not None]
                        pad = max(set(used), key=used.count) if used else 0
                        for i, l in enumerate(lanes):
                            e = placed[keys[i]][s]
                            out[w][l][off + s] = (pad | PAD) if e is None else e
                    for key, r in placed.items():
                        canon.setdefault(key, tuple(e for e in r if e is not None))
        base += ta + tb
    return out


def header_text(lmax_values=range(1, 9)) -> str:
    out = [
        "// Generated by yasf_b200/panel_sched.py at build time: the W-generation schedule of the",
        "// tensor-core panel kernel. Do not edit.",
        "#pragma once",
        "",
        "namespace yasf {",
        "",
        "template <int L>",
        "struct PanelSched;",
        "",
    ]
    for L in lmax_values:
        steps, table = schedule(L)
        slots = sum(a + b for a, b in steps)
        out.append(f"template <>\nstruct PanelSched<{L}> {{")
        out.append(f"  static constexpr int kSteps = {len(steps)};")
        out.append(f"  static constexpr int kSlots = {slots};")
        out.append(f"  static constexpr int kWarps = {WARPS};")
        out.append("};")
        items, base = [], 0
        for k, (ta, tb) in enumerate(steps):
            items.append(f"G({k}, {base}, {ta}, {tb})")
            base += ta + tb
        out.append("// (step, first slot, Wa slots, Wb slots)")
        out.append(f"#define YASF_PANEL_STEPS_{L}(G) " + " ".join(items))
        out.append(f"static const unsigned char kPanelStepWa{L}[{len(steps)}] = {{"
                   + ", ".join(str(a) for a, _ in steps) + "};")
        out.append(f"static const unsigned char kPanelStepWb{L}[{len(steps)}] = {{"
                   + ", ".join(str(b) for _, b in steps) + "};")
        flat = [(q1 << 8) | q2 for w in range(WARPS) for k in range(len(steps)) for (q1, q2) in table[w][k]]
        out.append("// primary entry (q1 << 8 | q2) of [warp][step][lane]")
        out.append(f"static const unsigned short kPanelEntry{L}[{len(flat)}] = {{")
        for i in range(0, len(flat), 16):
            out.append("    " + ", ".join(str(v) for v in flat[i:i + 16]) + ",")
        out.append("};")
        if L <= 6:
            st = slot_tables(L, steps, table)
            flat = [st[w][l][q] for w in range(WARPS) for l in range(32) for q in range(slots)]
            out.append("// pair-table entry read per slot (lmax <= 6; | 0x100: no term, zero coefficient),")
            out.append("// [warp][lane][slot]")
            out.append(f"static const unsigned short kPanelSlot{L}[{len(flat)}] = {{")
            for i in range(0, len(flat), 24):
                out.append("    " + ", ".join(str(v) for v in flat[i:i + 24]) + ",")
            out.append("};")
        else:
            out.append(f"static const unsigned short* const kPanelSlot{L} = nullptr;  // packed variant")
        win = window_starts(L, steps, table)
        flat = [a | (b << 8) for w in range(WARPS) for k in range(len(steps)) for (a, b) in win[w][k]]
        out.append("// term windows of the packed variant: p0 of Wa | p0 of Wb << 8, [warp][step][lane]")
        out.append(f"static const unsigned short kPanelWindow{L}[{len(flat)}] = {{")
        for i in range(0, len(flat), 16):
            out.append("    " + ", ".join(str(v) for v in flat[i:i + 16]) + ",")
        out.append("};")
        out.append("")
    out.append("}  // namespace yasf")
    out.append("")
    return "\n".join(out)


def write_header(path: Path) -> Path:
    text = header_text()
    path.parent.mkdir(parents=True, exist_ok=True)
    if not path.exists() or path.read_text() != text:
        path.write_text(text)
    return path


if __name__ == "__main__":
    import sys

    print(header_text() if len(sys.argv) < 2 else write_header(Path(sys.argv[1])))
