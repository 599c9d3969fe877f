"""The block-Jacobi factorisation and apply as the kernels perform them, emulated in numpy (no GPU).

The device code (yasf_b200/csrc/blocklu.cuh, precond.cu) factors every block by a right-looking
tile LU with 64 x 64 tiles: the diagonal tile with partial pivoting inside it, its L and U
inverses, the tile row as L_kk^{-1} (P A_kj) (interchanges only left of the diagonal), the tile
column as A_ik U_kk^{-1}, the trailing update. The one-column apply runs both triangular sweeps in
one launch whose blocks take tile rows by ticket and wait for the rows they depend on; it makes
progress in any scheduling order only if every row a ticket waits for holds a smaller ticket.
These tests emulate the same steps on ragged block orders and check P A = L U, that the sweeps
solve the block system, and the ticket rule on the C2 partition's real block orders. The kernels
themselves are checked against dense solves on the GPU (tests/test_gpu_precond_lu.py).
"""

from __future__ import annotations

import numpy as np
import pytest

T = 64


def _tile_lu(A0: np.ndarray):
    A = A0.copy()
    dim = A.shape[0]
    nt = -(-dim // T)
    piv = np.zeros(dim, dtype=int)
    Linv, Uinv = [], []
    for k in range(nt):
        k0 = k * T
        vk = min(T, dim - k0)
        t = A[k0:k0 + vk, k0:k0 + vk].copy()
        perm = np.arange(vk)
        for c in range(vk):  # partial pivoting inside the diagonal tile
            p = c + int(np.argmax(np.abs(t[c:, c])))
            if p != c:
                t[[c, p]] = t[[p, c]]
                perm[[c, p]] = perm[[p, c]]
            t[c + 1:, c] /= t[c, c]
            t[c + 1:, c + 1:] -= np.outer(t[c + 1:, c], t[c, c + 1:])
        A[k0:k0 + vk, k0:k0 + vk] = t
        piv[k0:k0 + vk] = perm
        li = np.linalg.inv(np.tril(t, -1) + np.eye(vk))
        ui = np.linalg.inv(np.triu(t))
        Linv.append(li)
        Uinv.append(ui)
        for j in range(nt):  # tile row k: interchanges, then L_kk^{-1} right of the diagonal
            if j == k:
                continue
            j0, vj = j * T, min(T, dim - j * T)
            blk = A[k0 + perm, j0:j0 + vj]
            A[k0:k0 + vk, j0:j0 + vj] = li @ blk if j > k else blk
        for i in range(k + 1, nt):  # tile column k
            i0, vi = i * T, min(T, dim - i * T)
            A[i0:i0 + vi, k0:k0 + vk] = A[i0:i0 + vi, k0:k0 + vk] @ ui
        for i in range(k + 1, nt):  # trailing update
            i0, vi = i * T, min(T, dim - i * T)
            for j in range(k + 1, nt):
                j0, vj = j * T, min(T, dim - j * T)
                A[i0:i0 + vi, j0:j0 + vj] -= A[i0:i0 + vi, k0:k0 + vk] @ A[k0:k0 + vk, j0:j0 + vj]
    P = np.concatenate([k * T + piv[k * T:k * T + min(T, dim - k * T)] for k in range(nt)])
    return A, P, Linv, Uinv


def _sweeps(LU: np.ndarray, P: np.ndarray, Linv, Uinv, b: np.ndarray) -> np.ndarray:
    """Gather with the pivots, forward rows z_i = Linv_i (z_i - sum_{j<i} L_ij z_j), backward rows
    z_i = Uinv_i (z_i - sum_{j>i} U_ij z_j): the row form of the one-launch solve."""
    dim = LU.shape[0]
    nt = -(-dim // T)
    z = b[P].astype(complex)
    sl = [slice(i * T, min(dim, (i + 1) * T)) for i in range(nt)]
    for i in range(nt):
        acc = sum((LU[sl[i], sl[j]] @ z[sl[j]] for j in range(i)), np.zeros(sl[i].stop - sl[i].start, complex))
        z[sl[i]] = Linv[i] @ (z[sl[i]] - acc)
    for i in reversed(range(nt)):
        acc = sum((LU[sl[i], sl[j]] @ z[sl[j]] for j in range(i + 1, nt)),
                  np.zeros(sl[i].stop - sl[i].start, complex))
        z[sl[i]] = Uinv[i] @ (z[sl[i]] - acc)
    return z


@pytest.mark.parametrize("dim", [64, 100, 3 * 64 + 32, 5 * 48])
def test_tile_lu_factors_and_sweeps_solve(dim):
    rng = np.random.default_rng(dim)
    M = np.eye(dim) + 0.3 * (rng.normal(size=(dim, dim)) + 1j * rng.normal(size=(dim, dim))) / np.sqrt(dim)
    LU, P, Linv, Uinv = _tile_lu(M)
    L = np.tril(LU, -1) + np.eye(dim)
    U = np.triu(LU)
    assert np.abs(M[P] - L @ U).max() <= 1e-12 * np.abs(M).max()
    # P permutes rows only within 64-row tile rows
    assert all(P[i] // T == i // T for i in range(dim))
    b = rng.normal(size=dim) + 1j * rng.normal(size=dim)
    x = _sweeps(LU, P, Linv, Uinv, b)
    assert np.linalg.norm(M @ x - b) <= 1e-11 * np.linalg.norm(b)


def _tickets(dims: list[int]):
    """(block, tile row) per ticket as the preconditioner builds them: forward rows ordered by row
    then block, then backward rows ordered by distance from the block's last row, then block."""
    nts = [-(-d // T) for d in dims]
    steps = max(nts)
    order = []
    for upper in (0, 1):
        for c in range(steps):
            for b, nt in enumerate(nts):
                if c < nt:
                    order.append((upper, b, nt - 1 - c if upper else c))
    return order, nts


def test_every_row_a_ticket_waits_for_holds_a_smaller_ticket():
    """On the C2 partition's block orders (4 x 4 x 4 cells of the 2000-sphere aggregate, lmax 6):
    a forward row waits for the earlier rows of its block, a backward row for its block's whole
    forward sweep and the later rows of its block; all of them come earlier in the ticket order,
    so the CTA holding the smallest unfinished ticket can always finish."""
    from yasf_b200.preconditioner import make_particle_partition
    from yasf_b200.workloads import aggregate_c2

    agg = aggregate_c2(seed=0)
    ext = agg.positions.max(axis=0) - agg.positions.min(axis=0)
    blocks = make_particle_partition(agg.positions, (ext + 2.0) / 4)
    dims = [len(b) * 96 for b in blocks]
    order, nts = _tickets(dims)
    ticket = {key: t for t, key in enumerate(order)}
    assert len(order) == 2 * sum(nts)
    for t, (upper, b, i) in enumerate(order):
        if upper:
            deps = [(0, b, r) for r in range(nts[b])] + [(1, b, j) for j in range(i + 1, nts[b])]
        else:
            deps = [(0, b, j) for j in range(i)]
        assert all(ticket[d] < t for d in deps)
