"""Integer QUBOs at the edge of the tensor-core form's exact-digit range.

The tensor-core form treats integer Q with sum|Q_ij| <= 2^22 as exact: every coefficient
the contraction sees is split into two base-2048 digits (d0 in [0, 2048), d1 in
[-2048, 2048], both exact in fp16), the products are exact in fp32, and every partial sum of
the 16 products stays below 2^23 in magnitude, so fp32 accumulation loses nothing.  The
cases below push that argument to its limits: the budget of 2^22 is spent on the
coefficients of one contraction row (d1 near -2048), spread over all 16 products of a row
(large addends of one sign), split between terms of opposite sign that cancel in the
accumulator (a small exact remainder under large addends), or spent on heavily tied
optima; one case sits exactly at 2^22 and one just above it (the error-bounded path).

Variable groups of the tensor-core form (MSB-first variable order): t = variables
0 .. n-16 (the tile index), y = n-15 .. n-9 (the 128 MMA rows), u = n-8 .. n-1 (the 256 MMA
columns).  Every case also carries pairs of t variables with E = -c when exactly one of
the pair is set, so that the minimum has many tied states in different records and the
tie rule decides the answer.
"""
from __future__ import annotations

import numpy as np

LIMIT = 1 << 22
KINDS = ("v_row", "v_spread", "cancel", "ties", "at_limit", "over_limit")


def groups(n: int):
    t = list(range(0, n - 15))
    y = list(range(n - 15, n - 8))
    u = list(range(n - 8, n))
    return t, y, u


def _split(total: int, parts: int, rng) -> np.ndarray:
    """`parts` positive integers with the given sum, uneven low bits."""
    w = rng.random(parts) + 0.5
    v = np.floor(w / w.sum() * total).astype(np.int64)
    v[0] += total - int(v.sum())
    return v


def make_case(n: int, kind: str, seed: int = 0) -> np.ndarray:
    """int64 Q (upper triangle + diagonal) of one boundary kind; sum|Q| as the kind states."""
    rng = np.random.default_rng(1000 * n + KINDS.index(kind) * 17 + seed)
    T, Y, U = groups(n)
    Q = np.zeros((n, n), np.int64)
    c = 50000 if kind == "ties" else 1 + int(rng.integers(0, 3))
    for a in range(0, len(T) - 1, 2):  # tied pairs among the t variables
        i, j = T[a], T[a + 1]
        Q[i, i] -= c
        Q[j, j] -= c
        Q[i, j] += 2 * c
    for _ in range(3 * n):  # light +-1 noise anywhere
        i, j = sorted(rng.integers(0, n, 2))
        Q[i, j] += int(rng.choice([-1, 1]))
    used = int(np.abs(Q).sum())
    if kind in ("v_row", "at_limit", "over_limit"):
        # one contraction row carries the rest of the budget: digit d1 of (V u)_0 near -2048
        target = LIMIT - 1 if kind == "v_row" else (LIMIT if kind == "at_limit" else LIMIT + 1)
        Q[Y[0], U] -= _split(target - used, len(U), rng)
    elif kind == "v_spread":
        # all 7 coupling rows and the column terms large and negative: 16 large addends of one
        # sign in every accumulator of the all-ones rows
        rest = LIMIT - 1 - used
        vpart = rest // 2
        w = _split(vpart, len(Y) * len(U), rng).reshape(len(Y), len(U))
        for a, i in enumerate(Y):
            Q[i, U] -= w[a]
        cpart = rest - vpart
        cu = _split(cpart // 2, len(U), rng)
        for b, j in enumerate(U):
            Q[j, j] -= cu[b]
        ct = _split(cpart - cpart // 2, len(T) * len(U), rng).reshape(len(T), len(U))
        for a, i in enumerate(T):
            Q[i, U] -= ct[a]
    elif kind == "cancel":
        # positive couplings of y_0 with u against negative column terms: the minimum sits where
        # both are switched on, the accumulator adding addends near +-2^20 to a small remainder
        rest = LIMIT - 1 - used
        big = rest // 3
        wp = _split(big, len(U), rng)
        wn = _split(big, len(U), rng)
        Q[Y[0], U] += wp
        for b, j in enumerate(U):
            Q[j, j] -= wn[b]
        # the row term of y_0 makes switching it on pay by a small margin
        Q[Y[0], Y[0]] -= rest - 2 * big
    elif kind == "ties":
        # heavy ties (c = 50000 above) and the remaining budget on one coupling row
        Q[Y[0], U] -= _split(LIMIT - 1 - used, len(U), rng)
    else:
        raise ValueError(kind)
    # noise that landed on a heavy entry changed the total: settle it on the largest entry
    target = {"at_limit": LIMIT, "over_limit": LIMIT + 1}.get(kind, LIMIT - 1)
    i, j = np.unravel_index(int(np.argmax(np.abs(Q))), Q.shape)
    Q[i, j] += int(np.sign(Q[i, j])) * (target - abs_sum(Q))
    assert abs_sum(Q) == target
    return Q


def abs_sum(Q: np.ndarray) -> int:
    return int(np.abs(Q.astype(np.int64)).sum())


def coupling_sums(Q: np.ndarray) -> np.ndarray:
    """|(V u)_i| at u = all ones for each contraction row i (W = Q + Q^T off the diagonal)."""
    n = Q.shape[0]
    _, Y, U = groups(n)
    W = Q.astype(np.int64) + Q.astype(np.int64).T
    return np.array([abs(int(W[i, U].sum())) for i in Y])
