"""Tensor-core form at the edge of its exact-digit range (sum|Q| <= 2^22), against the oracle.

At and below 2^22 the form runs with a zero error band (pass 2 re-walks only the records
whose fp32 pass-1 minimum equals the global one), so a single accumulation that lost an
integer bit would silently drop the true argmin.  Each case here is built to make that
happen if the tensor core's fp32 accumulation were not exact on integer addends below 2^23
(tests/tc_boundary_cases.py says how), and is compared bit for bit (state and energy) with
the C restatement of the reference's QBF loop, through the single-problem kernel and the
batched (multi-item) kernel.
"""
import numpy as np
import pytest

import oracle
import qubo_b200  # noqa: F401
import tc_boundary_cases as tcb
from qubo_b200 import _lib
from qubo_b200.problems import Just_Q
from qubo_b200.solvers import QBF

pytestmark = pytest.mark.gpu

CASES = [(n, k) for n in (24, 32, 36) for k in tcb.KINDS]
_REF = {}


def _case(n, kind, layout="upper"):
    Q = tcb.make_case(n, kind)
    if layout == "sym":  # the same W with every coupling split over Q_ij and Q_ji
        U = np.triu(Q, 1)
        lo = U // 2
        Q = np.diag(np.diag(Q)) + (U - lo) + lo.T
    return Q.astype(np.int32)


def _ref(n, kind, layout="upper"):
    key = (n, kind, layout)
    if key not in _REF:
        _REF[key] = oracle.qbf_port(_case(n, kind, layout))
    return _REF[key]


@pytest.mark.parametrize("n,kind", CASES, ids=[f"n{n}-{k}" for n, k in CASES])
def test_single_problem_kernel(cuda_ok, n, kind):
    Q = _case(n, kind)
    ref = _ref(n, kind)
    r = _lib.handle(0).solve(Q, form="tc")
    assert r["form"] == "tc"
    # at or below 2^22 the integer digits are exact and the error band is zero
    assert (r["err_bound"] == 0.0) == (kind != "over_limit"), r
    assert (r["best_X_int"], r["best_E_int"]) == (ref["best_X_int"], ref["best_E"]), (r, ref)
    assert r["candidate_records"] >= 1


@pytest.mark.parametrize("kind", ["v_row", "cancel", "at_limit"])
def test_symmetric_layout(cuda_ok, kind):
    Q = _case(32, kind, "sym")
    assert tcb.abs_sum(Q) == tcb.abs_sum(_case(32, kind))
    ref = _ref(32, kind, "sym")
    sol = QBF().solve(Just_Q(Q), device="cuda", form="tc")
    assert sol.search["form"] == "tc"
    x = int("".join(map(str, sol.best_X)), 2)
    assert (x, int(sol.best_E)) == (ref["best_X_int"], ref["best_E"])


def test_batched_kernel(cuda_ok):
    Qs = [_case(n, k) for n, k in CASES]
    res = _lib.handle(0).solve_batch(Qs)
    for (n, k), Q, r in zip(CASES, Qs, res):
        ref = _ref(n, k)
        assert r["form"] == "tc", (n, k, r["form"])
        assert (r["err_bound"] == 0.0) == (k != "over_limit"), (n, k, r)
        assert (r["best_X_int"], r["best_E_int"]) == (ref["best_X_int"], ref["best_E"]), (n, k, r, ref)


def test_batched_kernel_other_splits(cuda_ok):
    """The tie rule follows the split (A) on the boundary cases too."""
    Qs = [_case(n, k) for n in (24, 32) for k in ("ties", "cancel")]
    for A in (3, 11):
        res = _lib.handle(0).solve_batch(Qs, prefix_bits=A)
        for Q, r in zip(Qs, res):
            ref = oracle.qbf_port(Q, A=A)
            assert (r["best_X_int"], r["best_E_int"]) == (ref["best_X_int"], ref["best_E"])


@pytest.mark.parametrize("n,kind", [(24, "v_row"), (32, "cancel"), (36, "at_limit"), (32, "over_limit")])
def test_pair_kernel(cuda_ok, n, kind):
    """The tensor-core pair form (QB_FLAG_TC_PAIR: two states per accumulator) on the same
    edge cases: the same answer as the default one-state kernel and the oracle."""
    Q = _case(n, kind)
    ref = _ref(n, kind)
    h = _lib.handle(0)
    one = h.solve(Q, form="tc")
    two = h.solve(Q, form="tc", tc_pair=True)
    assert (one["best_X_int"], one["best_E_int"]) == (ref["best_X_int"], ref["best_E"])
    assert (two["best_X_int"], two["best_E_int"]) == (ref["best_X_int"], ref["best_E"])
    if kind != "over_limit":
        assert one["pass1_min"] == two["pass1_min"] == ref["best_E"]
