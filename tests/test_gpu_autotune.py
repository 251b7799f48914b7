"""qb_autotune: times the Gray-code form over its prefix/suffix split and record granularity
and the tensor-core form over its record granularity on the device, keeps the fastest per
(dtype class, n) in the handle; QB_FORM_AUTO then uses that form, every solve of the class
and n uses the tuned parameters (single and batched searches), results report them, and
answers stay equal to the oracle's."""
import numpy as np
import pytest

import oracle
import qubo_b200  # noqa: F401
from qubo_b200 import _lib
from qubo_b200.problems import Just_Q
from qubo_b200.solvers import QBF

pytestmark = pytest.mark.gpu


def _problem(n, dtype, seed):
    rng = np.random.default_rng(seed)
    return (rng.integers(-50, 51, (n, n)) if np.issubdtype(dtype, np.integer)
            else rng.standard_normal((n, n))).astype(dtype)


def _check(Q, r):
    ref = oracle.qbf_port(Q)
    assert r["best_X_int"] == ref["best_X_int"]
    assert abs(r["best_E"] - ref["best_E"]) <= 1e-9 * max(1.0, abs(ref["best_E"]))


@pytest.mark.parametrize("n,dtype", [(12, np.int32), (26, np.int16), (30, np.float32)])
def test_autotune_choice_is_used(cuda_ok, n, dtype):
    h = _lib.Handle(0)
    try:
        Q = _problem(n, dtype, n)
        before = h.solve(Q, form="auto")
        assert not before["plan"]["tuned"]
        form = h.autotune(n, dtype)
        assert form in (("exact",) if n < 20 else ("gray", "tc"))
        r = h.solve(Q, form="auto")
        assert r["form"] == form
        _check(Q, r)
        if n >= 20:
            assert r["plan"]["tuned"]
            # the other dtype class keeps the defaults
            other = np.float64 if np.issubdtype(dtype, np.integer) else np.int32
            assert not h.solve(_problem(n, other, 1), form="auto")["plan"]["tuned"]
            # the batch uses the tuned plan of the class too
            Qs = [_problem(n, dtype, s) for s in range(3)] + [_problem(21, dtype, 9)]
            res = h.solve_batch(Qs)
            for Qb, rb in zip(Qs, res):
                _check(Qb, rb)
            drop = lambda p: {k: v for k, v in p.items() if k != "tc_kernel"}  # noqa: E731 (the batch's own kernel choice)
            assert res[0]["form"] == form and drop(res[0]["plan"]) == drop(r["plan"])
    finally:
        h.close()


def test_tuned_plan_reported_in_solution(cuda_ok):
    n = 27
    h = _lib.handle(0)
    h.autotune(n, np.int32)
    Q = _problem(n, np.int32, 3)
    sol = QBF().solve(Just_Q(Q), device="cuda")
    plan = sol.search["plan"]
    assert plan["tuned"] and plan["rec_log2"] >= 5
    if sol.search["form"] == "gray":
        assert plan["suffix_bits"] >= 13 and plan["unit_log2"] >= 7
    else:
        assert plan["suffix_bits"] == 15
    _check(Q, {"best_X_int": int("".join(map(str, sol.best_X)), 2), "best_E": float(sol.best_E)})
