"""QB_F1 with the reference's int16 arithmetic (int16_wrap=True): the state and reported
best_E equal the oracle's restatement of the reference QB_F1 (oracle.qbf1_int16_numpy),
including inputs whose int16 sums overflow; without overflow it equals the exact QB_F1
answer; at n = 44 it reproduces the reference notebook's printed QB_F1 result."""
import numpy as np
import pytest

import oracle
import qubo_b200  # noqa: F401
from conftest import bits_to_int, dec_q, load_golden
from qubo_b200.problems import Just_Q, ReducedProblem
from qubo_b200.solvers import QB_F1, Parallel

pytestmark = pytest.mark.gpu


def _xint(sol):
    return bits_to_int("".join(map(str, sol.best_X)))


# n < 29: chunks shorter than 32 steps (the per-step loop); n >= 29: aligned groups of 32 steps
@pytest.mark.parametrize("n,hi,seed", [(19, 100, 1), (20, 100, 2), (21, 3000, 3), (22, 30000, 4), (23, 900, 5),
                                       (29, 3000, 8), (30, 200, 9)])
def test_int16_wrap_matches_restated_reference(cuda_ok, n, hi, seed):
    Q = np.random.default_rng(seed).integers(-hi, hi, (n, n)).astype(np.int16)
    ref = oracle.qbf1_int16_numpy(Q)
    sol = QB_F1().solve(Just_Q(Q), device="cuda", int16_wrap=True)
    assert _xint(sol) == ref["best_X_int"]
    assert sol.best_E == ref["best_E"]
    assert sol.search["exact_E"] == ref["exact_E"]
    if hi <= 100:  # no int16 overflow: the exact answer
        ex = QB_F1().solve(Just_Q(Q), device="cuda")
        assert (_xint(ex), ex.best_E) == (_xint(sol), sol.best_E)


def test_parallel_int16_wrap(cuda_ok):
    n, k = 21, 1
    Q = np.random.default_rng(7).integers(-2000, 2000, (n, n)).astype(np.int16)
    best = None
    for task in range(1 << k):
        rp = ReducedProblem(Just_Q(Q), np.array([(task >> (k - 1 - i)) & 1 for i in range(k)]))
        r = oracle.qbf1_int16_numpy(rp.build_Q_matrix())
        adj = r["best_E"] + rp.prefix_E
        if best is None or adj < best[0]:
            best = (adj, (task << (n - k)) | r["best_X_int"])
    sol = Parallel(base_solver=QB_F1, splits_cnt=1 << k, devices=["cuda"]).solve(Just_Q(Q), int16_wrap=True)
    assert (sol.best_E, _xint(sol)) == best


def test_notebook_qb_f1_n44_in_int16(cuda_ok):
    nb = load_golden("notebook.json")
    Q = dec_q(nb["rerun_here"]["rq44_i16_seed42_Q"])
    rec = [r for r in nb["notebook"] if r["N"] == 44][0]
    sol = QB_F1().solve(Just_Q(Q), device="cuda", int16_wrap=True)
    assert sol.best_E == -6902
    e = oracle.energy(Q, _xint(sol))
    assert e == -6902
    # the notebook ran Parallel(QB_F1, 2 splits): same minimum; its state is the first task's
    par = Parallel(base_solver=QB_F1, splits_cnt=2, devices=["cuda"]).solve(Just_Q(Q), int16_wrap=True)
    assert _xint(par) == bits_to_int(rec["best_X"]) and par.best_E == -6902
