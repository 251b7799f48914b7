"""Parallel with several real CUDA workers (spawned processes, repeated device entries kept
as separate workers, as the reference's scheduler does: src/qubo_lib/solvers/scheduler.py:
5-45, parallel.py:99-103).  Each worker takes task ids from a shared queue and solves the
task's reduced problem on its device; the merge takes the lowest task among equal energies.
Answers are checked against the oracle and against the one-worker (fused) search, and the
per-task worker_logs against the reference's schema (task_id, worker_id, device,
time_to_solve_ms: parallel.py:314-318).  Only one GPU is used: both workers share cuda:0."""
import numpy as np
import pytest

import oracle
import qubo_b200  # noqa: F401
from conftest import bits_to_int
from qubo_b200.problems import Just_Q
from qubo_b200.solvers import QB_F1, QBF, Parallel, reduce_exact

pytestmark = pytest.mark.gpu


def _xint(sol):
    return bits_to_int("".join(map(str, sol.best_X)))


def _tied(n, seed, dtype=np.int32):
    """Pairs (i, i+1) with E = -c when exactly one is set: many optima across tasks."""
    rng = np.random.default_rng(seed)
    Q = np.zeros((n, n), np.int64)
    for i in range(0, n - 1, 2):
        c = int(rng.integers(1, 3))
        Q[i, i] -= c
        Q[i + 1, i + 1] -= c
        Q[i, i + 1] += 2 * c
    for _ in range(n):
        i, j = sorted(rng.integers(0, n, 2))
        Q[i, j] += int(rng.integers(-1, 2))
    return Q.astype(dtype)


def _check_logs(sol, n_tasks, n_workers, device="cuda:0"):
    logs = sol.worker_logs
    assert [w["task_id"] for w in logs] == list(range(n_tasks))
    assert all(set(w) == {"task_id", "worker_id", "device", "time_to_solve_ms"} for w in logs)
    assert all(0 <= w["worker_id"] < n_workers and w["device"] == device for w in logs)
    assert all(w["time_to_solve_ms"] > 0 for w in logs)
    per = {}
    for w in logs:
        per[w["worker_id"]] = per.get(w["worker_id"], 0.0) + w["time_to_solve_ms"]
    assert sol.time_to_solve_ms == pytest.approx(max(per.values()))


@pytest.mark.parametrize("n,splits,seed", [(26, 8, 1), (28, 4, 2)])
def test_qbf_two_workers_on_one_device(cuda_ok, n, splits, seed):
    Q = _tied(n, seed)
    ref = oracle.parallel_port(Q, splits)
    sol = Parallel(base_solver=QBF, splits_cnt=splits, devices=["cuda:0", "cuda:0"]).solve(Just_Q(Q))
    assert (_xint(sol), float(sol.best_E)) == (ref["best_X_int"], float(ref["best_E"]))
    assert sol.search["workers"] == 2 and sol.search["states"] == 2 ** n
    assert sol.epochs_cnt == splits and sol.solver_class == "QBF"
    _check_logs(sol, splits, 2)
    one = Parallel(base_solver=QBF, splits_cnt=splits, devices=["cuda:0"]).solve(Just_Q(Q))
    assert (_xint(one), float(one.best_E)) == (_xint(sol), float(sol.best_E))
    _check_logs(one, splits, 1)


def test_qbf_float_three_workers(cuda_ok):
    rng = np.random.default_rng(12)
    G = rng.standard_normal((25, 25))
    Q = (G + G.T) / 2
    ref = oracle.parallel_port(Q, 4)
    sol = Parallel(base_solver=QBF, splits_cnt=4, devices=["cuda:0"] * 3).solve(Just_Q(Q))
    assert _xint(sol) == ref["best_X_int"]
    assert abs(float(sol.best_E) - ref["best_E"]) <= 1e-9 * max(1.0, abs(ref["best_E"]))
    _check_logs(sol, 4, 3)


def test_qb_f1_two_workers(cuda_ok):
    n, k = 22, 2
    Q = _tied(n, 5, np.int16)
    # the oracle: each task's reduced problem under QB_F1's order, lowest task among ties
    best = None
    for task in range(1 << k):
        Qr, pe = reduce_exact(Q, k, task)
        r = oracle.qbf1_numpy(Qr)
        if best is None or r["best_E"] + pe < best[0]:
            best = (r["best_E"] + pe, (task << (n - k)) | r["best_X_int"])
    sol = Parallel(base_solver=QB_F1, splits_cnt=1 << k, devices=["cuda:0", "cuda:0"]).solve(Just_Q(Q))
    assert (_xint(sol), sol.best_E) == (best[1], best[0])
    assert isinstance(sol.best_E, int) and sol.solver_class == "QB_F1"
    _check_logs(sol, 1 << k, 2)
    one = Parallel(base_solver=QB_F1, splits_cnt=1 << k, devices=["cuda:0"]).solve(Just_Q(Q))
    assert (_xint(one), one.best_E) == (_xint(sol), sol.best_E)


def test_qb_f1_int16_wrap_two_workers(cuda_ok):
    n, k = 21, 1
    Q = np.random.default_rng(7).integers(-2000, 2000, (n, n)).astype(np.int16)
    one = Parallel(base_solver=QB_F1, splits_cnt=2, devices=["cuda:0"]).solve(Just_Q(Q), int16_wrap=True)
    two = Parallel(base_solver=QB_F1, splits_cnt=2, devices=["cuda:0", "cuda:0"]).solve(Just_Q(Q), int16_wrap=True)
    assert (_xint(two), two.best_E) == (_xint(one), one.best_E)
    _check_logs(two, 2, 2)


def test_metrics_match_one_worker(cuda_ok):
    Q = _tied(24, 9)
    kw = dict(use_metrics="all", A=4)
    two = Parallel(base_solver=QBF, splits_cnt=4, devices=["cuda:0", "cuda:0"]).solve(Just_Q(Q), **kw)
    one = Parallel(base_solver=QBF, splits_cnt=4, devices=["cuda:0"]).solve(Just_Q(Q), **kw)
    e2, e1 = two.metrics[0]["energy_arr"], one.metrics[0]["energy_arr"]
    assert np.array_equal(e2, e1) and e1.shape == (4 * 16,)
    for sol in (one, two):
        t = sol.metrics[0]["time_arr"]
        assert t.shape == (4 * 16,) and (t > 0).all()
