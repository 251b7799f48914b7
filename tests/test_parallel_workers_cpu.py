"""Parallel's multi-worker task scheduling on CPU with stand-in workers (tests/_fake_workers.py):
every task is solved exactly once, by some worker, repeated devices are separate workers,
and failures are reported instead of merged -- an exception in a worker, a worker that
exits without finishing, and a timeout."""
import time

import numpy as np
import pytest

import qubo_b200  # noqa: F401
from qubo_b200.solvers import Parallel, reduce_exact

import _fake_workers as fw

Q = np.zeros((4, 4), np.int16)


def test_every_task_once_and_repeated_devices():
    done = Parallel._run_workers([0, 0, 1], Q, {}, 16, timeout=60, worker=fw.ok_worker)
    assert sorted(done) == list(range(16))
    assert all(r["task"] == t for t, (_, r) in done.items())
    used = {w for w, _ in done.values()}
    assert used <= {0, 1, 2}
    assert {r["device"] for w, r in done.values() if w in (0, 1)} <= {0}  # the two workers on device 0
    assert len({r["pid"] for _, r in done.values()}) == len(used)  # one process per worker


def test_worker_exception_is_raised():
    with pytest.raises(RuntimeError, match="injected"):
        Parallel._run_workers([0, 1], Q, {}, 8, timeout=60, worker=fw.err_worker)


def test_dead_worker_is_detected(tmp_path):
    t0 = time.time()
    with pytest.raises(RuntimeError, match="exited"):
        Parallel._run_workers([0, 1], Q, {"flag": str(tmp_path / "taken")}, 8, timeout=60, worker=fw.crash_worker)
    assert time.time() - t0 < 30


def test_timeout():
    t0 = time.time()
    with pytest.raises(TimeoutError):
        Parallel._run_workers([0, 1], Q, {}, 4, timeout=2, worker=fw.hang_worker)
    assert time.time() - t0 < 30


@pytest.mark.parametrize("dtype", [np.int16, np.int32, np.float32, np.float64])
def test_reduce_exact_matches_the_energy(dtype):
    """The task's reduced problem plus its prefix energy gives the full problem's energy of
    every state of the task (the reference's ReducedProblem rule without dtype wrap)."""
    rng = np.random.default_rng(4)
    n, k = 9, 3
    Q = (rng.integers(-30000, 30000, (n, n)) if np.issubdtype(dtype, np.integer)
         else rng.standard_normal((n, n))).astype(dtype)
    Qw = Q.astype(np.float64)
    for task in (0, 5, 7):
        Qr, pe = reduce_exact(Q, k, task)
        assert Qr.dtype == (np.int64 if np.issubdtype(dtype, np.integer) else np.float64)
        for s in (0, 17, 63):
            x = np.array([(task >> (k - 1 - i)) & 1 for i in range(k)] +
                         [(s >> (n - k - 1 - i)) & 1 for i in range(n - k)], dtype=np.float64)
            xs = x[k:]
            full = x @ Qw @ x
            assert abs((xs @ Qr.astype(np.float64) @ xs + pe) - full) <= 1e-9 * max(1.0, abs(full))
