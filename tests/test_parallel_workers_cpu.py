"""Parallel's multi-device exchange on CPU with stand-in workers (tests/_fake_workers.py):
the global minimum reaches every worker, results come back in device order, and failures
are reported instead of merged -- an exception in a worker, a worker that exits without a
result, and a timeout."""
import time

import numpy as np
import pytest

import qubo_b200  # noqa: F401
from qubo_b200.solvers import Parallel

import _fake_workers as fw

Q = np.zeros((4, 4), np.int16)


def test_exchange_and_order():
    res = Parallel._run_workers([0, 1, 2], Q, {}, timeout=60, worker=fw.ok_worker)
    assert [r["device"] for r in res] == [0, 1, 2]
    assert all(r["gmin"] == 8.0 for r in res)  # min of 10, 9, 8
    assert [r["found"] for r in res] == [False, False, True]


def test_worker_exception_is_raised():
    with pytest.raises(RuntimeError, match="injected"):
        Parallel._run_workers([0, 1], Q, {}, timeout=60, worker=fw.err_worker)


def test_dead_worker_is_detected():
    t0 = time.time()
    with pytest.raises(RuntimeError, match="exited"):
        Parallel._run_workers([0, 1], Q, {}, timeout=60, worker=fw.crash_worker)
    assert time.time() - t0 < 30


def test_timeout():
    t0 = time.time()
    with pytest.raises(TimeoutError):
        Parallel._run_workers([0, 1], Q, {}, timeout=2, worker=fw.hang_worker)
    assert time.time() - t0 < 30
