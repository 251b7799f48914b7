"""Stand-in device workers for the CPU tests of Parallel's multi-process task scheduling
(spawned by tests/test_parallel_workers_cpu.py; no GPU is touched).  Each has the signature
of qubo_b200.solvers._task_worker: it takes task ids from the shared queue until None."""
import os
import time


def _result(task, device):
    return {"task": task, "device": device, "time_ms": 1.0, "pid": os.getpid()}


def ok_worker(worker_id, device, Q, opts, tasks, results):
    while True:
        task = tasks.get()
        if task is None:
            return
        time.sleep(0.01)
        results.put(("res", task, worker_id, _result(task, device)))


def err_worker(worker_id, device, Q, opts, tasks, results):
    while True:
        task = tasks.get()
        if task is None:
            return
        if task == 3:
            results.put(("err", task, worker_id, "ValueError: injected"))
            return
        results.put(("res", task, worker_id, _result(task, device)))


def hang_worker(worker_id, device, Q, opts, tasks, results):
    time.sleep(120)


def crash_worker(worker_id, device, Q, opts, tasks, results):
    """Worker 0 takes a task and dies holding it (that task never completes); the others
    start only once it has taken its task (a flag file named in opts)."""
    if worker_id == 0:
        tasks.get()
        open(opts["flag"], "w").close()
        os._exit(3)
    t0 = time.time()
    while not os.path.exists(opts["flag"]) and time.time() - t0 < 60:
        time.sleep(0.01)
    ok_worker(worker_id, device, Q, opts, tasks, results)
