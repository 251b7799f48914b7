"""Exhaustive solvers: QBF, QB_F1 and Parallel over them (the reference's
``qubo_lib.solvers`` brute-force path), running on B200 through libqubo_b200.so.

Signatures, kwargs, errors and the returned Solution follow the reference:

* QBF    -- src/qubo_lib/solvers/qbf.py:20-548.  ``QBF().solve(problem, device=..., A=...,
            B=..., use_mem_GB=..., correction_period=..., use_metrics=...)``.  The answer is
            the state the reference's prefix loop would return: among minimal states, the
            smallest inverse-Gray rank of the A-bit prefix, then the smallest suffix
            (qbf.py:188-230, 395-412).  A comes from QBF.define_chunk_size exactly as in the
            reference; with neither A, B nor use_mem_GB given it is the reference's CPU
            default B = min(N, 20) (the reference's GPU default depends on free memory, pass
            use_mem_GB to reproduce a particular box).
* QB_F1  -- src/qubo_lib/solvers/qbf1.py:21-319: int16 Q only (TypeError otherwise), B = 18,
            answer chosen with QB_F1's kernel order (lowest of its 16,384 threads, then the
            earliest Gray prefix, then the smallest suffix).  Energies are exact: where the
            reference's int16 arithmetic could wrap, ``solution.search['int16_wrap_possible']``
            is set.  ``int16_wrap=True`` instead reproduces the reference's int16 arithmetic
            (state and reported best_E as the reference gives them, even where its sums
            overflow), for 19 <= N <= 46.
* Parallel -- src/qubo_lib/solvers/parallel.py:20-158: bit fixing over splits_cnt = 2^k
            tasks.  On one device the split is a tie-rule detail of a single GPU search
            (tasks are prefix tiles inside the kernel); with several devices one worker
            process per device searches a contiguous share, the workers exchange their
            minimum (as the reference's scheduler exchanges Solutions) and the best is
            merged.  Ties between tasks go to the lowest task id (the reference takes them
            in arrival order).

Every solve runs on a CUDA device: there is no CPU path (device='cpu' raises ValueError).
"""
from __future__ import annotations

import logging
import multiprocessing as mp
import os
import queue as _queue
import threading
import time

import numpy as np

from . import _json, _lib
from .abc import ProblemABC, SolverABC
from .solution import Solution
from .state_vectors import StateVectors
from .utils import PerformanceTimer

logger = logging.getLogger(__name__)

ALL_METRICS = {"time_arr", "energy_arr"}


def _torch_stream(device: int):
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("qubo_b200 needs a CUDA device; torch.cuda.is_available() is False")
    torch.cuda.set_device(device)
    return torch.cuda.current_stream(device).cuda_stream


_json_pool = None
_json_pool_lock = threading.Lock()


def _drop_json_pool():  # a forked child has the pool object but not its thread
    global _json_pool, _json_pool_lock
    _json_pool = None
    _json_pool_lock = threading.Lock()


os.register_at_fork(after_in_child=_drop_json_pool)


def _encode_async(problem, kwargs, Q=None):
    """A future of the Solution fields that depend on the problem alone: (problem.to_json(),
    the kwargs' JSON, the Ising offset of Q or None without Q).  They are computed on a worker
    thread while the library call, which releases the GIL, waits for the device (about 0.1 ms
    of host work per solve for a 36-variable problem)."""
    global _json_pool
    with _json_pool_lock:
        if _json_pool is None:
            from concurrent.futures import ThreadPoolExecutor
            _json_pool = ThreadPoolExecutor(max_workers=1, thread_name_prefix="qubo_b200-json")
    return _json_pool.submit(lambda: (problem.to_json(), _json.encode(kwargs, indent=4),
                                      None if Q is None else problem.get_Q_Ising_offset(np, Q)))


def _check_obsolete(kwargs):
    if "use_gpu" in kwargs:
        raise ValueError("use_gpu param is obsolete!")
    if "gpu_id" in kwargs:
        raise ValueError("gpu_id param is obsolete!")
    if "devices" in kwargs:
        raise ValueError("Use device argument")


def _int16_wrap_possible(Q: np.ndarray) -> bool:
    """True when some partial sum of Q's entries leaves int16 (the reference's QB_F1 and
    int16 QBF accumulate in int16)."""
    Q = Q.astype(np.int64)
    return bool(Q[Q > 0].sum() > 32767 or Q[Q < 0].sum() < -32768)


class QBF(SolverABC):
    """Exhaustive QUBO search (Gray-ordered prefix loop semantics) on a B200."""

    def __init__(self):
        super().__init__()
        self.glob_E = 0
        self.A = None
        self.B = None

    # -- split selection, identical to the reference (qbf.py:429-466) --------------------
    @staticmethod
    def define_chunk_size(N, **kwargs):
        if "A" in kwargs:
            return kwargs["A"], N - kwargs["A"]
        if "B" in kwargs:
            return N - kwargs["B"], kwargs["B"]
        if "use_mem_GB" in kwargs:
            return QBF.adjust_AB_to_fit_memory(N, kwargs["use_mem_GB"], kwargs.get("size_of", 4))
        B = min(N, 20)
        return N - B, B

    @staticmethod
    def estimate_memory_consumption_bytes(A, B, sizeof):
        return (B * 2 ** B + A * 2 ** B) * sizeof

    @staticmethod
    def adjust_AB_to_fit_memory(N, use_mem_GB, sizeof=4):
        limit = use_mem_GB * 2 ** 30
        best_b = N - 2
        for B in range(N - 2, 0, -1):
            best_b = B
            if QBF.estimate_memory_consumption_bytes(N - B, B, sizeof) <= limit:
                break
        return N - best_b, best_b

    @staticmethod
    def int_to_numpy_binary_array(num, bits_count, dtype=np.int32):
        if bits_count == 0:
            return np.array([], dtype=dtype)
        return np.array([int(b) for b in f"{int(num):b}".zfill(bits_count)], dtype=dtype)

    def check_obsolete_args(self, **kwargs):
        _check_obsolete(kwargs)

    def solve(self, problem: ProblemABC, **kwargs) -> Solution:
        self.check_obsolete_args(**kwargs)
        self.kwargs = kwargs
        dev = self.parse_device_arg(**kwargs)
        stream = _torch_stream(dev)
        self.timer = PerformanceTimer(use_gpu=True)
        self.N = problem.N
        Q = np.asarray(problem.build_Q_matrix(use_gpu=False))
        self.Q = Q
        self.timer.pick_time("build_Q")
        self.A, self.B = QBF.define_chunk_size(N=self.N, size_of=Q.dtype.itemsize, **kwargs)
        if self.A < 0 or self.B < 1 or self.A + self.B != self.N:
            raise ValueError(f"invalid split A={self.A}, B={self.B} for N={self.N}")
        form = kwargs.get("form", "auto")
        enc = _encode_async(problem, kwargs, Q)  # submitted last: it runs during the device search
        res = _lib.handle(dev).solve(Q, form=form, tie_rule="qbf", fixed_bits=0, prefix_bits=self.A,
                                     stream=stream)
        self.timer.pick_time("search")
        problem_json, self.json_str, offset = enc.result()
        return self._pack(problem, res, kwargs, problem_json, offset)

    def solve_batch(self, problems, **kwargs) -> list:
        """Solve many independent problems in one batched GPU search (qb_solve_batch) and
        return one Solution per problem, each the one ``solve(problem, **kwargs)`` returns.
        Problems with up to 36 variables share six kernel launches in total; larger ones are
        solved one by one.  ``graph=True`` runs that device work as one CUDA graph launch,
        captured once and replayed while later batches keep the same shape.  An addition:
        the reference solves one problem per call."""
        self.check_obsolete_args(**kwargs)
        if "B" in kwargs or "use_mem_GB" in kwargs:  # the split would differ per problem size
            return [QBF().solve(p, **kwargs) for p in problems]
        self.kwargs = kwargs
        self.json_str = _json.encode(kwargs, indent=4)
        dev = self.parse_device_arg(**kwargs)
        stream = _torch_stream(dev)
        self.timer = PerformanceTimer(use_gpu=True)
        Qs = [np.asarray(p.build_Q_matrix(use_gpu=False)) for p in problems]
        self.timer.pick_time("build_Q")
        results = _lib.handle(dev).solve_batch(Qs, form=kwargs.get("form", "auto"), tie_rule="qbf", fixed_bits=0,
                                               prefix_bits=int(kwargs.get("A", -1)), stream=stream,
                                               graph=bool(kwargs.get("graph", False)))
        self.timer.pick_time("search")
        out = []
        for problem, Q, res in zip(problems, Qs, results):
            self.N = problem.N
            self.Q = Q
            self.A, self.B = QBF.define_chunk_size(N=self.N, **kwargs)
            out.append(self._pack(problem, res, kwargs))
        return out

    def _pack(self, problem, res, kwargs, problem_json=None, ising_offset=None) -> Solution:
        best_X = res["best_X"]
        if problem_json is None:
            problem_json = problem.to_json()
        sol = Solution(self.N, 2 ** self.A, 1, problem_json, self.json_str)
        sol.state_vectors = StateVectors(wide_vector_matrix=best_X.reshape(1, -1))
        self.glob_E = np.float64(res["best_E"])
        sol.energies = np.array([self.glob_E])
        use_metrics = kwargs.get("use_metrics", set())
        if use_metrics == "all":
            use_metrics = ALL_METRICS
        metric_dict = {}
        if "energy_arr" in use_metrics:
            from .metrics import per_prefix_minima
            metric_dict["energy_arr"] = per_prefix_minima(self.Q, self.A, self.device_index)
        if "time_arr" in use_metrics:
            from .metrics import even_time_arr
            metric_dict["time_arr"] = even_time_arr(res["pass1_ms"] + res["pass2_ms"], self.A)
        sol.metrics = [metric_dict]
        sol.solver_class = "QBF"
        sol.best_E = self.glob_E
        sol.best_X = best_X
        sol.ising_offset = problem.get_Q_Ising_offset(np, self.Q) if ising_offset is None else ising_offset
        if hasattr(problem, "prefix_E"):
            sol.prefix_E = problem.prefix_E
        sol.time_to_solve_ms = self.timer.get_time_from_start()
        sol.timer = [(t, lbl) for t, lbl in self.timer.times if lbl != "epoch"]
        sol.search = {k: res[k] for k in ("form", "states", "candidate_records", "pass1_min", "err_bound",
                                          "pass1_ms", "pass2_ms", "kernel_ms", "order_key", "kernels",
                                          "h2d_bytes", "d2h_bytes", "plan")}
        sol.search["split"] = (self.A, self.B)
        return sol


class QB_F1(SolverABC):
    """int16 exhaustive search with QB_F1's answer order."""

    def __init__(self, **kwargs):
        super().__init__()
        self.A = None
        self.B = None

    def check_obsolete_args(self, **kwargs):
        _check_obsolete(kwargs)

    def parse_device_arg(self, **kwargs):
        device = kwargs.get("device", "cuda")
        if not isinstance(device, str) or device[:4] != "cuda":
            raise ValueError(f"QB_F1 solver is GPU only: {device}")
        return super().parse_device_arg(device=device)

    def solve(self, problem: ProblemABC, **kwargs) -> Solution:
        self.check_obsolete_args(**kwargs)
        dev = self.parse_device_arg(**kwargs)
        stream = _torch_stream(dev)
        self.timer = PerformanceTimer(use_gpu=True)
        self.N = problem.N
        self.B = 18
        self.A = self.N - self.B
        Q = np.asarray(problem.build_Q_matrix(use_gpu=False))
        if Q.dtype != np.int16:
            raise TypeError("Q dtype only np.int16 supported yet")
        if self.A < 1:
            raise ValueError(f"QB_F1 needs N >= 19 (B is fixed to 18), got N={self.N}")
        self.Q = Q
        self.timer.pick_time("build_Q")
        wrap = bool(kwargs.get("int16_wrap", False))
        enc = _encode_async(problem, kwargs, Q)  # submitted last: it runs during the device search
        res = _lib.handle(dev).solve(Q, form=kwargs.get("form", "auto"), tie_rule="qb_f1", fixed_bits=0,
                                     stream=stream, int16_wrap=wrap)
        self.timer.pick_time("Kernel run time")
        problem_json, self.json_str, offset = enc.result()
        best_X = res["best_X"]
        sol = Solution(self.N, 1, 1, problem_json, self.json_str)
        sol.state_vectors = StateVectors(wide_vector_matrix=best_X.reshape(1, -1))
        sol.energies = np.array([int(res["best_E_int"])])
        sol.metrics = [{}]
        sol.solver_class = "QB_F1"
        sol.best_E = int(res["best_E_int"])
        sol.best_X = best_X
        if hasattr(problem, "prefix_E"):
            sol.prefix_E = problem.prefix_E
        sol.ising_offset = offset
        sol.timer = [(t, lbl) for t, lbl in self.timer.times if lbl != "epoch"]
        sol.time_to_solve_ms = self.timer.get_time_from_start()
        sol.search = {k: res[k] for k in ("form", "states", "candidate_records", "pass1_ms", "pass2_ms", "kernel_ms",
                                          "kernels", "h2d_bytes", "d2h_bytes")}
        sol.search["int16_wrap_possible"] = _int16_wrap_possible(Q)
        sol.search["int16_wrap"] = wrap
        if wrap:  # the reference's answer: its int16 running value and the state it picks
            sol.search["exact_E"] = float(res["best_E"])
        elif sol.search["int16_wrap_possible"]:
            logger.warning("QB_F1: partial sums of Q exceed int16; the reference's int16 arithmetic could wrap, "
                           "this result is the exact minimum")
        return sol


BRUTEFORCE_SOLVERS = dict(QBF=QBF, QB_F1=QB_F1)
SUPPORTED_SOLVERS = dict(**BRUTEFORCE_SOLVERS)


def _parse_cuda(dev: str) -> int:
    if dev == "cuda":
        return 0
    if dev[:5] == "cuda:":
        return int(dev[5:])
    raise ValueError(f"Unknown device name: {dev}")


def reduce_exact(Q: np.ndarray, k: int, task: int):
    """Task ``task`` of Parallel's bit fixing: the first k variables fixed to the MSB-first
    bits of ``task``.  Returns (reduced Q, prefix_E) by ReducedProblem's rule
    (src/qubo_lib/problems/reduced_problem.py:31-46), Q' = Q[k:, k:] +
    diag(p (Q[:k, k:] + Q[k:, :k]^T)) and prefix_E = p^T Q[:k, :k] p, computed exactly (int64
    for integer Q, float64 otherwise) where the reference keeps the problem's dtype, so that a
    task's answer equals the same states' answer in the single-device search."""
    wide = np.int64 if np.issubdtype(Q.dtype, np.integer) else np.float64
    Qw = np.asarray(Q).astype(wide)
    p = np.array([(task >> (k - 1 - i)) & 1 for i in range(k)], dtype=wide)
    prefix_E = (p @ Qw[:k, :k] @ p).item()
    Qr = Qw[k:, k:] + np.diag(p @ (Qw[:k, k:] + Qw[k:, :k].T))
    return np.ascontiguousarray(Qr), prefix_E


def _task_worker(worker_id: int, device: int, Q: np.ndarray, opts: dict, tasks, results):
    """One worker of a multi-worker Parallel search (spawned process, the reference's
    scheduler.worker, src/qubo_lib/solvers/scheduler.py:48-59): takes task ids from the
    shared queue until it reads None, solves each task's reduced problem on its device and
    reports ("res", task, worker_id, result) or ("err", task, worker_id, message)."""
    try:
        stream = _torch_stream(device)
        h = _lib.handle(device)
    except Exception as e:  # noqa: BLE001 - reported to the parent
        results.put(("err", None, worker_id, f"{type(e).__name__}: {e}"))
        return
    k = int(opts["fixed_bits"])
    wrap = bool(opts.get("int16_wrap", False))
    solve_opts = {key: v for key, v in opts.items() if key not in ("fixed_bits", "int16_wrap")}
    while True:
        task = tasks.get()
        if task is None:
            break
        try:
            t0 = time.perf_counter()
            if wrap:  # the reference's own ReducedProblem: int16 arithmetic, wrapping as it does
                from .problems import Just_Q, ReducedProblem
                rp = ReducedProblem(Just_Q(Q), np.array([(task >> (k - 1 - i)) & 1 for i in range(k)]))
                Qr = rp.build_Q_matrix()
                pe = int(rp.prefix_E)
            else:
                Qr, pe = reduce_exact(Q, k, task)
            res = h.solve(Qr, stream=stream, fixed_bits=0, int16_wrap=wrap, **solve_opts)
            res["prefix_E"] = pe
            res["time_ms"] = (time.perf_counter() - t0) * 1000
            results.put(("res", task, worker_id, res))
        except Exception as e:  # noqa: BLE001 - reported to the parent like the reference's worker
            results.put(("err", task, worker_id, f"{type(e).__name__}: {e}"))


class Parallel(SolverABC):
    """Bit-fixing decomposition over splits_cnt = 2^k tasks (Embarrassingly Parallel
    Enumeration), on one or several CUDA devices."""

    def __init__(self, base_solver, splits_cnt: int, devices):
        self._base_solver = base_solver
        self._splits_cnt = splits_cnt
        self._devices = devices
        self._validate_config()

    def _validate_config(self):
        rev = {v: k for k, v in SUPPORTED_SOLVERS.items()}
        if self._base_solver not in rev:
            raise ValueError(f"Unsupported solver class: {self._base_solver}. "
                             f"Supported solvers: {', '.join(SUPPORTED_SOLVERS)}")
        self._solver_class_name = rev[self._base_solver]
        if not isinstance(self._splits_cnt, int) or self._splits_cnt <= 0:
            raise ValueError("splits_cnt must be a positive integer")
        if self._splits_cnt & (self._splits_cnt - 1) != 0:
            raise ValueError("For bruteforce solvers with Embarrassingly Parallel Enumeration / Bit-Fixing "
                             f"Decomposition, splits_cnt must be a power of 2, got {self._splits_cnt}")
        if not self._devices:
            raise ValueError("Devices list cannot be empty")
        has_cpu = any("cpu" in d for d in self._devices)
        has_gpu = any("cuda" in d for d in self._devices)
        if has_cpu and has_gpu:
            raise ValueError("Cannot mix CPU and GPU devices")
        if has_cpu:
            raise ValueError("qubo_b200 runs on CUDA devices only; use devices=['cuda', ...]")
        if all(d == "cuda" for d in self._devices):
            self._devices = [f"cuda:{i}" for i in range(len(self._devices))]
        else:
            self._devices = list(self._devices)
        for d in self._devices:
            _parse_cuda(d)

    def solve(self, problem: ProblemABC, timeout=None, **kwargs) -> Solution:
        _check_obsolete(kwargs)
        kw = dict(solver_type=self._solver_class_name, splits_cnt=self._splits_cnt, devices=self._devices,
                  timeout=timeout, **kwargs)
        json_str = _json.encode(kw, indent=4)
        k = self._splits_cnt.bit_length() - 1
        N = problem.N
        if k >= N:
            raise ValueError(f"splits_cnt={self._splits_cnt} fixes every one of the {N} variables")
        t0 = time.perf_counter()
        Q = np.asarray(problem.build_Q_matrix(use_gpu=False))
        m = N - k
        workers = [_parse_cuda(d) for d in self._devices]  # one worker per entry, repeats included
        if self._solver_class_name == "QBF":
            A_sub, _ = QBF.define_chunk_size(N=m, size_of=Q.dtype.itemsize, **kwargs)
            opts = dict(form=kwargs.get("form", "auto"), tie_rule="qbf", fixed_bits=k, prefix_bits=A_sub)
        else:
            if Q.dtype != np.int16:
                raise TypeError("Q dtype only np.int16 supported yet")
            if m < 19:
                raise ValueError(f"QB_F1 needs N - log2(splits_cnt) >= 19, got {m}")
            wrap = bool(kwargs.get("int16_wrap", False))
            if wrap and len(workers) == 1:
                return self._solve_qbf1_int16(problem, Q, k, json_str, t0, kwargs)
            opts = dict(form=kwargs.get("form", "auto"), tie_rule="qb_f1", fixed_bits=k)
            if wrap:
                opts["int16_wrap"] = True
        n_tasks = self._splits_cnt
        is_f1 = self._solver_class_name == "QB_F1"
        if len(workers) == 1:
            # one worker: every task is a prefix tile of one GPU search; the task bits lead
            # the search's order key, so ties between tasks go to the lowest task id
            stream = _torch_stream(workers[0])
            best = _lib.handle(workers[0]).solve(Q, stream=stream, **opts)
            total_ms = (time.perf_counter() - t0) * 1000
            best_E = int(best["best_E_int"]) if is_f1 else np.float64(best["best_E"])
            best_X = best["best_X"]
            # the tasks run interleaved inside one search of equal-sized shares: each task is
            # logged with an equal share of the search time
            logs = [dict(task_id=t, worker_id=0, device=self._devices[0], time_to_solve_ms=total_ms / n_tasks)
                    for t in range(n_tasks)]
            time_to_solve = total_ms
            parts = [best]
            task_ms = [total_ms / n_tasks] * n_tasks
        else:
            done = self._run_workers(workers, Q, opts, n_tasks, timeout)
            pick = None
            for task in range(n_tasks):  # task order, strict <: the lowest task id wins ties
                _, r = done[task]
                E = (int(r["best_E_int"]) + int(r["prefix_E"])) if (is_f1 or r["is_integer"]) else \
                    float(r["best_E"]) + float(r["prefix_E"])
                if pick is None or E < pick[0]:
                    pick = (E, task, r)
            E, task, best = pick
            prefix = np.array([(task >> (k - 1 - i)) & 1 for i in range(k)], dtype=best["best_X"].dtype)
            best_X = np.hstack([prefix, best["best_X"]])
            if is_f1:
                best_E = int(E)
            elif best["is_integer"]:
                best_E = np.float64(E)
            else:  # FP64 energy of the full state, as the single-device search reports it
                xf = best_X.astype(np.float64)
                best_E = np.float64(xf @ Q.astype(np.float64) @ xf)
            logs = [dict(task_id=t, worker_id=done[t][0], device=self._devices[done[t][0]],
                         time_to_solve_ms=done[t][1]["time_ms"]) for t in range(n_tasks)]
            per_worker = {}
            for t in range(n_tasks):
                per_worker[done[t][0]] = per_worker.get(done[t][0], 0.0) + done[t][1]["time_ms"]
            time_to_solve = max(per_worker.values())  # the busiest worker, as the reference reports
            parts = [done[t][1] for t in range(n_tasks)]
            task_ms = [done[t][1]["time_ms"] for t in range(n_tasks)]
        sol = Solution(N=N, epochs_cnt=self._splits_cnt, samples_cnt=1, problem_instance_json=problem.to_json(),
                       solver_params_json=json_str)
        sol.ising_offset = None
        sol.solver_class = self._solver_class_name
        sol.best_E = best_E
        sol.energies = np.array([best_E])
        sol.best_X = best_X
        sol.state_vectors = StateVectors(wide_vector_matrix=best_X.reshape(1, -1))
        metrics = {}
        use_metrics = kwargs.get("use_metrics", set())
        if use_metrics == "all":
            use_metrics = ALL_METRICS
        if not is_f1:
            if "energy_arr" in use_metrics:
                from .metrics import parallel_energy_arr
                metrics["energy_arr"] = parallel_energy_arr(Q, k, opts["prefix_bits"], workers[0])
            if "time_arr" in use_metrics:
                from .metrics import even_time_arr
                share = even_time_arr(1.0, k + opts["prefix_bits"])[: 1 << opts["prefix_bits"]] * (1 << k)
                metrics["time_arr"] = np.concatenate([ms * share for ms in task_ms])
        sol.metrics = [metrics]
        sol.time_to_solve_ms = time_to_solve
        sol.worker_logs = logs
        sol.search = {k2: best[k2] for k2 in ("form", "pass1_ms", "pass2_ms", "order_key")}
        sol.search["candidate_records"] = sum(r["candidate_records"] for r in parts)
        sol.search["states"] = sum(r["states"] for r in parts)
        sol.search["workers"] = len(workers)
        return sol

    def _solve_qbf1_int16(self, problem, Q, k, json_str, t0, kwargs) -> Solution:
        """Parallel(QB_F1) with the reference's int16 arithmetic, task by task as the reference
        runs it (parallel.py:145-157, 225-320): ReducedProblem in int16 (its prefix_E and
        reduced Q wrap as in reduced_problem.py:31-46), QB_F1 on each, the best of
        best_E + prefix_E with strict < in task order."""
        from .problems import Just_Q, ReducedProblem
        dev = _parse_cuda(self._devices[0])
        base = Just_Q(Q)
        best = None
        logs = []
        for task in range(self._splits_cnt):
            prefix = np.array([(task >> (k - 1 - i)) & 1 for i in range(k)])
            rp = ReducedProblem(base, prefix)
            part = QB_F1().solve(rp, device=f"cuda:{dev}", int16_wrap=True)
            adj = part.best_E + rp.prefix_E
            if best is None or adj < best[0]:
                best = (adj, task, part)
            logs.append(dict(task_id=task, worker_id=0, device=f"cuda:{dev}", time_to_solve_ms=part.time_to_solve_ms))
        adj, task, part = best
        N = problem.N
        sol = Solution(N=N, epochs_cnt=self._splits_cnt, samples_cnt=1, problem_instance_json=problem.to_json(),
                       solver_params_json=json_str)
        sol.ising_offset = None
        sol.solver_class = "QB_F1"
        sol.best_E = adj
        sol.energies = np.array([adj])
        prefix = np.array([(task >> (k - 1 - i)) & 1 for i in range(k)], dtype=part.best_X.dtype)
        sol.best_X = np.hstack([prefix, part.best_X])
        sol.state_vectors = StateVectors(wide_vector_matrix=sol.best_X.reshape(1, -1))
        sol.metrics = [{}]
        sol.time_to_solve_ms = (time.perf_counter() - t0) * 1000
        sol.worker_logs = logs
        sol.search = dict(part.search, task=task)
        return sol

    @staticmethod
    def _run_workers(workers, Q, opts, n_tasks, timeout, worker=None):
        """The reference's devices_scheduler (src/qubo_lib/solvers/scheduler.py:5-45): one
        spawned process per entry of ``workers`` (device ids, repeats allowed) takes task ids
        0 .. n_tasks-1 from a shared queue (``worker``, default _task_worker).  Returns
        {task: (worker_id, result)}.  A worker that reports an exception, or exits with a
        non-zero code, raises RuntimeError; tasks still missing at ``timeout`` seconds
        (default 24 h, as the reference's scheduler) raise TimeoutError.  Unlike the
        reference's scheduler, partial results are never merged."""
        ctx = mp.get_context("spawn")
        tasks = ctx.Queue()
        results = ctx.Queue()
        for t in range(n_tasks):
            tasks.put(t)
        for _ in workers:
            tasks.put(None)
        target = worker or _task_worker
        procs = [ctx.Process(target=target, args=(w, d, Q, opts, tasks, results)) for w, d in enumerate(workers)]
        for p in procs:
            p.start()
        deadline = time.time() + (timeout if timeout is not None else 24 * 3600)
        done = {}
        try:
            while len(done) < n_tasks:
                left = deadline - time.time()
                if left <= 0:
                    raise TimeoutError(f"Parallel: {n_tasks - len(done)} of {n_tasks} tasks unfinished at "
                                       f"timeout={timeout}")
                try:
                    kind, task, wid, val = results.get(timeout=min(0.5, left))
                except _queue.Empty:
                    for i, p in enumerate(procs):
                        if not p.is_alive() and p.exitcode not in (0, None) and results.empty():
                            raise RuntimeError(f"worker {i} exited (code {p.exitcode}) without a result") from None
                    if all(not p.is_alive() for p in procs) and results.empty():
                        raise RuntimeError(f"workers exited with {n_tasks - len(done)} tasks unfinished") from None
                    continue
                if kind == "err":
                    raise RuntimeError(f"worker {wid} (task {task}): {val}")
                done[task] = (wid, val)
        finally:
            for p in procs:
                p.join(timeout=5)
                if p.is_alive():
                    p.terminate()
                    p.join()
        return done
