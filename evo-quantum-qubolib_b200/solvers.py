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
import queue as _queue
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
        self.json_str = _json.encode(kwargs, indent=4)
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
        res = _lib.handle(dev).solve(Q, form=form, tie_rule="qbf", fixed_bits=0, prefix_bits=self.A,
                                     stream=stream)
        self.timer.pick_time("search")
        return self._pack(problem, res, kwargs)

    def solve_batch(self, problems, **kwargs) -> list:
        """Solve many independent problems in one batched GPU search (qb_solve_batch) and
        return one Solution per problem, each the one ``solve(problem, **kwargs)`` returns.
        Problems with up to 36 variables share six kernel launches in total; larger ones are
        solved one by one.  An addition: the reference solves one problem per call."""
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
                                               prefix_bits=int(kwargs.get("A", -1)), stream=stream)
        self.timer.pick_time("search")
        out = []
        for problem, Q, res in zip(problems, Qs, results):
            self.N = problem.N
            self.Q = Q
            self.A, self.B = QBF.define_chunk_size(N=self.N, **kwargs)
            out.append(self._pack(problem, res, kwargs))
        return out

    def _pack(self, problem, res, kwargs) -> Solution:
        best_X = res["best_X"]
        sol = Solution(self.N, 2 ** self.A, 1, problem.to_json(), self.json_str)
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
            metric_dict["time_arr"] = np.array([res["pass1_ms"] + res["pass2_ms"]])
        sol.metrics = [metric_dict]
        sol.solver_class = "QBF"
        sol.best_E = self.glob_E
        sol.best_X = best_X
        sol.ising_offset = problem.get_Q_Ising_offset(np, self.Q)
        if hasattr(problem, "prefix_E"):
            sol.prefix_E = problem.prefix_E
        sol.time_to_solve_ms = self.timer.get_time_from_start()
        sol.timer = [(t, lbl) for t, lbl in self.timer.times if lbl != "epoch"]
        sol.search = {k: res[k] for k in ("form", "states", "candidate_records", "pass1_min", "err_bound",
                                          "pass1_ms", "pass2_ms", "kernel_ms", "order_key", "kernels",
                                          "h2d_bytes", "d2h_bytes")}
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
        self.json_str = _json.encode(kwargs, indent=4)
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
        res = _lib.handle(dev).solve(Q, form=kwargs.get("form", "auto"), tie_rule="qb_f1", fixed_bits=0,
                                     stream=stream, int16_wrap=wrap)
        self.timer.pick_time("Kernel run time")
        best_X = res["best_X"]
        sol = Solution(self.N, 1, 1, problem.to_json(), self.json_str)
        sol.state_vectors = StateVectors(wide_vector_matrix=best_X.reshape(1, -1))
        sol.energies = np.array([int(res["best_E_int"])])
        sol.metrics = [{}]
        sol.solver_class = "QB_F1"
        sol.best_E = int(res["best_E_int"])
        sol.best_X = best_X
        if hasattr(problem, "prefix_E"):
            sol.prefix_E = problem.prefix_E
        sol.ising_offset = problem.get_Q_Ising_offset(np, Q)
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


def _worker_main(device: int, Q: np.ndarray, opts: dict, shard_index: int, shard_count: int, inbox, outbox):
    """One device's share of a multi-device Parallel search (spawned process)."""
    try:
        stream = _torch_stream(device)
        h = _lib.handle(device)
        t0 = time.perf_counter()
        lmin = h.solve_begin(Q, shard_index=shard_index, shard_count=shard_count, stream=stream, **opts)
        outbox.put(("min", shard_index, lmin))
        gmin = inbox.get()
        res = h.solve_finish(gmin, Q.shape[0])
        res["time_ms"] = (time.perf_counter() - t0) * 1000
        outbox.put(("res", shard_index, res))
    except Exception as e:  # noqa: BLE001 - reported to the parent like the reference's worker
        outbox.put(("err", shard_index, f"{type(e).__name__}: {e}"))


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
        if self._solver_class_name == "QBF":
            A_sub, _ = QBF.define_chunk_size(N=m, size_of=Q.dtype.itemsize, **kwargs)
            opts = dict(form=kwargs.get("form", "auto"), tie_rule="qbf", fixed_bits=k, prefix_bits=A_sub)
        else:
            if Q.dtype != np.int16:
                raise TypeError("Q dtype only np.int16 supported yet")
            if m < 19:
                raise ValueError(f"QB_F1 needs N - log2(splits_cnt) >= 19, got {m}")
            if kwargs.get("int16_wrap", False):
                return self._solve_qbf1_int16(problem, Q, k, json_str, t0, kwargs)
            opts = dict(form=kwargs.get("form", "auto"), tie_rule="qb_f1", fixed_bits=k)
        devs = sorted(set(_parse_cuda(d) for d in self._devices))
        if len(devs) == 1:
            stream = _torch_stream(devs[0])
            res = _lib.handle(devs[0]).solve(Q, stream=stream, **opts)
            results = [res]
            res["time_ms"] = (time.perf_counter() - t0) * 1000
        else:
            results = self._run_workers(devs, Q, opts, timeout)
        found = [r for r in results if r["found"]]
        if not found:
            raise RuntimeError("no worker reported a minimising state")
        best = min(found, key=lambda r: (r["best_E"], r["order_key"]))
        sol = Solution(N=N, epochs_cnt=self._splits_cnt, samples_cnt=1, problem_instance_json=problem.to_json(),
                       solver_params_json=json_str)
        sol.ising_offset = None
        sol.solver_class = self._solver_class_name
        best_E = int(best["best_E_int"]) if (self._solver_class_name == "QB_F1") else np.float64(best["best_E"])
        sol.best_E = best_E
        sol.energies = np.array([best_E])
        sol.best_X = best["best_X"]
        sol.state_vectors = StateVectors(wide_vector_matrix=best["best_X"].reshape(1, -1))
        metrics = {}
        use_metrics = kwargs.get("use_metrics", set())
        if use_metrics == "all":
            use_metrics = ALL_METRICS
        if "energy_arr" in use_metrics and self._solver_class_name == "QBF":
            from .metrics import parallel_energy_arr
            metrics["energy_arr"] = parallel_energy_arr(Q, k, opts["prefix_bits"], devs[0])
        sol.metrics = [metrics]
        sol.time_to_solve_ms = max(r["time_ms"] for r in results)
        sol.worker_logs = []
        n_tasks = self._splits_cnt
        for w, r in enumerate(results):
            first = w * n_tasks // len(results)
            last = (w + 1) * n_tasks // len(results) - 1
            sol.worker_logs.append(dict(worker_id=w, device=f"cuda:{devs[w]}", task_ids=(first, last),
                                        time_to_solve_ms=r["time_ms"], states=r["states"]))
        sol.search = {k2: best[k2] for k2 in ("form", "candidate_records", "pass1_ms", "pass2_ms", "order_key")}
        sol.search["states"] = sum(r["states"] for r in results)
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
    def _run_workers(devs, Q, opts, timeout, worker=None):
        """One spawned process per device (worker, default _worker_main) searches a contiguous
        share; the parent exchanges the pass-1 minima and collects the shares' results.  A
        worker that reports an exception or exits without reporting raises RuntimeError; no
        answer within ``timeout`` seconds (default 24 h, as the reference's scheduler) raises
        TimeoutError.  Unlike the reference's scheduler (scheduler.py:26-45), partial results
        are never merged."""
        ctx = mp.get_context("spawn")
        outbox = ctx.Queue()
        inboxes = [ctx.Queue() for _ in devs]
        target = worker or _worker_main
        procs = [ctx.Process(target=target, args=(d, Q, opts, i, len(devs), inboxes[i], outbox))
                 for i, d in enumerate(devs)]
        for p in procs:
            p.start()
        deadline = time.time() + (timeout if timeout is not None else 24 * 3600)

        def receive(done: dict):
            while True:
                left = deadline - time.time()
                if left <= 0:
                    raise _queue.Empty
                try:
                    kind, idx, val = outbox.get(timeout=min(0.5, left))
                    return kind, idx, val
                except _queue.Empty:
                    for i, p in enumerate(procs):
                        if i not in done and not p.is_alive() and outbox.empty():
                            raise RuntimeError(f"worker {i} exited (code {p.exitcode}) without a result")

        try:
            mins = {}
            while len(mins) < len(devs):
                kind, idx, val = receive(mins)
                if kind == "err":
                    raise RuntimeError(f"worker {idx}: {val}")
                mins[idx] = val
            gmin = min(mins.values())
            for q in inboxes:
                q.put(gmin)
            results = {}
            while len(results) < len(devs):
                kind, idx, val = receive(results)
                if kind == "err":
                    raise RuntimeError(f"worker {idx}: {val}")
                results[idx] = val
        except _queue.Empty:
            raise TimeoutError(f"Parallel: workers did not finish within timeout={timeout}") from None
        finally:
            for p in procs:
                p.join(timeout=5)
                if p.is_alive():
                    p.terminate()
                    p.join()
        return [results[i] for i in range(len(devs))]
