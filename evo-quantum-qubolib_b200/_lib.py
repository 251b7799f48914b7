"""ctypes binding of libqubo_b200.so (the C ABI in include/qubo_b200.h).

The library must be built in-tree (``python __graft_entry__.py`` or ``build.py`` beside
this file).  Importing the binding without it raises ImportError: there is no CPU path.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libqubo_b200.so")

_char_from_buffer = ctypes.c_char.from_buffer
_addressof = ctypes.addressof

QB_OK, QB_EINVAL, QB_ERANGE, QB_ENOMEM, QB_ECUDA, QB_ETIMEOUT, QB_ENODEV, QB_EOVERFLOW, QB_ETOOBIG = range(9)
QB_F32, QB_F64, QB_I8, QB_I16, QB_I32, QB_I64 = 1, 2, 3, 4, 5, 6
FORMS = {"auto": 0, "gray": 1, "tc": 2, "exact": 3}
FORM_NAMES = {v: k for k, v in FORMS.items()}
FORM_NAMES[4] = "qb_f1_int16"
QB_FLAG_INT16_WRAP = 1
QB_FLAG_TEST_STALL = 2
QB_FLAG_GRAPH = 4
QB_FLAG_TC_PAIR = 8
QB_FLAG_TC_NO16 = 16
QB_FLAG_TC_ONE = 32
TC_KERNELS = {0: None, 1: "fp32", 2: "pair", 3: "u16", 4: "pair_u16"}
TIE_RULES = {"qbf": 0, "qb_f1": 1, "natural": 2}

_DTYPES = {
    np.dtype(np.float32): QB_F32,
    np.dtype(np.float64): QB_F64,
    np.dtype(np.int8): QB_I8,
    np.dtype(np.int16): QB_I16,
    np.dtype(np.int32): QB_I32,
    np.dtype(np.int64): QB_I64,
}


class QbProblem(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32), ("dtype", ctypes.c_int32), ("q", ctypes.c_void_p), ("ldq", ctypes.c_int64),
                ("q_on_device", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class QbOptions(ctypes.Structure):
    _fields_ = [("form", ctypes.c_int32), ("tie_rule", ctypes.c_int32), ("fixed_bits", ctypes.c_int32),
                ("prefix_bits", ctypes.c_int32), ("shard_index", ctypes.c_int32), ("shard_count", ctypes.c_int32),
                ("max_candidates", ctypes.c_int32), ("flags", ctypes.c_int32), ("stream", ctypes.c_void_p)]


class QbResult(ctypes.Structure):
    _fields_ = [("best_x", ctypes.c_uint64), ("best_e", ctypes.c_double), ("best_e_int", ctypes.c_int64),
                ("order_key", ctypes.c_uint64), ("pass1_min", ctypes.c_double), ("err_bound", ctypes.c_double),
                ("states", ctypes.c_int64), ("candidate_records", ctypes.c_int64), ("form_used", ctypes.c_int32),
                ("is_integer", ctypes.c_int32), ("found", ctypes.c_int32), ("status", ctypes.c_int32),
                ("pass1_ms", ctypes.c_float), ("pass2_ms", ctypes.c_float), ("kernels", ctypes.c_int32),
                ("kernel_ms", ctypes.c_float), ("h2d_bytes", ctypes.c_int64), ("d2h_bytes", ctypes.c_int64),
                ("rec_log2", ctypes.c_int32), ("suffix_bits", ctypes.c_int32), ("unit_log2", ctypes.c_int32),
                ("tuned", ctypes.c_int32), ("tc_kernel", ctypes.c_int32)]


class QbNoAllocResult(ctypes.Structure):
    _fields_ = [("best_e", ctypes.c_double), ("best_x", ctypes.c_uint64), ("order_key", ctypes.c_uint64),
                ("status", ctypes.c_int32), ("candidates", ctypes.c_int32)]


class QbError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        super().__init__(f"{where}: {strerror(status)} (status {status})")


_lib = None
_lock = threading.Lock()


def load():
    """Load libqubo_b200.so (raises ImportError when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build the CUDA library first (python __graft_entry__.py)")
    L = ctypes.CDLL(LIB_PATH)
    H = ctypes.c_void_p
    L.qb_version.restype = ctypes.c_int
    L.qb_strerror.argtypes = [ctypes.c_int]
    L.qb_strerror.restype = ctypes.c_char_p
    L.qb_handle_create.argtypes = [ctypes.c_int, ctypes.POINTER(H)]
    L.qb_handle_destroy.argtypes = [H]
    for name in ("qb_solve",):
        getattr(L, name).argtypes = [H, ctypes.POINTER(QbProblem), ctypes.POINTER(QbOptions), ctypes.POINTER(QbResult)]
    L.qb_solve_begin.argtypes = [H, ctypes.POINTER(QbProblem), ctypes.POINTER(QbOptions),
                                 ctypes.POINTER(ctypes.c_double)]
    L.qb_solve_finish.argtypes = [H, ctypes.c_double, ctypes.POINTER(QbResult)]
    L.qb_solve_batch.argtypes = [H, ctypes.POINTER(QbProblem), ctypes.c_int32, ctypes.POINTER(QbOptions),
                                 ctypes.POINTER(QbResult)]
    L.qb_autotune.argtypes = [H, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]
    L.qb_prefix_minima.argtypes = [H, ctypes.POINTER(QbProblem), ctypes.c_int32, ctypes.c_void_p]
    L.qb_solve_noalloc.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                   ctypes.c_void_p, ctypes.c_void_p]
    _lib = L
    return L


def strerror(status: int) -> str:
    try:
        return load().qb_strerror(int(status)).decode()
    except ImportError:
        return f"status {status}"


def _raise(status: int, where: str):
    if status == QB_EINVAL:
        raise ValueError(f"{where}: {strerror(status)}")
    if status == QB_ERANGE:
        raise OverflowError(f"{where}: {strerror(status)}")
    raise QbError(status, where)


class Handle:
    """One library handle (device stream + scratch).  Not shared between threads."""

    def __init__(self, device: int):
        L = load()
        self.device = device
        self._h = ctypes.c_void_p()
        rc = L.qb_handle_create(int(device), ctypes.byref(self._h))
        if rc:
            _raise(rc, f"qb_handle_create(device={device})")

    def close(self):
        if self._h:
            load().qb_handle_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    @staticmethod
    def _problem(Q: np.ndarray) -> tuple[QbProblem, np.ndarray]:
        Q = np.ascontiguousarray(Q)
        if Q.ndim != 2 or Q.shape[0] != Q.shape[1]:
            raise ValueError(f"Q must be square, got shape {Q.shape}")
        code = _DTYPES.get(Q.dtype)
        if code is None:
            raise TypeError(f"unsupported Q dtype {Q.dtype}")
        n = Q.shape[0]
        p = QbProblem(n, code, Q.__array_interface__["data"][0], n, 0, 0)
        return p, Q

    @staticmethod
    def options(form="auto", tie_rule="qbf", fixed_bits=0, prefix_bits=-1, shard_index=0, shard_count=1,
                max_candidates=0, stream=None, int16_wrap=False, flags=0, graph=False,
                tc_pair=False, tc_no16=False, tc_one=False) -> QbOptions:
        return QbOptions(form=FORMS[form], tie_rule=TIE_RULES[tie_rule], fixed_bits=int(fixed_bits),
                         prefix_bits=int(prefix_bits), shard_index=int(shard_index), shard_count=int(shard_count),
                         max_candidates=int(max_candidates),
                         flags=int(flags) | (QB_FLAG_INT16_WRAP if int16_wrap else 0) | (QB_FLAG_GRAPH if graph else 0) |
                         (QB_FLAG_TC_PAIR if tc_pair else 0) | (QB_FLAG_TC_NO16 if tc_no16 else 0) |
                         (QB_FLAG_TC_ONE if tc_one else 0),
                         stream=stream)

    def solve(self, Q: np.ndarray, **opts) -> dict:
        p, keep = self._problem(Q)
        o = self.options(**opts)
        r = QbResult()
        rc = load().qb_solve(self._h, ctypes.byref(p), ctypes.byref(o), ctypes.byref(r))
        del keep
        if rc:
            _raise(rc, "qb_solve")
        return result_dict(r, p.n)

    def solve_device(self, ptr: int, n: int, dtype, **opts) -> dict:
        """Solve a Q already resident in device memory (row-major n x n at `ptr`)."""
        p = QbProblem(n=int(n), dtype=_DTYPES[np.dtype(dtype)], q=int(ptr), ldq=int(n), q_on_device=1)
        o = self.options(**opts)
        r = QbResult()
        rc = load().qb_solve(self._h, ctypes.byref(p), ctypes.byref(o), ctypes.byref(r))
        if rc:
            _raise(rc, "qb_solve")
        return result_dict(r, int(n))

    def solve_begin_device(self, ptr: int, n: int, dtype, **opts) -> float:
        p = QbProblem(n=int(n), dtype=_DTYPES[np.dtype(dtype)], q=int(ptr), ldq=int(n), q_on_device=1)
        o = self.options(**opts)
        v = ctypes.c_double()
        rc = load().qb_solve_begin(self._h, ctypes.byref(p), ctypes.byref(o), ctypes.byref(v))
        if rc:
            _raise(rc, "qb_solve_begin")
        return v.value

    def solve_begin(self, Q: np.ndarray, **opts) -> float:
        p, keep = self._problem(Q)
        o = self.options(**opts)
        v = ctypes.c_double()
        rc = load().qb_solve_begin(self._h, ctypes.byref(p), ctypes.byref(o), ctypes.byref(v))
        del keep
        if rc:
            _raise(rc, "qb_solve_begin")
        return v.value

    def solve_finish(self, global_min: float, n: int) -> dict:
        r = QbResult()
        rc = load().qb_solve_finish(self._h, ctypes.c_double(global_min), ctypes.byref(r))
        if rc:
            _raise(rc, "qb_solve_finish")
        return result_dict(r, n)

    @staticmethod
    def _batch_problems(Qs: list) -> tuple:
        """The qb_problem descriptors of the matrices Qs (host memory, row-major, ldq = n), the
        problem sizes as an int64 array and the arrays the descriptors point into (which must
        outlive the call that reads them)."""
        count = len(Qs)
        probs = (QbProblem * count)()
        keep = [Q if (isinstance(Q, np.ndarray) and Q.flags.c_contiguous) else np.ascontiguousarray(Q) for Q in Qs]
        nl, cl, pl = [0] * count, [0] * count, [0] * count
        for i, Q in enumerate(keep):
            sh = Q.shape
            if len(sh) != 2 or sh[0] != sh[1]:
                raise ValueError(f"Q must be square, got shape {sh}")
            code = _DTYPES.get(Q.dtype)
            if code is None:
                raise TypeError(f"unsupported Q dtype {Q.dtype}")
            nl[i] = sh[0]
            cl[i] = code
            # the data address: through the buffer protocol for writable non-empty arrays (a
            # third of the cost of building __array_interface__), else the interface dict
            pl[i] = _addressof(_char_from_buffer(Q)) if (sh[0] and Q.flags.writeable) else Q.__array_interface__["data"][0]
        ns = np.array(nl, dtype=np.int64)
        if count:
            # the problem descriptors filled column by column through a structured view
            view = np.frombuffer(probs, dtype=np.dtype(QbProblem))
            view["n"] = ns
            view["ldq"] = ns
            view["dtype"] = cl
            view["q"] = pl
        return probs, ns, keep

    def solve_batch(self, Qs: list, **opts) -> "BatchResults":
        """qb_solve_batch over the matrices Qs; returns a BatchResults (a sequence of per-problem
        result dicts, decoded on access, with every field also available as one array)."""
        count = len(Qs)
        probs, ns, keep = self._batch_problems(Qs)
        o = self.options(**opts)
        res = np.zeros(count, dtype=np.dtype(QbResult))  # written in place by the library
        rc = load().qb_solve_batch(self._h, probs, count, ctypes.byref(o), res.ctypes.data_as(ctypes.POINTER(QbResult)))
        del keep
        if rc:
            _raise(rc, "qb_solve_batch")
        return BatchResults(res, ns)

    def prefix_minima(self, Q: np.ndarray, prefix_bits: int = -1) -> np.ndarray:
        """Per-prefix minimum energies in QBF's Gray visiting order (qb_prefix_minima)."""
        p, keep = self._problem(Q)
        n = p.n
        A = n - min(n, 20) if prefix_bits < 0 else int(prefix_bits)
        if A < 0 or A > 26:
            raise ValueError(f"prefix_bits={prefix_bits} out of range for n={n}")
        out = np.empty(1 << A, dtype=np.float64)
        rc = load().qb_prefix_minima(self._h, ctypes.byref(p), int(prefix_bits), out.ctypes.data)
        del keep
        if rc:
            _raise(rc, "qb_prefix_minima")
        return out

    def autotune(self, n: int, dtype) -> str:
        f = ctypes.c_int32()
        rc = load().qb_autotune(self._h, int(n), _DTYPES[np.dtype(dtype)], ctypes.byref(f))
        if rc:
            _raise(rc, "qb_autotune")
        return FORM_NAMES[f.value]


class BatchResults:
    """Results of qb_solve_batch: ``results[i]`` is problem i's result dict (the keys of
    result_dict), built when it is first read; ``results.field(name)`` is one field of every
    problem as an array, and ``results.best_X_int`` / ``results.best_E`` are shortcuts."""

    def __init__(self, arr: np.ndarray, ns: np.ndarray):
        self._arr = arr
        self._ns = ns
        self._cache = {}

    def __len__(self) -> int:
        return len(self._arr)

    def __iter__(self):
        return (self[i] for i in range(len(self)))

    def __getitem__(self, i):
        if isinstance(i, slice):
            return [self[j] for j in range(*i.indices(len(self)))]
        if i < 0:
            i += len(self)
        d = self._cache.get(i)
        if d is None:
            r = self._arr[i]
            d = result_row(r, int(self._ns[i]))
            self._cache[i] = d
        return d

    def __eq__(self, other):
        if isinstance(other, (list, tuple)):
            return list(self) == list(other)
        return NotImplemented

    def field(self, name: str) -> np.ndarray:
        return self._arr[name]

    @property
    def best_X_int(self) -> np.ndarray:
        return self._arr["best_x"]

    @property
    def best_E(self) -> np.ndarray:
        return self._arr["best_e"]


def result_row(r, n: int) -> dict:
    """result_dict of one row of a structured QbResult array."""
    x = int(r["best_x"])
    return {
        "found": bool(r["found"]),
        "best_X_int": x,
        "best_X": np.array([(x >> (n - 1 - i)) & 1 for i in range(n)], dtype=np.int32),
        "best_E": float(r["best_e"]),
        "best_E_int": int(r["best_e_int"]),
        "order_key": int(r["order_key"]),
        "pass1_min": float(r["pass1_min"]),
        "err_bound": float(r["err_bound"]),
        "states": int(r["states"]),
        "candidate_records": int(r["candidate_records"]),
        "form": FORM_NAMES.get(int(r["form_used"]), str(int(r["form_used"]))),
        "is_integer": bool(r["is_integer"]),
        "pass1_ms": float(r["pass1_ms"]),
        "pass2_ms": float(r["pass2_ms"]),
        "kernels": int(r["kernels"]),
        "kernel_ms": float(r["kernel_ms"]),
        "h2d_bytes": int(r["h2d_bytes"]),
        "d2h_bytes": int(r["d2h_bytes"]),
        "plan": {"rec_log2": int(r["rec_log2"]), "suffix_bits": int(r["suffix_bits"]),
                 "unit_log2": int(r["unit_log2"]), "tuned": bool(r["tuned"]),
                 "tc_kernel": TC_KERNELS.get(int(r["tc_kernel"]))},
    }


def result_dict(r: QbResult, n: int) -> dict:
    x = int(r.best_x)
    return {
        "found": bool(r.found),
        "best_X_int": x,
        "best_X": np.array([(x >> (n - 1 - i)) & 1 for i in range(n)], dtype=np.int32),
        "best_E": float(r.best_e),
        "best_E_int": int(r.best_e_int),
        "order_key": int(r.order_key),
        "pass1_min": float(r.pass1_min),
        "err_bound": float(r.err_bound),
        "states": int(r.states),
        "candidate_records": int(r.candidate_records),
        "form": FORM_NAMES.get(int(r.form_used), str(r.form_used)),
        "is_integer": bool(r.is_integer),
        "pass1_ms": float(r.pass1_ms),
        "pass2_ms": float(r.pass2_ms),
        "kernels": int(r.kernels),
        "kernel_ms": float(r.kernel_ms),
        "h2d_bytes": int(r.h2d_bytes),
        "d2h_bytes": int(r.d2h_bytes),
        "plan": {"rec_log2": int(r.rec_log2), "suffix_bits": int(r.suffix_bits), "unit_log2": int(r.unit_log2),
                 "tuned": bool(r.tuned), "tc_kernel": TC_KERNELS.get(int(r.tc_kernel))},
    }


_handles: dict[tuple[int, int], Handle] = {}


def handle(device: int = 0) -> Handle:
    """The calling thread's handle on `device` (created on first use)."""
    key = (int(device), threading.get_ident())
    with _lock:
        h = _handles.get(key)
        if h is None:
            h = Handle(device)
            _handles[key] = h
        return h
