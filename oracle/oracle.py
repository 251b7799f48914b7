"""oracle/oracle.py -- TEST INFRASTRUCTURE ONLY.

The checker for the CUDA path: a CPU restatement of the reference's exhaustive QUBO
search (cloud-ru-tech/evo-quantum-qubolib).  Only tests/, the smoke() check of
__graft_entry__.py and bench.py's CPU-baseline / reference legs may import this module.
The product package never does.

Two independent restatements live here:

* ``qbf_port`` / ``parallel_port`` call the C port in ``qbf_port.c`` (built into
  ``oracle/liboracle_qbf.so``): the reference's own algorithm -- Gray-ordered prefix loop,
  cached suffix energies and cross rows, first-index argmin per prefix, strict ``<``
  against a running best that starts at (E=0, x=0) (src/qubo_lib/solvers/qbf.py:188-230,
  :291-325, :395-412) and the bit-fixing of Parallel (src/qubo_lib/solvers/parallel.py:
  145-157, 273-300; src/qubo_lib/problems/reduced_problem.py:31-46).
* ``qbf_numpy`` evaluates every state with numpy (small n only) and applies the tie rule
  that the reference's loop implies: among minimal-energy states, the smallest inverse-Gray
  rank of the A-bit prefix, then the smallest suffix integer.

Parity status: pinned.  Both restatements are checked against golden vectors produced by
running the reference itself (tests/golden/make_golden.py) and against the notebook outputs
of the reference (showcase.ipynb).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_qbf.so")
_SRC = os.path.join(_HERE, "qbf_port.c")


class OqResult(ctypes.Structure):
    _fields_ = [
        ("best_e", ctypes.c_double),
        ("best_e_int", ctypes.c_int64),
        ("best_x", ctypes.c_uint64),
        ("glob_pref", ctypes.c_uint64),
        ("glob_x", ctypes.c_uint64),
        ("epochs", ctypes.c_int64),
        ("A", ctypes.c_int32),
        ("B", ctypes.c_int32),
        ("status", ctypes.c_int32),
    ]


def build(force: bool = False) -> str:
    """Compile qbf_port.c into liboracle_qbf.so (gcc, OpenMP)."""
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(_SRC):
        cmd = ["gcc", "-O3", "-march=x86-64-v2", "-fopenmp", "-fPIC", "-shared", _SRC, "-o", _LIB_PATH, "-lm"]
        subprocess.run(cmd, check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        L.oq_qbf_solve.argtypes = [ctypes.c_int, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(OqResult)]
        L.oq_qbf_solve.restype = ctypes.c_int
        L.oq_parallel_solve.argtypes = [ctypes.c_int, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, ctypes.POINTER(OqResult)]
        L.oq_parallel_solve.restype = ctypes.c_int
        L.oq_energy.argtypes = [ctypes.c_int, dp, ctypes.c_uint64]
        L.oq_energy.restype = ctypes.c_double
        L.oq_all_minimisers.argtypes = [ctypes.c_int, dp, ctypes.POINTER(ctypes.c_uint64), ctypes.c_int64, dp]
        L.oq_all_minimisers.restype = ctypes.c_int64
        L.oq_reduce.argtypes = [ctypes.c_int, dp, ctypes.c_int, ctypes.c_uint64, dp]
        L.oq_reduce.restype = ctypes.c_double
        _lib = L
    return _lib


def _as_f64(Q: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(Q), dtype=np.float64)


def _is_int(Q: np.ndarray) -> bool:
    return np.issubdtype(np.asarray(Q).dtype, np.integer)


def qbf_port(Q, A: int = -1, correction_period: int = 1024) -> dict:
    """QBF().solve(Just_Q(Q), A=A) restated in C.  A < 0 selects QBF's default CPU split."""
    Qd = _as_f64(Q)
    n = Qd.shape[0]
    r = OqResult()
    rc = lib().oq_qbf_solve(n, Qd.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), int(_is_int(Q)), int(A),
                            int(correction_period), ctypes.byref(r))
    if rc:
        raise RuntimeError(f"oq_qbf_solve failed: {rc}")
    return _pack(r, n, _is_int(Q))


def parallel_port(Q, splits_cnt: int, A_sub: int = -1, nthreads: int = 0, correction_period: int = 1024) -> dict:
    """Parallel(QBF, splits_cnt).solve(Just_Q(Q)) restated in C (lowest task id wins ties)."""
    Qd = _as_f64(Q)
    n = Qd.shape[0]
    k = int(splits_cnt).bit_length() - 1
    r = OqResult()
    rc = lib().oq_parallel_solve(n, Qd.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), int(_is_int(Q)), k,
                                 int(A_sub), int(correction_period), int(nthreads), ctypes.byref(r))
    if rc:
        raise RuntimeError(f"oq_parallel_solve failed: {rc}")
    return _pack(r, n, _is_int(Q))


def _pack(r: OqResult, n: int, is_int: bool) -> dict:
    x = int(r.best_x)
    return {
        "best_E": int(r.best_e_int) if is_int else float(r.best_e),
        "best_X_int": x,
        "best_X": [(x >> (n - 1 - i)) & 1 for i in range(n)],
        "glob_pref": int(r.glob_pref),
        "glob_X": int(r.glob_x),
        "epochs": int(r.epochs),
        "A": int(r.A),
        "B": int(r.B),
    }


def energy(Q, X: int) -> float:
    """E(x) = x^T Q x of the MSB-first state integer X (FP64; exact for integer Q)."""
    Qd = _as_f64(Q)
    return lib().oq_energy(Qd.shape[0], Qd.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), int(X))


def all_minimisers(Q, cap: int = 1 << 16):
    """(E_min, [X...]) of an integer-valued Q by brute force, n <= 26."""
    Qd = _as_f64(Q)
    n = Qd.shape[0]
    out = (ctypes.c_uint64 * cap)()
    emin = ctypes.c_double()
    cnt = lib().oq_all_minimisers(n, Qd.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), out, cap,
                                  ctypes.byref(emin))
    return emin.value, [int(out[i]) for i in range(min(cnt, cap))], int(cnt)


# ---------------------------------------------------------------------------------------
# numpy restatement (small n)
# ---------------------------------------------------------------------------------------

def grayrank(g: int) -> int:
    """Inverse Gray code: the step index i with i ^ (i >> 1) == g."""
    i = 0
    while g:
        i ^= g
        g >>= 1
    return i


def all_energies(Q) -> np.ndarray:
    """E[X] for every MSB-first state X (FP64; exact for integer Q), n <= 24."""
    Qd = _as_f64(Q)
    n = Qd.shape[0]
    X = ((np.arange(1 << n, dtype=np.int64)[:, None] >> np.arange(n - 1, -1, -1)) & 1).astype(np.float64)
    out = np.empty(1 << n)
    step = 1 << 16
    for s in range(0, 1 << n, step):
        xs = X[s:s + step]
        out[s:s + step] = np.einsum("ij,jk,ik->i", xs, Qd, xs)
    return out


def qbf_key(X: int, n: int, A: int) -> tuple:
    """Order key of the reference QBF loop for split (A, n-A): (grayrank(prefix), suffix)."""
    B = n - A
    return (grayrank(X >> B), X & ((1 << B) - 1))


def parallel_key(X: int, n: int, k: int, A_sub: int) -> tuple:
    """Order key of Parallel(QBF, 2^k) with each task split (A_sub, n-k-A_sub)."""
    m = n - k
    B = m - A_sub
    sub = X & ((1 << m) - 1)
    return (X >> m, grayrank(sub >> B), sub & ((1 << B) - 1))


def qbf_numpy(Q, A: int | None = None) -> dict:
    """Exhaustive minimum with the QBF tie rule, by full enumeration (n <= 24)."""
    Qd = _as_f64(Q)
    n = Qd.shape[0]
    if A is None:
        A = n - min(n, 20)
    E = all_energies(Q)
    emin = E.min()
    if emin >= 0:
        X = 0
    else:
        cands = np.flatnonzero(E == emin)
        X = int(min(cands, key=lambda c: qbf_key(int(c), n, A)))
    return {"best_E": (int(round(E[X])) if _is_int(Q) else float(E[X])), "best_X_int": X,
            "best_X": [(X >> (n - 1 - i)) & 1 for i in range(n)]}


def default_split(n: int) -> tuple[int, int]:
    b = min(n, 20)
    return n - b, b


def qbf1_tid(s: int) -> int:
    """Thread of the reference QB_F1 kernel that owns 18-bit suffix column s
    (grid 256 x 64, column = block*1024 + 64*col + thread; src/qubo_lib/solvers/qbf1.py:195)."""
    return (s >> 10) * 64 + (s & 63)


def qbf1_numpy(Q) -> dict:
    """Answer order of the reference QB_F1 (src/qubo_lib/solvers/qbf1.py:214-264) on exact
    energies: among minimal states, the lowest owning thread, then the earliest Gray prefix
    step; the suffix is then the smallest one of that prefix with the minimal energy.
    n in [19, 24]."""
    Qd = _as_f64(Q)
    n = Qd.shape[0]
    A = n - 18
    E = all_energies(Q)
    emin = E.min()
    if emin >= 0:
        X = 0
    else:
        cands = np.flatnonzero(E == emin)
        Xw = int(min(cands, key=lambda c: (qbf1_tid(int(c) & ((1 << 18) - 1)), grayrank(int(c) >> 18))))
        p = Xw >> 18
        row = E[p << 18:(p + 1) << 18]
        X = (p << 18) | int(np.flatnonzero(row == emin)[0])
    return {"best_E": int(round(E[X])), "best_X_int": X, "best_X": [(X >> (n - 1 - i)) & 1 for i in range(n)]}


def prefix_minima_numpy(Q, A: int) -> np.ndarray:
    """QBF's energy_arr restated: entry i is the smallest energy over all suffixes of the
    prefix visited at Gray step i, i.e. the A MSB-first bits of gray(i)
    (src/qubo_lib/solvers/qbf.py:291-325 visiting order, :395-412 one value per step).
    FP64; exact for integer Q.  n <= 24."""
    E = all_energies(Q)
    n = np.asarray(Q).shape[0]
    per_prefix = E.reshape(1 << A, 1 << (n - A)).min(axis=1)
    i = np.arange(1 << A)
    return per_prefix[i ^ (i >> 1)]


def parallel_energy_arr_numpy(Q, k: int, A_sub: int) -> np.ndarray:
    """Parallel(QBF)'s energy_arr restated: tasks in task order (one worker), each task's
    per-prefix minima of its ReducedProblem plus the task's prefix_E, which is the full
    problem's energy (src/qubo_lib/solvers/parallel.py:250-270, 145-157)."""
    E = all_energies(Q)
    n = np.asarray(Q).shape[0]
    B = n - k - A_sub
    per = E.reshape(1 << k, 1 << A_sub, 1 << B).min(axis=2)
    i = np.arange(1 << A_sub)
    return per[:, i ^ (i >> 1)].reshape(-1)


def qbf1_int16_numpy(Q) -> dict:
    """The reference QB_F1 restated with its int16 arithmetic (numpy int16 wraps modulo 2^16
    as the reference's cupy int16 arrays and int16 kernel variables do):
      prepare (src/qubo_lib/solvers/qbf1.py:86-133): B = 18, A = n - 18; BB = int16 suffix
      energies; AA[i] = int16 E_pre(gray(i)); ABBA = (Q_0B + Q_1A^T) X_B^T in int16;
      QB_F1_kernel (:179-249): 256 x 64 threads, thread tid owns columns
      (tid >> 6) * 1024 + 64 * c + (tid & 63), c < 16; running int16 sums updated by the
      flipped prefix row per Gray step; tested = int16(AA[i] + min); strict < keeps the
      earliest step; the initial best is the min over the columns at prefix 0;
      pack_results (:253-289): lowest thread with the smallest int16 best; its prefix's
      int16 row argmin (first) gives the suffix; best_E is the thread's int16 value.
    n in [19, 31] (vectorised over the 16384 threads; 2^(n-18) steps, about 2.5 s at n = 29)."""
    Q = np.asarray(Q)
    assert Q.dtype == np.int16
    n = Q.shape[0]
    A, B = n - 18, 18
    S = np.arange(1 << B, dtype=np.int64)
    XB = ((S[:, None] >> np.arange(B - 1, -1, -1)) & 1).astype(np.int64)       # 2^18 x 18
    Q64 = Q.astype(np.int64)
    BB = np.einsum("sj,jl,sl->s", XB, Q64[A:, A:], XB).astype(np.int16)
    C = (Q[:A, A:] + Q[A:, :A].T).astype(np.int16).astype(np.int64)            # int16 sum, wraps
    ABBA = (C @ XB.T).astype(np.int16)                                          # A x 2^18
    I = np.arange(1 << A, dtype=np.int64)
    G = I ^ (I >> 1)
    XA = ((G[:, None] >> np.arange(A - 1, -1, -1)) & 1).astype(np.int64)
    AA = np.einsum("ik,kl,il->i", XA, Q64[:A, :A], XA).astype(np.int16)
    tid = np.arange(16384)
    cols = ((tid >> 6) * 1024)[:, None] + 64 * np.arange(16)[None, :] + (tid & 63)[:, None]
    E = BB[cols]                                                                # int16
    best = E.min(axis=1)
    bx = np.zeros(16384, dtype=np.int64)
    for i in range(1, 1 << A):
        g = i ^ (i >> 1)
        prev = (i - 1) ^ ((i - 1) >> 1)
        kb = (i & -i).bit_length() - 1
        row = A - 1 - kb
        if g > prev:
            E = E + ABBA[row][cols]
        else:
            E = E - ABBA[row][cols]
        m = E.min(axis=1)
        t = (AA[i] + m).astype(np.int16)
        upd = t < best
        bx = np.where(upd, g, bx)
        best = np.minimum(best, t)
    idx = int(np.argmin(best))
    p = int(bx[idx])
    tmp = BB.copy()
    for k in range(A):
        if (p >> (A - 1 - k)) & 1:
            tmp = tmp + ABBA[k]
    s = int(np.argmin(tmp))
    X = (p << B) | s
    return {"best_E": int(best[idx]), "best_X_int": X, "exact_E": energy(Q, X)}
