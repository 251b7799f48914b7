"""The ``energy_arr`` and ``time_arr`` metrics of ``use_metrics``, one entry per prefix in
the order the reference's prefix loop visits the prefixes.

QBF records one value per Gray step of its prefix loop: the smallest energy over all
suffixes of that prefix (src/qubo_lib/solvers/qbf.py:395-412, returned as
``metrics[0]['energy_arr']`` at qbf.py:342-351).  Parallel concatenates its tasks' arrays,
each shifted by the task's prefix_E (src/qubo_lib/solvers/parallel.py:250-270).  Here the
values come from the library's exact per-prefix kernel (qb_prefix_minima); they are exact
FP64 sums, where the reference's float path carries fp32 accumulation drift.

``time_arr`` in the reference holds the duration of each epoch of the prefix loop, one per
prefix (PerformanceTimer picks labelled 'epoch', src/qubo_lib/solvers/qbf.py:362-365).  The
GPU search has no per-prefix epochs: all prefixes of a solve are searched at once by one
kernel, and every prefix covers the same number of states.  So each of the 2^A entries is
an equal share of the solve's device time (pass 1 + pass 2), and the entries sum to it.
"""
from __future__ import annotations

import numpy as np

from . import _lib

MAX_PREFIX_BITS = 26  # 2^26 entries (512 MiB of float64): the limit of qb_prefix_minima too


def _grayrank(g: np.ndarray) -> np.ndarray:
    """Inverse Gray code, elementwise (r with r ^ (r >> 1) == g)."""
    r = g.copy()
    s = 1
    while s < 64:
        r ^= r >> np.uint64(s)
        s <<= 1
    return r


def per_prefix_minima(Q: np.ndarray, prefix_bits: int, device: int = 0) -> np.ndarray:
    """QBF's energy_arr: entry i = min over suffixes of E(x) with the first ``prefix_bits``
    variables set to the MSB-first bits of gray(i)."""
    return _lib.handle(device).prefix_minima(np.asarray(Q), prefix_bits=int(prefix_bits))


def parallel_energy_arr(Q: np.ndarray, task_bits: int, prefix_bits: int, device: int = 0) -> np.ndarray:
    """Parallel(QBF)'s energy_arr: for task t = 0 .. 2^k - 1 (first k variables = the bits
    of t) the task's per-prefix minima over its next ``prefix_bits`` variables, with the
    task's prefix energy included (the full problem's energy)."""
    k, A = int(task_bits), int(prefix_bits)
    out = _lib.handle(device).prefix_minima(np.asarray(Q), prefix_bits=k + A)  # out[i] = rec[gray(i)]
    t = np.arange(1 << k, dtype=np.uint64)[:, None]
    i = np.arange(1 << A, dtype=np.uint64)[None, :]
    v = (t << np.uint64(A)) | (i ^ (i >> np.uint64(1)))  # natural prefix value of (task t, Gray step i)
    return out[_grayrank(v).astype(np.int64)].reshape(-1)


def even_time_arr(total_ms: float, prefix_bits: int) -> np.ndarray:
    """QBF's time_arr for one solve: 2^prefix_bits equal shares of total_ms (float64, ms)."""
    A = int(prefix_bits)
    if A > MAX_PREFIX_BITS:
        raise ValueError(f"time_arr needs 2^{A} entries; at most 2^{MAX_PREFIX_BITS} are kept")
    return np.full(1 << A, float(total_ms) / float(1 << A), dtype=np.float64)
