"""The ``energy_arr`` metric of ``use_metrics``: minimum energy per prefix, in the order the
reference's prefix loop visits the prefixes.

QBF records one value per Gray step of its prefix loop: the smallest energy over all
suffixes of that prefix (src/qubo_lib/solvers/qbf.py:395-412, returned as
``metrics[0]['energy_arr']`` at qbf.py:342-351).  Parallel concatenates its tasks' arrays,
each shifted by the task's prefix_E (src/qubo_lib/solvers/parallel.py:250-270).  Here the
values come from the library's exact per-prefix kernel (qb_prefix_minima); they are exact
FP64 sums, where the reference's float path carries fp32 accumulation drift.
"""
from __future__ import annotations

import numpy as np

from . import _lib


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
