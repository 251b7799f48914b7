"""Resumable exhaustive search: the search space cut into contiguous shares (the same
prefix-tile shares the multi-GPU path uses), solved one after another with the running best
written to a small JSON checkpoint after each share.  A run that stops (a job time limit, a
preempted node) restarts where it stopped.  The reference has no checkpoint for QBF; its
closest equivalents are QBF's fixed-prefix sub-interval and ReducedProblem task ids
(src/qubo_lib/solvers/qbf.py:188, src/qubo_lib/problems/reduced_problem.py).
"""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np

from . import _lib


def _fingerprint(Q: np.ndarray, opts: dict) -> str:
    h = hashlib.sha256()
    h.update(str(Q.dtype).encode())
    h.update(str(Q.shape).encode())
    h.update(np.ascontiguousarray(Q).tobytes())
    h.update(json.dumps(opts, sort_keys=True).encode())
    return h.hexdigest()


def _better(a: dict, b: dict | None) -> bool:
    """a before b in (energy, tie key) order."""
    return b is None or (a["best_E"], a["order_key"]) < (b["best_E"], b["order_key"])


def solve_resumable(Q: np.ndarray, chunks: int, path: str, device: int = 0, form: str = "auto",
                    tie_rule: str = "qbf", fixed_bits: int = 0, prefix_bits: int = -1,
                    max_chunks_this_call: int | None = None) -> dict:
    """Exhaustive minimum of Q over ``chunks`` shares, checkpointed in ``path``.

    Returns a dict with ``done`` (all shares searched), ``next`` (first share not yet
    searched), ``best_E``, ``best_X_int``, ``best_X`` and ``order_key`` of the best state so
    far (the tie rule's choice, as one call over the whole space would give), and
    ``states`` searched so far.  ``max_chunks_this_call`` stops early (for time-boxed jobs).
    A checkpoint written for another Q, tie rule or number of shares raises ValueError."""
    Q = np.ascontiguousarray(Q)
    n = Q.shape[0]
    opts = dict(form=form, tie_rule=tie_rule, fixed_bits=int(fixed_bits), prefix_bits=int(prefix_bits),
                chunks=int(chunks))
    fp = _fingerprint(Q, opts)
    state = {"fingerprint": fp, "next": 0, "best": None, "states": 0}
    if os.path.exists(path):
        with open(path) as f:
            state = json.load(f)
        if state.get("fingerprint") != fp:
            raise ValueError(f"checkpoint {path} belongs to another problem or options")
    h = _lib.handle(device)
    done_now = 0
    while state["next"] < chunks and (max_chunks_this_call is None or done_now < max_chunks_this_call):
        i = state["next"]
        lmin = h.solve_begin(Q, form=form, tie_rule=tie_rule, fixed_bits=fixed_bits, prefix_bits=prefix_bits,
                             shard_index=i, shard_count=chunks)
        r = h.solve_finish(lmin, n)
        if r["found"]:
            cand = {"best_E": float(r["best_E"]), "order_key": int(r["order_key"]), "best_X_int": int(r["best_X_int"])}
            if _better(cand, state["best"]):
                state["best"] = cand
        state["states"] += int(r["states"])
        state["next"] = i + 1
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(state, f)
        os.replace(tmp, path)  # the checkpoint is either the old or the new one, never torn
        done_now += 1
    best = state["best"]
    out = {"done": state["next"] >= chunks, "next": state["next"], "states": state["states"]}
    if best is not None:
        x = best["best_X_int"]
        out.update(best_E=best["best_E"], order_key=best["order_key"], best_X_int=x,
                   best_X=np.array([(x >> (n - 1 - k)) & 1 for k in range(n)], dtype=np.int32))
    return out
