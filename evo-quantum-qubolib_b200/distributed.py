"""Multi-GPU exhaustive search with one process per GPU over torch.distributed.

The search space is split into contiguous shares of prefix tiles, one per rank (the
reference's bit fixing, src/qubo_lib/solvers/parallel.py:145-157, without process pickling).
There are two collectives, both a few bytes: an all-reduce (MIN) of the ranks' pass-1
minima, so that every rank selects its candidate records against the global minimum, and an
all-gather of each rank's best (energy, tie key, state) record.  Ties across ranks resolve
by the tie key, i.e. exactly as on one GPU.
"""
from __future__ import annotations

import numpy as np

from . import _lib


def _gather_best(res: dict, device):
    import torch
    import torch.distributed as dist
    # (found, E, key_hi, key_lo, x_hi, x_lo): keys and states travel as two 32-bit halves
    rec = torch.tensor([float(res["found"]), res["best_E"] if res["found"] else float("inf"),
                        float(res["order_key"] >> 32), float(res["order_key"] & 0xFFFFFFFF),
                        float(res["best_X_int"] >> 32), float(res["best_X_int"] & 0xFFFFFFFF)],
                       dtype=torch.float64, device=device)
    out = [torch.empty_like(rec) for _ in range(dist.get_world_size())]
    dist.all_gather(out, rec)
    best = None
    for t in out:
        f, e, kh, kl, xh, xl = t.tolist()
        if not f:
            continue
        key = (int(kh) << 32) | int(kl)
        x = (int(xh) << 32) | int(xl)
        if best is None or (e, key) < (best[0], best[1]):
            best = (e, key, x)
    return best


def combine_ranks(begin, finish, comm_device):
    """The exchange of a sharded search, independent of how a shard is searched.

    begin() searches this rank's share and returns its pass-1 minimum; finish(global_min)
    re-evaluates the share's candidates against the global minimum and returns the share's
    result dict (found, best_E, order_key, best_X_int).  The collectives run on tensors of
    comm_device ("cuda:i" under NCCL, "cpu" under gloo).  Returns (this rank's result,
    (E, key, X) of the global winner)."""
    import torch
    import torch.distributed as dist
    lmin = begin()
    t = torch.tensor([lmin], dtype=torch.float64, device=comm_device)
    dist.all_reduce(t, op=dist.ReduceOp.MIN)
    res = finish(float(t.item()))
    best = _gather_best(res, comm_device)
    if best is None:
        raise RuntimeError("no rank holds a minimising state")
    return res, best


def solve_sharded(Q: np.ndarray, form: str = "auto", tie_rule: str = "qbf", fixed_bits: int = 0,
                  prefix_bits: int = -1, device: int | None = None, Q_device_ptr: int | None = None) -> dict:
    """Exhaustive minimum of Q across all ranks of the default process group.

    Every rank passes the same Q (host array, or a device copy through Q_device_ptr).
    Returns the global answer on every rank, plus this rank's own search statistics.
    """
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(), dist.get_world_size()
    if device is None:
        device = torch.cuda.current_device()
    h = _lib.handle(device)
    stream = torch.cuda.current_stream(device).cuda_stream
    opts = dict(form=form, tie_rule=tie_rule, fixed_bits=fixed_bits, prefix_bits=prefix_bits, shard_index=rank,
                shard_count=world, stream=stream)
    n = Q.shape[0]

    def begin():
        if Q_device_ptr is not None:
            return h.solve_begin_device(Q_device_ptr, n, Q.dtype, **opts)
        return h.solve_begin(Q, **opts)

    res, (e, key, x) = combine_ranks(begin, lambda gmin: h.solve_finish(gmin, n), f"cuda:{device}")
    out = dict(res)
    out.update(best_E=e, order_key=key, best_X_int=x,
               best_X=np.array([(x >> (n - 1 - i)) & 1 for i in range(n)], dtype=np.int32),
               local_found=res["found"], found=True, world_size=world)
    return out


def merge_shard_results(results: list[dict]) -> dict:
    """Host-side merge of per-shard results (same rule as the all-gather above)."""
    found = [r for r in results if r["found"]]
    if not found:
        raise RuntimeError("no shard holds a minimising state")
    return min(found, key=lambda r: (r["best_E"], r["order_key"]))
