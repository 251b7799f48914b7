"""The N > 1 exchange (qubo_b200.distributed.combine_ranks) on CPU: two gloo ranks, each
searching half of the state space with the oracle as its shard searcher.  Checks the
global answer and the cross-rank tie rule (the lower order key wins, as on one GPU)."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

import oracle

N = 12


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _shard_searcher(Q, rank, world):
    """begin/finish over the states whose first variables spell this rank's share."""
    n = Q.shape[0]
    E = oracle.all_energies(Q)
    lo, hi = (1 << n) * rank // world, (1 << n) * (rank + 1) // world
    A = n - min(n, 20)

    def key(x):
        return (oracle.grayrank(x >> (n - A)) << (n - A)) | (x & ((1 << (n - A)) - 1))

    def begin():
        return float(E[lo:hi].min())

    def finish(gmin):
        xs = [x for x in range(lo, hi) if E[x] == gmin]
        if not xs:
            return {"found": False, "best_E": float("inf"), "order_key": 0, "best_X_int": 0}
        x = min(xs, key=key)
        return {"found": True, "best_E": float(E[x]), "order_key": key(x), "best_X_int": x}

    return begin, finish


def _rank_main(rank, world, port, Q, out_q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import torch.distributed as dist
    import qubo_b200  # noqa: F401
    from qubo_b200.distributed import combine_ranks
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        begin, finish = _shard_searcher(Q, rank, world)
        res, best = combine_ranks(begin, finish, "cpu")
        out_q.put((rank, bool(res["found"]), best))
    finally:
        dist.destroy_process_group()


def _run(Q, world=2):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, Q, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return sorted(got)


def test_two_ranks_random():
    rng = np.random.default_rng(5)
    U = rng.integers(-40, 41, (N, N)).astype(np.int64)
    Q = np.triu(U) + np.triu(U, 1).T
    got = _run(Q)
    ref = oracle.qbf_numpy(Q)
    for rank, found, (e, key, x) in got:
        assert e == ref["best_E"] and x == ref["best_X_int"]
    assert sum(f for _, f, _ in got) >= 1


def test_two_ranks_tie_goes_to_lower_key():
    # max-cut Q: x and its complement tie, and they sit in different halves (first bit differs)
    rng = np.random.default_rng(9)
    Q = np.zeros((N, N), np.int64)
    for i in range(N):
        for j in range(i + 1, N):
            if rng.random() < 0.5:
                w = int(rng.integers(0, 2)) * 2 - 1
                Q[i, i] -= w
                Q[j, j] -= w
                Q[i, j] += 2 * w
    got = _run(Q)
    ref = oracle.qbf_numpy(Q)
    assert all(f for _, f, _ in got)  # both ranks hold a minimiser
    for _, _, (e, key, x) in got:
        assert (e, x) == (ref["best_E"], ref["best_X_int"])
        assert x >> (N - 1) == 0  # rank 0's minimiser wins the tie
