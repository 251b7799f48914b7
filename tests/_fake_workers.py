"""Stand-in device workers for the CPU tests of Parallel's multi-process exchange (spawned
by tests/test_parallel_workers_cpu.py; no GPU is touched)."""
import os
import time


def ok_worker(device, Q, opts, shard_index, shard_count, inbox, outbox):
    outbox.put(("min", shard_index, float(10 - shard_index)))
    gmin = inbox.get(timeout=60)
    outbox.put(("res", shard_index, {"found": shard_index == shard_count - 1, "gmin": gmin, "device": device,
                                     "time_ms": 1.0, "states": 1 << 10}))


def err_worker(device, Q, opts, shard_index, shard_count, inbox, outbox):
    if shard_index == 1:
        outbox.put(("err", shard_index, "ValueError: injected"))
        return
    ok_worker(device, Q, opts, shard_index, shard_count, inbox, outbox)


def hang_worker(device, Q, opts, shard_index, shard_count, inbox, outbox):
    time.sleep(120)


def crash_worker(device, Q, opts, shard_index, shard_count, inbox, outbox):
    if shard_index == 0:
        os._exit(3)
    ok_worker(device, Q, opts, shard_index, shard_count, inbox, outbox)
