"""Interval timer with the reference's semantics (src/qubo_lib/utils/perf_timer.py:4-39).

On a GPU every ``pick_time`` records a CUDA event on the current stream and synchronises it,
so each interval covers the device work issued since the previous pick; on the host it is a
``perf_counter`` interval.  ``get_time_from_start`` is the sum of all intervals in ms.
"""
from __future__ import annotations

import time


class PerformanceTimer:
    def __init__(self, use_gpu: bool = False):
        self.times = []
        self.use_gpu = bool(use_gpu)
        if self.use_gpu:
            import torch
            self._torch = torch
            self.start_event = torch.cuda.Event(enable_timing=True)
            self.start_event.record()
            self.last_event = self.start_event
        else:
            self.start_time = time.perf_counter()

    def pick_time(self, label=None):
        if self.use_gpu:
            ev = self._torch.cuda.Event(enable_timing=True)
            ev.record()
            ev.synchronize()
            ms = self.last_event.elapsed_time(ev)
            self.last_event = ev
        else:
            now = time.perf_counter()
            ms = (now - self.start_time) * 1000
            self.start_time = now
        self.times.append((ms, label))

    def get_time_from_start(self):
        return sum(t for t, _ in self.times)
