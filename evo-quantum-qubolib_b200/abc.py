"""Problem and solver contracts, mirroring the reference's ``qubo_lib.abc``.

ProblemABC follows src/qubo_lib/abc/problem_abc.py:6-89 (N, dtype, lazily built Q,
to_json / init_from_json, init_random_instance, get_Q_Ising_offset).
SolverABC follows src/qubo_lib/abc/solver_abc.py:18-92 (no constructor arguments, kwargs
only in ``solve``, the ``device`` kwarg).  Unlike the reference, solvers here run on CUDA
devices only: ``device='cpu'`` raises ValueError, and the default device is ``'cuda'``.
"""
from __future__ import annotations

from abc import ABC, abstractmethod
from typing import Optional

import numpy as np

from . import _json


class ProblemABC(ABC):
    """A QUBO instance: minimise x^T Q x over x in {0,1}^N with the full (possibly
    asymmetric) matrix Q, built on demand by ``build_Q_matrix``."""

    def __init__(self, N: int, dtype=np.float32):
        self.N = N
        self.dtype = dtype
        self.seed = None
        self.ground_E = None
        self.ground_state = None
        self.ground_utility = None

    @abstractmethod
    def build_Q_matrix(self, use_gpu: bool = False):
        """Return Q as an (N, N) numpy array (``use_gpu=True``: a CUDA torch tensor)."""

    def to_json(self) -> str:
        return _json.encode(self, indent=4)

    @staticmethod
    def init_from_json(json_str: str) -> "ProblemABC":
        return _json.decode(json_str)

    @staticmethod
    def init_random_instance(seed: int, N: int, dtype=np.float32) -> "ProblemABC":
        raise NotImplementedError

    def calculate_utility_metric(self, states) -> Optional[np.ndarray]:
        return None

    def calculate_ground(self):
        return None

    @staticmethod
    def get_Q_Ising_offset(lib, Q):
        """1/4 sum(Q) + 1/4 sum(diag Q) (src/qubo_lib/abc/problem_abc.py:86-89)."""
        return 1 / 4 * lib.sum(Q) + 1 / 4 * lib.sum(lib.diag(Q))


def _to_device(Q: np.ndarray, use_gpu: bool):
    if not use_gpu:
        return Q
    import torch
    return torch.as_tensor(np.ascontiguousarray(Q), device="cuda")


class SolverABC(ABC):
    """Base of the solvers.  Solvers take no constructor arguments and read every option
    from ``solve(problem, **kwargs)``."""

    def __init__(self):
        self.use_gpu = None
        self.kwargs = None
        self.json_str = None
        self.timer = None
        self.N = None
        self.Q = None
        self.epochs_cnt = None
        self.samples_cnt = None
        self.device_name = None
        self.device_index = None

    @abstractmethod
    def solve(self, problem: ProblemABC, **kwargs):
        ...

    def parse_device_arg(self, **kwargs):
        """'cuda' | 'cuda:N' (src/qubo_lib/abc/solver_abc.py:62-75).  'cpu' is rejected:
        the search runs only in CUDA kernels."""
        device = kwargs.get("device", "cuda")
        if not isinstance(device, str):
            raise ValueError(f"Unknown device name: {device}")
        if device == "cpu":
            raise ValueError(f"{type(self).__name__} runs on CUDA devices only: {device}")
        if device[:4] != "cuda":
            raise ValueError(f"Unknown device name: {device}")
        idx = int(device[5:]) if len(device) > 5 else 0
        self.use_gpu = True
        self.device_index = idx
        self.device_name = device
        return idx

    @staticmethod
    def gimme_lib():
        return np
