"""Seeded synthetic inputs for the benchmark configurations.

Each builder returns the Q matrix (numpy) the way the workload is defined; the matrices
come from this package's problem classes, which draw the same numbers as the reference's
generators (tests check them against matrices produced by the reference itself).

1. ``random_f32_n20``     RandomQUBO(seed 0, N=20, U[-1, 1), float32), symmetrised (Q + Q^T) / 2
2. ``random_i16_n32``     RandomQUBO(seed 0, N=32, integers in [-100, 100], int16),
                          Q = triu(U) + triu(U, 1)^T
3. ``tsp6_int``           6-city TSP (36 variables): integer distances U{1..100} from
                          default_rng(seed), symmetric; Q = TSP.qubo_from_distances(w), int32
                          (penalty 2 * max(w) + 1, the reference's formula)
4. ``maxcut_er_n40``      MaxCut on G(40, 0.5) with weights in {-1, +1} from default_rng(seed)
5. ``batch_f32``          4096 instances, instance i: n_i = U{16..28} and G ~ N(0, 1)^{n x n}
                          from default_rng(seed + i); Q = ((G + G^T) / 2).astype(float32)
"""
from __future__ import annotations

import numpy as np

from .problems import MaxCut, RandomQUBO, TSP


def random_f32_n20(seed: int = 0) -> np.ndarray:
    q0 = RandomQUBO.init_random_instance(seed=seed, N=20, low=-1, high=1, dtype=np.float32).build_Q_matrix()
    return ((q0 + q0.T) / 2).astype(np.float32)


def random_i16_n32(seed: int = 0, n: int = 32) -> np.ndarray:
    U = RandomQUBO.init_random_instance(seed=seed, N=n, low=-100, high=101, dtype=np.int16).build_Q_matrix()
    return (np.triu(U) + np.triu(U, 1).T).astype(np.int16)


def tsp_int(n_cities: int = 6, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    w = rng.integers(1, 101, (n_cities, n_cities))
    w = np.triu(w, 1)
    w = w + w.T
    return TSP.qubo_from_distances(w.astype(np.float64)).astype(np.int32)


def tsp6_int(seed: int = 0) -> np.ndarray:
    return tsp_int(6, seed)


def maxcut_er(n: int = 40, seed: int = 0, p: float = 0.5) -> np.ndarray:
    return MaxCut.init_random_instance(seed=seed, N=n, p=p).build_Q_matrix()


def batch_instance(i: int, seed: int = 0, n_lo: int = 16, n_hi: int = 28) -> np.ndarray:
    rng = np.random.default_rng(seed + i)
    n = int(rng.integers(n_lo, n_hi + 1))
    G = rng.standard_normal((n, n))
    return ((G + G.T) / 2).astype(np.float32)


def batch_f32(count: int = 4096, seed: int = 0, n_lo: int = 16, n_hi: int = 28) -> list:
    return [batch_instance(i, seed, n_lo, n_hi) for i in range(count)]
