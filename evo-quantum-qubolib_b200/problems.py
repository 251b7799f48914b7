"""QUBO problem classes (the reference's ``qubo_lib.problems``).

Every class builds the same Q matrix as its reference counterpart from the same
parameters; the random generators draw from numpy's PCG64 in the same call order, so a
seed gives an identical matrix:

* RandomQUBO     -- src/qubo_lib/problems/random_qubo.py:7-61
* Just_Q         -- src/qubo_lib/problems/just_Q.py:5-38
* TSP            -- src/qubo_lib/problems/tsp.py:15-321 (Q construction, path encoding;
                    the OR-Tools ground-state helper is not part of this package)
* MaxCut         -- Q rule of src/qubo_lib/problems/max_cut.py:56-62 (per edge (i, j, w):
                    Q_ii -= w, Q_jj -= w, Q_ij += 2w, so E(x) = -cut(x)); graphs come from
                    an edge list, a G-set text file, or a seeded Erdos-Renyi draw
* ReducedProblem -- src/qubo_lib/problems/reduced_problem.py:7-57 (bit fixing)
"""
from __future__ import annotations

import numpy as np

from .abc import ProblemABC, _to_device


class RandomQUBO(ProblemABC):
    """Q with i.i.d. entries: integers uniform in [low, high) for integer dtypes, else
    ``low + U[0,1) * (high - low)`` in the problem dtype.  Not symmetric."""

    def __init__(self, N: int, dtype=np.float32):
        super().__init__(N, dtype)
        self.low = -100
        self.high = 100

    def build_Q_matrix(self, use_gpu: bool = False):
        gen = np.random.Generator(np.random.PCG64(self.seed))
        shape = (self.N, self.N)
        if np.issubdtype(self.dtype, np.integer):
            Q = gen.integers(low=self.low, high=self.high, size=shape, dtype=self.dtype)
        else:
            Q = self.low + gen.random(size=shape, dtype=self.dtype) * (self.high - self.low)
        assert Q.dtype == self.dtype
        return _to_device(Q, use_gpu)

    @staticmethod
    def init_random_instance(seed: int, N: int, low=-100, high=100, dtype=np.float32) -> "RandomQUBO":
        obj = RandomQUBO(N, dtype)
        obj.seed = seed
        obj.low = low
        obj.high = high
        return obj


class Just_Q(ProblemABC):
    """A user-given matrix; N and dtype are taken from it."""

    def __init__(self, Q):
        Q = np.asarray(Q)
        self.Q_matrix = Q
        super().__init__(Q.shape[0], Q.dtype)

    def build_Q_matrix(self, use_gpu: bool = False):
        assert self.Q_matrix.dtype == self.dtype
        return _to_device(self.Q_matrix, use_gpu)

    @staticmethod
    def init_random_instance(*args, **kwargs):
        raise NotImplementedError("It's a user-defined matrix, for random instance better use RandomQUBO class")


class TSP(ProblemABC):
    """Travelling salesman as QUBO: x[city * n + position] = 1 when ``city`` is visited at
    ``position``; open-path cost plus one-hot penalties of weight 2 * max(w) + 1."""

    def __init__(self, N: int, dtype=np.float32):
        self.cities = None
        self.best_path = None
        self.n_cities = None
        super().__init__(N, dtype)

    @staticmethod
    def init_from_cities(cities, dtype=np.float32) -> "TSP":
        n = cities.shape[0]
        obj = TSP(n * n, dtype=dtype)
        obj.n_cities = n
        obj.cities = cities.astype(dtype)
        return obj

    @staticmethod
    def init_random_instance(seed: int, n_cities: int, low=0, high=100, dtype=np.float32) -> "TSP":
        gen = np.random.Generator(np.random.PCG64(seed))
        cities = gen.uniform(low=low, high=high, size=(n_cities, 2)).astype(dtype)
        obj = TSP.init_from_cities(cities, dtype)
        obj.seed = seed
        return obj

    def build_Q_matrix(self, use_gpu: bool = False):
        xs, ys = self.cities[:, 0], self.cities[:, 1]
        return _to_device(self.qubo_from_positions(xs, ys).astype(self.dtype), use_gpu)

    @staticmethod
    def qubo_from_positions(x_pos, y_pos, lib=np):
        """Euclidean distances (computed in the coordinates' dtype, stored as float64)."""
        n = x_pos.shape[0]
        dist = np.zeros((n, n))
        for i in range(n):
            for j in range(i + 1, n):
                d = np.sqrt((x_pos[i] - x_pos[j]) ** 2 + (y_pos[i] - y_pos[j]) ** 2)
                dist[i][j] = d
                dist[j][i] = d
        return TSP.qubo_from_distances(dist)

    @staticmethod
    def qubo_from_distances(w, lib=np):
        """Upper-triangular QUBO of the open-path TSP with distance matrix w
        (src/qubo_lib/problems/tsp.py:286-321).

        cost:     Q[(i, p), (j, p+1)] += w[i, j] for p < n-1
        penalty:  P = 2 * max(w) + 1 times C, where C[(i, p), (j, p)] = 1 (i != j) and
                  C[(i, p), (i, k)] = 1 (p != k), C[(i, p), (i, p)] = -1
        result:   triu(Q) + tril(Q, -1)^T
        """
        w = np.asarray(w)
        n = w.shape[0]
        N = n * n
        idx = np.arange(N).reshape(n, n)  # idx[city, pos]
        Q = np.zeros((N, N))
        for p in range(n - 1):
            # every (i at p) -> (j at p+1) pair carries w[i, j]
            Q[np.ix_(idx[:, p], idx[:, p + 1])] += w
        penalty = 2 * np.max(w) + 1
        C = np.zeros((N, N))
        same_pos = np.equal.outer(np.arange(N) % n, np.arange(N) % n)
        same_city = np.equal.outer(np.arange(N) // n, np.arange(N) // n)
        C[same_pos | same_city] = 1.0
        C[np.arange(N), np.arange(N)] = -1.0
        Q += penalty * C
        return np.triu(Q) + np.tril(Q, k=-1).T

    @staticmethod
    def encode_path_to_x(path):
        n = len(path)
        x = np.zeros(n * n)
        for pos, city in enumerate(path):
            x[city * n + pos] = 1
        return x

    @staticmethod
    def decode_x_to_path(wide_x):
        wide_x = np.asarray(wide_x)
        N = wide_x.shape[0]
        n = int(round(N ** 0.5))
        assert n * n == N
        assert wide_x.sum() == n
        path = np.zeros(n, dtype=np.int32)
        for k in np.flatnonzero(wide_x == 1):
            path[k % n] = k // n
        return path

    @staticmethod
    def is_valid_tour(wide_x) -> bool:
        x = np.asarray(wide_x).reshape(-1)
        n = int(round(x.shape[0] ** 0.5))
        m = x.reshape(n, n)
        return bool((m.sum(axis=0) == 1).all() and (m.sum(axis=1) == 1).all())

    @staticmethod
    def get_path_length(path, xs, ys):
        total = 0
        for u, v in zip(path[:-1], path[1:]):
            total += ((xs[u] - xs[v]) ** 2 + (ys[u] - ys[v]) ** 2) ** 0.5
        return total

    def calculate_state_utility_metric(self, x):
        path = TSP.decode_x_to_path(x)
        return TSP.get_path_length(path, self.cities[:, 0], self.cities[:, 1])

    def calculate_utility_metric(self, states) -> np.ndarray:
        xs = states.get_wide_vectors()
        return np.array([self.calculate_state_utility_metric(x) for x in xs])

    def calculate_ground(self, use_gpu: bool = False):
        raise NotImplementedError("the OR-Tools ground-state heuristic is not part of qubo_b200")


class MaxCut(ProblemABC):
    """MaxCut as QUBO with E(x) = -cut(x).  Build from an edge list (0-based vertices)."""

    def __init__(self, N: int, edges, dtype=np.int32, name: str | None = None):
        super().__init__(N, dtype)
        self.edges = [(int(i), int(j), w) for i, j, w in edges]
        self.instance_name = name

    def build_Q_matrix(self, use_gpu: bool = False):
        Q = np.zeros((self.N, self.N), dtype=self.dtype)
        for i, j, w in self.edges:
            Q[i, i] -= w
            Q[j, j] -= w
            Q[i, j] += 2 * w
        return _to_device(Q, use_gpu)

    @staticmethod
    def from_gset_text(text: str, dtype=np.int32, name: str | None = None) -> "MaxCut":
        """Parse the G-set format: ``V E`` then ``i j w`` lines with 1-based vertices."""
        lines = [ln.split() for ln in text.strip().splitlines() if ln.strip()]
        nv, ne = int(lines[0][0]), int(lines[0][1])
        edges = [(int(a) - 1, int(b) - 1, int(c)) for a, b, c in lines[1:1 + ne]]
        return MaxCut(nv, edges, dtype=dtype, name=name)

    @staticmethod
    def init_random_instance(seed: int, N: int, p: float = 0.5, dtype=np.int32) -> "MaxCut":
        """Erdos-Renyi G(N, p) with weights uniform in {-1, +1}: edge (i<j) present when
        U[i, j] < p for U = rng.random((N, N)); weight = 2 * rng.integers(0, 2, (N, N))[i, j] - 1."""
        rng = np.random.default_rng(seed)
        present = rng.random((N, N)) < p
        sign = rng.integers(0, 2, (N, N)) * 2 - 1
        edges = [(i, j, int(sign[i, j])) for i in range(N) for j in range(i + 1, N) if present[i, j]]
        obj = MaxCut(N, edges, dtype=dtype)
        obj.seed = seed
        return obj

    def cut_value(self, x) -> int:
        x = np.asarray(x).reshape(-1)
        return int(sum(w for i, j, w in self.edges if x[i] != x[j]))


class ReducedProblem(ProblemABC):
    """The base problem with its first ``len(prefix)`` variables fixed to ``prefix``.

    prefix_E = p^T Q[:k, :k] p and the reduced matrix is
    Q[k:, k:] + diag(p (Q[:k, k:] + Q[k:, :k]^T)), in the base problem's dtype; prefix_E is
    set when the matrix is built."""

    def __init__(self, problem: ProblemABC, prefix):
        prefix = np.asarray(prefix)
        self.base_problem = problem
        self.A = prefix.shape[0]
        self.prefix = prefix
        self.prefix_E = None
        super().__init__(problem.N - self.A, problem.dtype)

    def build_Q_matrix(self, use_gpu: bool = False):
        Q = self.base_problem.build_Q_matrix(use_gpu=False)
        Q = np.asarray(Q)
        k = self.A
        x = np.array(self.prefix, dtype=self.dtype)
        self.prefix_E = (x @ Q[:k, :k] @ x.T).item()
        diag = x @ (Q[:k, k:] + Q[k:, :k].T)
        out = Q[k:, k:] + np.diag(diag)
        assert out.dtype == self.dtype
        return _to_device(out, use_gpu)

    @staticmethod
    def init_random_instance(*args, **kwargs):
        raise NotImplementedError("It's a user-defined matrix, for random instance better use RandomQUBO class")
