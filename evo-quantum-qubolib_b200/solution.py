"""Result record returned by every solver (src/qubo_lib/solution.py:3-85).

Same fields as the reference: N, epochs_cnt, samples_cnt, problem_instance_json,
solver_params_json, metrics, state_vectors, energies, ising_offset, solver_class, best_E,
best_X, error, time_to_solve_ms; solvers add prefix_E (reduced problems), timer and
worker_logs (Parallel) as the reference does.  This build also attaches ``search`` -- a dict
describing how the answer was obtained on the GPU (form, split, states, candidate records,
FP64 error of a float result).
"""
from __future__ import annotations

from . import _json


class Solution:
    def __init__(self, N: int, epochs_cnt: int, samples_cnt: int, problem_instance_json: str,
                 solver_params_json: str):
        self.N = N
        self.epochs_cnt = epochs_cnt
        self.samples_cnt = samples_cnt
        self.problem_instance_json: str = problem_instance_json
        self.solver_params_json: str = solver_params_json
        self.metrics = []
        self.state_vectors = None
        self.energies = None
        self.ising_offset = None
        self.solver_class = None
        self.best_E = None
        self.best_X = None
        self.error = ""
        self.time_to_solve_ms = None

    def to_json(self):
        return _json.encode(self, indent=4)

    @staticmethod
    def init_from_json(json_str: str) -> "Solution":
        return _json.decode(json_str)

    def __str__(self):
        if self.error:
            return f"Error: {self.error}"
        best_x_str = "".join(map(str, self.best_X)) if self.best_X is not None else None
        return (
            f"Solution(\n"
            f"  N={self.N},\n"
            f"  best_E={self.best_E:.3f},\n"
            f"  time_to_solve_ms={self.time_to_solve_ms:.1f},\n"
            f"  samples_cnt={self.samples_cnt},\n"
            f"  solver_class='{self.solver_class}',\n"
            f"  best_X='{best_x_str}'\n"
            f")"
        )
