"""Time the reference's own CPU QBF against the C restatement (oracle/qbf_port.c) on the
same slice of the benchmark problem, one core each, and check that both give the same answer.

This ties the benchmark's CPU figure (the C restatement on all host cores) to the
reference's own numpy loop (src/qubo_lib/solvers/qbf.py:188-230).  Run it in a container
that holds the reference source, with QUBO_REFERENCE_ROOT naming its checkout (the
directory holding src/qubo_lib):

    QUBO_REFERENCE_ROOT=<checkout> python oracle/time_reference_cpu.py [fixed_bits] [slices]

Workload: the 6-city TSP QUBO with integer distances U{1..100} (seed 0, 36 variables,
int32), its first ``fixed_bits`` variables (default 8) fixed to ``slices`` (default 3)
seeded prefixes; each slice is the reference's ``ReducedProblem`` (36 - fixed_bits
variables) solved by ``QBF().solve`` with its default CPU split, and by the restatement
with the same split.  Prints one JSON line.  Nothing here runs at test or benchmark time.
"""
from __future__ import annotations

import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF_ROOT = os.environ.get("QUBO_REFERENCE_ROOT", "")
if not REF_ROOT or not os.path.isdir(os.path.join(REF_ROOT, "src", "qubo_lib")):
    sys.exit("set QUBO_REFERENCE_ROOT to the reference checkout (the directory holding src/qubo_lib)")
STUB = os.path.join(ROOT, "tests", "golden", "refstub")  # jsonpickle / ortools stand-ins, off the arithmetic

if os.environ.get("_QB_TIMING_CHILD") != "1":
    env = dict(os.environ)
    paths = [STUB, os.path.join(REF_ROOT, "src"), ROOT, HERE]
    env["PYTHONPATH"] = os.pathsep.join(paths + ([env["PYTHONPATH"]] if env.get("PYTHONPATH") else []))
    env["_QB_TIMING_CHILD"] = "1"
    env.setdefault("OMP_NUM_THREADS", "1")
    for var in ("OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        env.setdefault(var, "1")
    os.execve(sys.executable, [sys.executable] + sys.argv, env)

import numpy as np  # noqa: E402
from qubo_lib.problems import Just_Q, ReducedProblem  # noqa: E402
from qubo_lib.solvers import QBF  # noqa: E402

import oracle  # noqa: E402
import qubo_b200  # noqa: E402,F401
from qubo_b200 import configs  # noqa: E402


def main(fixed_bits: int = 8, slices: int = 3) -> dict:
    Q = configs.tsp6_int()
    n = Q.shape[0]
    rng = np.random.default_rng(0)
    rows = []
    for _ in range(slices):
        prefix = rng.integers(0, 2, fixed_bits)
        rp = ReducedProblem(Just_Q(Q), prefix)
        Qr = np.asarray(rp.build_Q_matrix())
        m = Qr.shape[0]
        t0 = time.perf_counter()
        sol = QBF().solve(rp, device="cpu")
        t_ref = time.perf_counter() - t0
        t0 = time.perf_counter()
        port = oracle.qbf_port(Qr, A=m - min(m, 20))
        t_port = time.perf_counter() - t0
        x_ref = int("".join(str(int(b)) for b in np.asarray(sol.best_X)), 2)
        same = x_ref == port["best_X_int"] and int(sol.best_E) == port["best_E"]
        rows.append({"prefix": "".join(map(str, prefix)), "states": 1 << m, "reference_s": t_ref,
                     "port_s": t_port, "same_answer": bool(same)})
    states = sum(r["states"] for r in rows)
    t_ref = sum(r["reference_s"] for r in rows)
    t_port = sum(r["port_s"] for r in rows)
    return {"workload": f"6-city TSP QUBO (36 variables, int32), {slices} slices with the first {fixed_bits} "
                        f"variables fixed ({n - fixed_bits} free, default CPU split)",
            "cores": 1, "reference_states_per_s": states / t_ref, "port_states_per_s": states / t_port,
            "port_over_reference": t_ref / t_port, "all_same_answer": all(r["same_answer"] for r in rows),
            "slices": rows}


if __name__ == "__main__":
    args = [int(a) for a in sys.argv[1:3]]
    print(json.dumps(main(*args)))
