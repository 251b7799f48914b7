"""Generate the golden fixtures in tests/golden/ by running the reference itself.

Run in a container that holds the reference source (cloud-ru-tech/evo-quantum-qubolib),
with QUBO_REFERENCE_ROOT naming its checkout (the directory holding src/ and
showcase.ipynb):

    QUBO_REFERENCE_ROOT=<checkout> python tests/golden/make_golden.py           # all fixtures
    QUBO_REFERENCE_ROOT=<checkout> python tests/golden/make_golden.py metrics   # metrics.json
    QUBO_REFERENCE_ROOT=<checkout> python tests/golden/make_golden.py schema    # solution_schema.json

The reference is imported from <checkout>/src with the test-only stubs in
tests/golden/refstub (jsonpickle and ortools are not installed; neither is on the search
arithmetic).  Each fixture records the inputs (Q as integers or float bit-exact decimal
strings), the kwargs, and what the reference returned.  Nothing here is needed at test
time: the tests read the JSON files only.
"""
from __future__ import annotations

import json
import os
import re
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
REF_ROOT = os.environ.get("QUBO_REFERENCE_ROOT", "")
if not REF_ROOT or not os.path.isdir(os.path.join(REF_ROOT, "src", "qubo_lib")):
    sys.exit("set QUBO_REFERENCE_ROOT to the reference checkout (the directory holding src/qubo_lib)")
REF_SRC = os.path.join(REF_ROOT, "src")
STUB = os.path.join(HERE, "refstub")

if os.environ.get("_QB_GOLDEN_CHILD") != "1":
    env = dict(os.environ)
    env["PYTHONPATH"] = os.pathsep.join([STUB, REF_SRC] + ([env["PYTHONPATH"]] if env.get("PYTHONPATH") else []))
    env["_QB_GOLDEN_CHILD"] = "1"
    os.execve(sys.executable, [sys.executable] + sys.argv, env)

import numpy as np  # noqa: E402
from qubo_lib.problems import Just_Q, RandomQUBO, ReducedProblem, TSP, MaxCut  # noqa: E402
from qubo_lib.solvers import QBF, Parallel  # noqa: E402
from qubo_lib.state_vectors import StateVectors  # noqa: E402
from qubo_lib.abc import ProblemABC  # noqa: E402


def enc_q(Q: np.ndarray) -> dict:
    Q = np.asarray(Q)
    if np.issubdtype(Q.dtype, np.integer):
        data = Q.astype(np.int64).tolist()
    else:
        data = [[float.hex(float(v)) for v in row] for row in Q]
    return {"dtype": Q.dtype.name, "n": int(Q.shape[0]), "data": data}


def bits(x) -> str:
    return "".join(str(int(b)) for b in x)


def sol_record(sol, kwargs: dict, wall: float) -> dict:
    rec = {
        "kwargs": kwargs,
        "best_E": float(sol.best_E),
        "best_X": bits(sol.best_X),
        "epochs_cnt": int(sol.epochs_cnt),
        "samples_cnt": int(sol.samples_cnt),
        "solver_class": sol.solver_class,
        "wall_s": round(wall, 3),
    }
    if sol.state_vectors is not None:
        rec["packed"] = sol.state_vectors.bitwise_vectors.astype(int).tolist()
    if getattr(sol, "ising_offset", None) is not None:
        rec["ising_offset"] = float(sol.ising_offset)
    if hasattr(sol, "prefix_E"):
        rec["prefix_E"] = float(sol.prefix_E)
    return rec


def run_qbf(Q, **kw):
    t = time.time()
    sol = QBF().solve(Just_Q(Q), **kw)
    return sol_record(sol, kw, time.time() - t)


def run_parallel(Q, splits, ncpu, **kw):
    t = time.time()
    sol = Parallel(base_solver=QBF, splits_cnt=splits, devices=["cpu"] * ncpu).solve(Just_Q(Q), **kw)
    rec = sol_record(sol, kw, time.time() - t)
    rec["splits_cnt"] = splits
    rec["devices"] = ncpu
    return rec


def brute_minimisers(Q) -> tuple[float, int]:
    """Minimum energy and number of minimisers (integer Q, small n) -- tie evidence."""
    n = Q.shape[0]
    X = ((np.arange(1 << n)[:, None] >> np.arange(n - 1, -1, -1)) & 1).astype(np.float64)
    E = np.einsum("ij,jk,ik->i", X, Q.astype(np.float64), X)
    m = E.min()
    return float(m), int((E == m).sum())


def tsp_int_q(n_cities: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    w = rng.integers(1, 101, (n_cities, n_cities))
    w = np.triu(w, 1)
    w = w + w.T
    return TSP.qubo_from_distances(w.astype(np.float64)).astype(np.int32)


def small_cases() -> list:
    rng = np.random.default_rng(2024)
    cases = []
    for n in (1, 2, 3, 5, 8, 11, 14, 17, 20, 22):
        for dt in (np.int8, np.int16, np.int32, np.int64):
            hi = 10 if dt == np.int8 else 100
            U = rng.integers(-hi, hi + 1, (n, n)).astype(dt)
            sym = (np.triu(U) + np.triu(U, 1).T).astype(dt)
            cases.append((f"sym_{np.dtype(dt).name}_n{n}", sym, {}))
            cases.append((f"asym_{np.dtype(dt).name}_n{n}", U, {}))
            cases.append((f"triu_{np.dtype(dt).name}_n{n}", np.triu(U).astype(dt), {}))
        F = rng.standard_normal((n, n)).astype(np.float32)
        cases.append((f"f32_n{n}", F, {}))
        cases.append((f"f32sym_n{n}", ((F + F.T) / 2).astype(np.float32), {}))
        cases.append((f"f64_n{n}", rng.standard_normal((n, n)), {}))
    # explicit splits (the tie rule depends on A)
    for n in (12, 16, 21):
        U = rng.integers(-5, 6, (n, n)).astype(np.int32)
        Q = np.triu(U) + np.triu(U, 1).T
        for A in (0, 1, 3, n // 2, n - 1, n):
            cases.append((f"splitA{A}_n{n}", Q, {"A": A}))
        cases.append((f"splitB7_n{n}", Q, {"B": 7}))
    # heavy ties: small TSPs (each path ties with its reverse), max-cut (x ties with ~x)
    for nc, seed in ((3, 0), (3, 1), (4, 0), (4, 5)):
        Q = tsp_int_q(nc, seed)
        for A in (None, 0, 2, 5, 9):
            if A is not None and A > Q.shape[0]:
                continue
            cases.append((f"tsp{nc}_s{seed}_A{A}", Q, {} if A is None else {"A": A}))
    for n in (6, 10, 13, 18):
        m = rng.random((n, n)) < 0.5
        w = rng.integers(0, 2, (n, n)) * 2 - 1
        Q = np.zeros((n, n), np.int32)
        for i in range(n):
            for j in range(i + 1, n):
                if m[i, j]:
                    Q[i, i] -= w[i, j]; Q[j, j] -= w[i, j]; Q[i, j] += 2 * w[i, j]
        cases.append((f"maxcut_n{n}", Q, {}))
        cases.append((f"maxcut_n{n}_A4", Q, {"A": min(4, n)}))
    # degenerate inputs
    cases.append(("zeros_n9", np.zeros((9, 9), np.int16), {}))
    cases.append(("positive_n9", np.abs(rng.integers(1, 5, (9, 9))).astype(np.int32), {}))
    cases.append(("all_equal_neg_diag_n7", -np.eye(7, dtype=np.int32), {}))
    cases.append(("single_neg_n1", np.array([[-3]], np.int32), {}))
    return cases


def metrics_fixture():
    """energy_arr (use_metrics='all') of QBF and of Parallel(QBF) with one worker, which
    visits the tasks in task order."""
    rng = np.random.default_rng(515)
    recs = []
    for name, A in (("i32sym_n12_A4", 4), ("i16asym_n14_A5", 5), ("f32_n12_A3", 3), ("f64_n10_A4", 4),
                    ("i32sym_n9_A4", 4)):
        n = int(name.split("_n")[1].split("_")[0])
        if name.startswith("i32sym"):
            U = rng.integers(-30, 31, (n, n)).astype(np.int32)
            Q = np.triu(U) + np.triu(U, 1).T
        elif name.startswith("i16"):
            Q = rng.integers(-30, 31, (n, n)).astype(np.int16)
        elif name.startswith("f32"):
            Q = rng.standard_normal((n, n)).astype(np.float32)
        else:
            Q = rng.standard_normal((n, n))
        sol = QBF().solve(Just_Q(Q), A=A, use_metrics="all")
        recs.append({"name": name, "solver": "QBF", "Q": enc_q(Q), "A": A, "best_E": float(sol.best_E),
                     "energy_arr": [float(v) for v in sol.metrics[0]["energy_arr"]],
                     "time_arr_len": int(len(sol.metrics[0]["time_arr"]))})
    for name, n, splits, A in (("par_i32_n12_k4_A3", 12, 4, 3), ("par_i32_n11_k2_A0", 11, 2, 0)):
        U = rng.integers(-30, 31, (n, n)).astype(np.int32)
        Q = np.triu(U) + np.triu(U, 1).T
        sol = Parallel(base_solver=QBF, splits_cnt=splits, devices=["cpu"]).solve(Just_Q(Q), A=A, use_metrics="all")
        recs.append({"name": name, "solver": "Parallel", "splits_cnt": splits, "Q": enc_q(Q), "A": A,
                     "best_E": float(sol.best_E), "energy_arr": [float(v) for v in sol.metrics[0]["energy_arr"]]})
    json.dump({"source": "reference QBF / Parallel(QBF, devices=['cpu']) with use_metrics='all'", "cases": recs},
              open(os.path.join(HERE, "metrics.json"), "w"))
    print("metrics", len(recs))


def _field_types(obj) -> dict:
    return {k: type(v).__name__ for k, v in sorted(vars(obj).items())}


def schema_fixture():
    """The attribute set (and value types) of the Solution objects the reference returns,
    which is what Solution.to_json serialises (jsonpickle writes an object's __dict__ under a
    py/object tag, src/qubo_lib/solution.py:64-69): QBF with and without use_metrics, a
    reduced problem (prefix_E), and Parallel(QBF) with its worker_logs."""
    rng = np.random.default_rng(77)
    U = rng.integers(-30, 31, (12, 12)).astype(np.int32)
    Q = np.triu(U) + np.triu(U, 1).T
    out = {}
    sol = QBF().solve(Just_Q(Q), A=3)
    out["qbf"] = {"fields": _field_types(sol), "metrics": [sorted(m) for m in sol.metrics],
                  "timer_labels": sorted({lbl for _, lbl in sol.timer})}
    sol = QBF().solve(Just_Q(Q), A=3, use_metrics="all")
    out["qbf_metrics"] = {"fields": _field_types(sol),
                          "metrics": {k: [type(v).__name__, str(v.dtype), list(v.shape)]
                                      for k, v in sorted(sol.metrics[0].items())}}
    sol = QBF().solve(ReducedProblem(Just_Q(Q), np.array([1, 0])), A=2)
    out["qbf_reduced"] = {"fields": _field_types(sol)}
    sol = Parallel(base_solver=QBF, splits_cnt=4, devices=["cpu"] * 2).solve(Just_Q(Q), A=2, use_metrics="all")
    out["parallel"] = {"fields": _field_types(sol),
                       "worker_log_fields": sorted(sol.worker_logs[0]),
                       "worker_logs": len(sol.worker_logs),
                       "metrics": {k: [type(v).__name__, str(v.dtype), list(v.shape)]
                                   for k, v in sorted(sol.metrics[0].items())}}
    json.dump({"source": "attribute sets of the reference's Solution objects (QBF, Parallel(QBF) on CPU)",
               "cases": out}, open(os.path.join(HERE, "solution_schema.json"), "w"), indent=1)
    print("schema", sorted(out))


def main():
    if sys.argv[1:] == ["metrics"]:
        metrics_fixture()
        return
    if sys.argv[1:] == ["schema"]:
        schema_fixture()
        return
    out = {}
    # ------------------------------------------------------------------ QBF small
    recs = []
    for name, Q, kw in small_cases():
        try:
            rec = run_qbf(Q, **kw)
        except Exception as e:  # the reference rejects some splits (e.g. B == 0)
            rec = {"kwargs": kw, "error": f"{type(e).__name__}: {e}"}
        rec["name"] = name
        rec["Q"] = enc_q(Q)
        if np.issubdtype(Q.dtype, np.integer) and Q.shape[0] <= 22:
            rec["brute_min"], rec["n_minimisers"] = brute_minimisers(Q)
        recs.append(rec)
    json.dump({"source": "reference QBF().solve(Just_Q(Q), **kwargs) on CPU", "cases": recs},
              open(os.path.join(HERE, "qbf_small.json"), "w"))
    print("qbf_small", len(recs))

    # ------------------------------------------------------------------ Parallel small
    rng = np.random.default_rng(77)
    recs = []
    for n, splits, ncpu in ((10, 2, 2), (12, 4, 2), (16, 8, 3), (20, 2, 2), (23, 4, 4)):
        U = rng.integers(-50, 51, (n, n)).astype(np.int32)
        Q = np.triu(U) + np.triu(U, 1).T
        rec = run_parallel(Q, splits, ncpu)
        rec["name"] = f"par_sym_n{n}_k{splits}"
        rec["Q"] = enc_q(Q)
        rec["brute_min"], rec["n_minimisers"] = brute_minimisers(Q)
        recs.append(rec)
        F = rng.standard_normal((n, n)).astype(np.float32)
        rec = run_parallel(F, splits, ncpu)
        rec["name"] = f"par_f32_n{n}_k{splits}"
        rec["Q"] = enc_q(F)
        recs.append(rec)
    Q = rng.integers(-20, 21, (14, 14)).astype(np.int16)
    rec = run_parallel(Q, 4, 2, A=3)
    rec["name"] = "par_asym_i16_n14_k4_A3"
    rec["Q"] = enc_q(Q)
    rec["brute_min"], rec["n_minimisers"] = brute_minimisers(Q)
    recs.append(rec)
    json.dump({"source": "reference Parallel(QBF, splits_cnt, ['cpu']*k).solve(Just_Q(Q), **kwargs)",
               "cases": recs}, open(os.path.join(HERE, "parallel_small.json"), "w"))
    print("parallel_small", len(recs))

    # ------------------------------------------------------------------ generators & host types
    gen = {"random_qubo": [], "tsp": [], "reduced": [], "state_vectors": [], "chunk": [], "ising": []}
    for seed, n, dt, lo, hi in ((0, 5, "float32", -100, 100), (3, 7, "int16", -100, 100),
                                (42, 6, "int32", -5, 9), (0, 4, "float64", -1, 1),
                                (0, 32, "int16", -100, 101), (0, 20, "float32", -1, 1), (7, 5, "int8", -3, 3)):
        p = RandomQUBO.init_random_instance(seed=seed, N=n, low=lo, high=hi, dtype=np.dtype(dt).type)
        gen["random_qubo"].append({"seed": seed, "N": n, "dtype": dt, "low": lo, "high": hi,
                                   "Q": enc_q(p.build_Q_matrix())})
    for nc, seed in ((3, 1), (4, 42), (5, 42), (6, 42)):
        p = TSP.init_random_instance(n_cities=nc, seed=seed)
        gen["tsp"].append({"kind": "random_instance", "n_cities": nc, "seed": seed, "Q": enc_q(p.build_Q_matrix()),
                           "cities": [[float.hex(float(v)) for v in c] for c in p.cities]})
    for nc, seed in ((3, 0), (5, 1), (6, 0)):
        gen["tsp"].append({"kind": "int_distances", "n_cities": nc, "seed": seed, "Q": enc_q(tsp_int_q(nc, seed))})
    for n, k, dt in ((8, 2, np.int32), (10, 3, np.float32), (12, 1, np.int16)):
        base = np.random.default_rng(n).integers(-9, 10, (n, n)).astype(dt)
        for task in range(1 << k):
            prefix = np.array([(task >> (k - 1 - i)) & 1 for i in range(k)])
            rp = ReducedProblem(Just_Q(base), prefix)
            Qr = rp.build_Q_matrix()
            gen["reduced"].append({"Q": enc_q(base), "k": k, "task": task, "prefix_E": float(rp.prefix_E),
                                   "Qr": enc_q(Qr)})
    for rows in ([[1, 0, 1]], [[0] * 8 + [1]], [[1] * 17], [[0, 1, 1, 0, 1, 0, 0, 1, 1, 1], [1] * 10]):
        sv = StateVectors(np.array(rows))
        gen["state_vectors"].append({"wide": rows, "packed": sv.bitwise_vectors.astype(int).tolist()})
    for N in (3, 10, 20, 21, 30, 36, 44):
        for kw in ({}, {"A": 5}, {"B": 4}, {"use_mem_GB": 1.0, "size_of": 4}, {"use_mem_GB": 135.0, "size_of": 4},
                   {"use_mem_GB": 0.001, "size_of": 2}):
            if ("A" in kw and kw["A"] > N) or ("B" in kw and kw["B"] > N):
                continue
            gen["chunk"].append({"N": N, "kwargs": kw, "AB": list(QBF.define_chunk_size(N=N, **kw))})
    for Q in (np.arange(16).reshape(4, 4).astype(np.int32), np.random.default_rng(1).standard_normal((5, 5))):
        gen["ising"].append({"Q": enc_q(Q), "offset": float(ProblemABC.get_Q_Ising_offset(np, Q))})
    json.dump(gen, open(os.path.join(HERE, "generators.json"), "w"))
    print("generators done")

    # ------------------------------------------------------------------ notebook goldens
    nb = json.load(open(os.path.join(REF_ROOT, "showcase.ipynb")))
    nbrec = []
    for c in nb["cells"]:
        if c["cell_type"] != "code":
            continue
        src = "".join(c["source"])
        txt = "".join("".join(o.get("text", "")) for o in c.get("outputs", []))
        mE = re.search(r"best_E=(-?[0-9.]+)", txt)
        mX = re.search(r"best_X='([01]+)'", txt)
        mN = re.search(r"N=(\d+)", txt)
        mC = re.search(r"solver_class='(\w+)'", txt)
        if mE and mX and mC and mC.group(1) in ("QBF", "QB_F1"):
            nbrec.append({"source_code": src, "N": int(mN.group(1)), "best_E_printed": mE.group(1),
                          "best_X": mX.group(1), "solver_class": mC.group(1)})
    # re-run what is cheap on this CPU: TSP-5 seed 42 with the reference QBF
    p = TSP.init_random_instance(n_cities=5, seed=42)
    t = time.time()
    sol = QBF().solve(p)
    nb_rerun = {"tsp5_seed42": sol_record(sol, {}, time.time() - t)}
    nb_rerun["tsp5_seed42"]["Q"] = enc_q(p.build_Q_matrix())
    p6 = TSP.init_random_instance(n_cities=6, seed=42)
    nb_rerun["tsp6_seed42_Q"] = enc_q(p6.build_Q_matrix())
    r37 = RandomQUBO.init_random_instance(seed=42, N=37)
    nb_rerun["rq37_seed42_Q"] = enc_q(r37.build_Q_matrix())
    r44 = RandomQUBO.init_random_instance(N=44, seed=42, dtype=np.int16)
    nb_rerun["rq44_i16_seed42_Q"] = enc_q(r44.build_Q_matrix())
    t = time.time()
    sol = Parallel(base_solver=QBF, splits_cnt=8, devices=["cpu"] * 8).solve(p6)
    nb_rerun["tsp6_seed42_parallel8cpu"] = sol_record(sol, {}, time.time() - t)
    json.dump({"notebook": nbrec, "rerun_here": nb_rerun},
              open(os.path.join(HERE, "notebook.json"), "w"))
    print("notebook done")

    # ------------------------------------------------------------------ MaxCut 'test' known answer
    mc = MaxCut("test")
    sol = QBF().solve(mc)
    json.dump({"instance": "test", "N": mc.N, "ground_E": float(mc.ground_E), "qbf_best_E": float(sol.best_E),
               "note": "graph loaded at run time from the reference's MaxCut.zip; not stored here"},
              open(os.path.join(HERE, "maxcut_test.json"), "w"))

    # ------------------------------------------------------------------ benchmark configs
    cfg = {}
    q0 = RandomQUBO.init_random_instance(seed=0, N=20, low=-1, high=1, dtype=np.float32).build_Q_matrix()
    Q1 = ((q0 + q0.T) / 2).astype(np.float32)
    cfg["cfg1"] = {"Q": enc_q(Q1), "ref": run_qbf(Q1)}
    U = RandomQUBO.init_random_instance(seed=0, N=32, low=-100, high=101, dtype=np.int16).build_Q_matrix()
    Q2 = (np.triu(U) + np.triu(U, 1).T).astype(np.int16)
    cfg["cfg2"] = {"Q": enc_q(Q2), "ref": run_qbf(Q2, A=12)}
    Q3 = tsp_int_q(6, 0)
    cfg["cfg3"] = {"Q": enc_q(Q3), "ref": run_parallel(Q3, 16, 8)}
    n = 40
    rng = np.random.default_rng(0)
    m = rng.random((n, n)) < 0.5
    w = rng.integers(0, 2, (n, n)) * 2 - 1
    Q4 = np.zeros((n, n), np.int32)
    for i in range(n):
        for j in range(i + 1, n):
            if m[i, j]:
                Q4[i, i] -= w[i, j]; Q4[j, j] -= w[i, j]; Q4[i, j] += 2 * w[i, j]
    t = time.time()
    rp = ReducedProblem(Just_Q(Q4), np.zeros(10, dtype=np.int64))
    sol = QBF().solve(rp)
    cfg["cfg4"] = {"Q": enc_q(Q4), "slice_prefix_bits": [0] * 10,
                   "ref_slice": sol_record(sol, {}, time.time() - t)}
    batch = []
    for i in range(12):
        r = np.random.default_rng(1000 + i)
        nn = int(r.integers(16, 29))
        if nn > 24:
            continue
        G = r.standard_normal((nn, nn))
        Q5 = ((G + G.T) / 2).astype(np.float32)
        batch.append({"index": i, "seed": 1000 + i, "Q": enc_q(Q5), "ref": run_qbf(Q5)})
    cfg["cfg5_subset"] = batch
    json.dump(cfg, open(os.path.join(HERE, "configs.json"), "w"))
    print("configs done")
    metrics_fixture()


if __name__ == "__main__":
    main()
