"""use_metrics: the per-prefix energy_arr of QBF and Parallel(QBF) against the reference's
own arrays (tests/golden/metrics.json) -- the oracle restatement on the CPU, the library's
qb_prefix_minima kernel on the GPU."""
import numpy as np
import pytest

import oracle
import qubo_b200  # noqa: F401
from conftest import dec_q, load_golden

CASES = load_golden("metrics.json")["cases"]
QBF_CASES = [c for c in CASES if c["solver"] == "QBF"]
PAR_CASES = [c for c in CASES if c["solver"] == "Parallel"]


def _close(got, ref, Q):
    got, ref = np.asarray(got, dtype=np.float64), np.asarray(ref, dtype=np.float64)
    assert got.shape == ref.shape
    if np.issubdtype(Q.dtype, np.integer):
        np.testing.assert_array_equal(got, ref)
    else:
        # the reference accumulates float32 suffix energies; these values are FP64 sums
        np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("case", QBF_CASES, ids=[c["name"] for c in QBF_CASES])
def test_oracle_prefix_minima_matches_reference(case):
    Q = dec_q(case["Q"])
    _close(oracle.prefix_minima_numpy(Q, case["A"]), case["energy_arr"], Q)


@pytest.mark.parametrize("case", PAR_CASES, ids=[c["name"] for c in PAR_CASES])
def test_oracle_parallel_energy_arr_matches_reference(case):
    Q = dec_q(case["Q"])
    k = case["splits_cnt"].bit_length() - 1
    _close(oracle.parallel_energy_arr_numpy(Q, k, case["A"]), case["energy_arr"], Q)


@pytest.mark.gpu
@pytest.mark.parametrize("case", QBF_CASES, ids=[c["name"] for c in QBF_CASES])
def test_qbf_energy_arr(cuda_ok, case):
    from qubo_b200.problems import Just_Q
    from qubo_b200.solvers import QBF
    Q = dec_q(case["Q"])
    sol = QBF().solve(Just_Q(Q), device="cuda", A=case["A"], use_metrics="all")
    _close(sol.metrics[0]["energy_arr"], case["energy_arr"], Q)
    assert float(sol.best_E) == pytest.approx(case["best_E"], rel=1e-6, abs=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("case", PAR_CASES, ids=[c["name"] for c in PAR_CASES])
def test_parallel_energy_arr(cuda_ok, case):
    from qubo_b200.problems import Just_Q
    from qubo_b200.solvers import QBF, Parallel
    Q = dec_q(case["Q"])
    sol = Parallel(base_solver=QBF, splits_cnt=case["splits_cnt"], devices=["cuda"]).solve(
        Just_Q(Q), A=case["A"], use_metrics="all")
    _close(sol.metrics[0]["energy_arr"], case["energy_arr"], Q)


@pytest.mark.gpu
@pytest.mark.parametrize("n,A", [(20, 3), (22, 6), (24, 0)])
def test_prefix_minima_random_against_oracle(cuda_ok, n, A):
    from qubo_b200 import _lib
    rng = np.random.default_rng(n * 100 + A)
    for Q in (rng.integers(-50, 51, (n, n)).astype(np.int32), rng.standard_normal((n, n))):
        got = _lib.handle(0).prefix_minima(Q, prefix_bits=A)
        ref = oracle.prefix_minima_numpy(Q, A)
        if Q.dtype == np.int32:
            np.testing.assert_array_equal(got, ref)
        else:
            np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12)


# ---------------------------------------------------------------------- time_arr and the
# Solution layout (src/qubo_lib/solution.py:46-69; qbf.py:342-365; parallel.py:250-318)

SCHEMA = load_golden("solution_schema.json")["cases"]


def _schema_q():
    """The 12-variable problem the schema fixture was recorded on."""
    rng = np.random.default_rng(77)
    U = rng.integers(-30, 31, (12, 12)).astype(np.int32)
    return np.triu(U) + np.triu(U, 1).T


def _fields(sol) -> dict:
    """Attribute -> type name, without this build's extra ``search`` record."""
    return {k: type(v).__name__ for k, v in sorted(vars(sol).items()) if k != "search"}


def _metric_layout(m: dict) -> dict:
    return {k: [type(v).__name__, str(v.dtype), list(v.shape)] for k, v in sorted(m.items())}


def test_schema_fixture_is_the_reference_layout():
    assert set(SCHEMA) == {"qbf", "qbf_metrics", "qbf_reduced", "parallel"}
    assert SCHEMA["parallel"]["worker_log_fields"] == ["device", "task_id", "time_to_solve_ms", "worker_id"]
    # time_arr: one entry per prefix of the loop (2^A), and per task prefix under Parallel
    assert SCHEMA["qbf_metrics"]["metrics"]["time_arr"] == ["ndarray", "float64", [8]]
    assert SCHEMA["parallel"]["metrics"]["time_arr"] == ["ndarray", "float64", [16]]


def test_solution_json_round_trip_keeps_every_field():
    """to_json writes the object under a py/object tag with one key per attribute, as
    jsonpickle does for a plain object, and init_from_json restores every field."""
    import json
    from qubo_b200.solution import Solution
    from qubo_b200.state_vectors import StateVectors
    s = Solution(4, 8, 1, "{}", "{}")
    s.best_X = np.array([1, 0, 1, 1], np.int32)
    s.best_E = np.float64(-3.5)
    s.energies = np.array([s.best_E])
    s.state_vectors = StateVectors(wide_vector_matrix=s.best_X.reshape(1, -1))
    s.metrics = [{"time_arr": np.full(8, 0.25), "energy_arr": np.arange(8.0)}]
    s.ising_offset = np.float64(1.25)
    s.solver_class = "QBF"
    s.time_to_solve_ms = 2.0
    s.timer = [(1.0, "build_Q"), (1.0, "search")]
    s.prefix_E = 3
    doc = json.loads(s.to_json())
    assert doc["py/object"].endswith(".Solution")
    assert set(doc) - {"py/object"} == set(vars(s))
    back = Solution.init_from_json(s.to_json())
    assert _fields(back) == _fields(s)
    assert np.array_equal(back.best_X, s.best_X) and back.best_E == s.best_E
    np.testing.assert_array_equal(back.metrics[0]["time_arr"], s.metrics[0]["time_arr"])
    np.testing.assert_array_equal(back.state_vectors.bitwise_vectors, s.state_vectors.bitwise_vectors)


@pytest.mark.gpu
def test_solution_fields_match_reference(cuda_ok):
    from qubo_b200.problems import Just_Q, ReducedProblem
    from qubo_b200.solvers import QBF, Parallel
    Q = _schema_q()
    sol = QBF().solve(Just_Q(Q), device="cuda", A=3)
    assert _fields(sol) == SCHEMA["qbf"]["fields"]
    assert [sorted(m) for m in sol.metrics] == SCHEMA["qbf"]["metrics"]
    sol = QBF().solve(Just_Q(Q), device="cuda", A=3, use_metrics="all")
    assert _fields(sol) == SCHEMA["qbf_metrics"]["fields"]
    assert _metric_layout(sol.metrics[0]) == SCHEMA["qbf_metrics"]["metrics"]
    sol = QBF().solve(ReducedProblem(Just_Q(Q), np.array([1, 0])), device="cuda", A=2)
    assert _fields(sol) == SCHEMA["qbf_reduced"]["fields"]
    sol = Parallel(base_solver=QBF, splits_cnt=4, devices=["cuda"]).solve(Just_Q(Q), A=2, use_metrics="all")
    assert _fields(sol) == SCHEMA["parallel"]["fields"]
    assert sorted(sol.worker_logs[0]) == SCHEMA["parallel"]["worker_log_fields"]
    assert len(sol.worker_logs) == SCHEMA["parallel"]["worker_logs"]
    assert _metric_layout(sol.metrics[0]) == SCHEMA["parallel"]["metrics"]
    from qubo_b200.solution import Solution
    back = Solution.init_from_json(sol.to_json())
    assert _fields(back) == _fields(sol)


@pytest.mark.gpu
@pytest.mark.parametrize("case", QBF_CASES, ids=[c["name"] for c in QBF_CASES])
def test_qbf_time_arr_has_one_entry_per_prefix(cuda_ok, case):
    from qubo_b200.problems import Just_Q
    from qubo_b200.solvers import QBF
    Q = dec_q(case["Q"])
    sol = QBF().solve(Just_Q(Q), device="cuda", A=case["A"], use_metrics={"time_arr"})
    t = sol.metrics[0]["time_arr"]
    assert t.shape == (case["time_arr_len"],) and t.dtype == np.float64
    assert (t > 0).all()
    # equal shares of the solve's device time (every prefix covers the same states)
    assert t.sum() == pytest.approx(sol.search["pass1_ms"] + sol.search["pass2_ms"], rel=1e-9)
