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
