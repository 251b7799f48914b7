"""Host-side logic on the CPU against the reference's own outputs (tests/golden/
generators.json): problem generators, ReducedProblem, state-vector packing, the (A, B)
split rule, the Ising offset, Solution JSON round trips, error behaviour at the boundary,
and the C ABI library's exported symbols (loaded, not called: no GPU here)."""
import ctypes
import os
import re

import numpy as np
import pytest

import qubo_b200  # noqa: F401
from conftest import dec_q, load_golden
from qubo_b200 import _lib
from qubo_b200.abc import ProblemABC
from qubo_b200.problems import Just_Q, MaxCut, RandomQUBO, ReducedProblem, TSP
from qubo_b200.solution import Solution
from qubo_b200.solvers import QB_F1, QBF, Parallel
from qubo_b200.state_vectors import StateVectors

GEN = load_golden("generators.json")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("rec", GEN["random_qubo"], ids=lambda r: f"s{r['seed']}_n{r['N']}_{r['dtype']}")
def test_random_qubo_matches_reference(rec):
    p = RandomQUBO.init_random_instance(seed=rec["seed"], N=rec["N"], low=rec["low"], high=rec["high"],
                                        dtype=np.dtype(rec["dtype"]).type)
    Q = p.build_Q_matrix()
    ref = dec_q(rec["Q"])
    assert Q.dtype == ref.dtype
    np.testing.assert_array_equal(Q, ref)


@pytest.mark.parametrize("rec", GEN["tsp"], ids=lambda r: f"{r['kind']}_{r['n_cities']}_{r['seed']}")
def test_tsp_matches_reference(rec):
    ref = dec_q(rec["Q"])
    if rec["kind"] == "random_instance":
        p = TSP.init_random_instance(n_cities=rec["n_cities"], seed=rec["seed"])
        cities = np.array([[float.fromhex(v) for v in c] for c in rec["cities"]])
        np.testing.assert_array_equal(p.cities.astype(np.float64), cities)
        Q = p.build_Q_matrix()
    else:
        rng = np.random.default_rng(rec["seed"])
        w = rng.integers(1, 101, (rec["n_cities"], rec["n_cities"]))
        w = np.triu(w, 1)
        w = w + w.T
        Q = TSP.qubo_from_distances(w.astype(np.float64)).astype(np.int32)
    assert Q.dtype == ref.dtype
    np.testing.assert_array_equal(Q, ref)


@pytest.mark.parametrize("rec", GEN["reduced"], ids=lambda r: f"n{r['Q']['n']}_k{r['k']}_t{r['task']}")
def test_reduced_problem_matches_reference(rec):
    Q = dec_q(rec["Q"])
    k, task = rec["k"], rec["task"]
    prefix = np.array([(task >> (k - 1 - i)) & 1 for i in range(k)])
    rp = ReducedProblem(Just_Q(Q), prefix)
    Qr = rp.build_Q_matrix()
    ref = dec_q(rec["Qr"])
    assert Qr.dtype == ref.dtype
    np.testing.assert_array_equal(Qr, ref)
    assert float(rp.prefix_E) == rec["prefix_E"]


@pytest.mark.parametrize("rec", GEN["state_vectors"], ids=lambda r: f"rows{len(r['wide'])}x{len(r['wide'][0])}")
def test_state_vector_packing_matches_reference(rec):
    sv = StateVectors(np.array(rec["wide"]))
    np.testing.assert_array_equal(sv.bitwise_vectors.astype(int), np.array(rec["packed"]))
    np.testing.assert_array_equal(sv.get_wide_vectors(), np.array(rec["wide"]))


@pytest.mark.parametrize("rec", GEN["chunk"], ids=lambda r: f"N{r['N']}_{sorted(r['kwargs'].items())}")
def test_define_chunk_size_matches_reference(rec):
    assert list(QBF.define_chunk_size(N=rec["N"], **rec["kwargs"])) == rec["AB"]


@pytest.mark.parametrize("rec", GEN["ising"], ids=lambda r: f"n{r['Q']['n']}")
def test_ising_offset_matches_reference(rec):
    assert float(ProblemABC.get_Q_Ising_offset(np, dec_q(rec["Q"]))) == pytest.approx(rec["offset"], rel=1e-12)


def test_maxcut_rule_and_cut_value():
    mc = MaxCut(4, [(0, 1, 1), (1, 2, 1), (2, 3, 1), (0, 3, 1)])
    Q = mc.build_Q_matrix()
    x = np.array([1, 0, 1, 0])
    assert int(x @ Q @ x) == -mc.cut_value(x) == -4


def test_solution_json_round_trip():
    sol = Solution(5, 4, 1, Just_Q(np.eye(5, dtype=np.int32)).to_json(), "{}")
    sol.best_E = np.float64(-3.5)
    sol.best_X = np.array([1, 0, 1, 1, 0], dtype=np.int32)
    sol.energies = np.array([-3.5])
    sol.state_vectors = StateVectors(sol.best_X.reshape(1, -1))
    sol.metrics = [{"energy_arr": np.array([-1.0, -3.5])}]
    back = Solution.init_from_json(sol.to_json())
    assert float(back.best_E) == -3.5
    np.testing.assert_array_equal(np.asarray(back.best_X), sol.best_X)
    np.testing.assert_array_equal(np.asarray(back.metrics[0]["energy_arr"]), [-1.0, -3.5])
    assert back.N == 5 and back.epochs_cnt == 4


def test_solution_json_encoded_on_worker_thread():
    """The Solution's JSON fields, encoded on a worker thread during the device search, equal
    the direct encodings; a forked child gets a pool of its own."""
    from qubo_b200 import _json, solvers
    prob = Just_Q(np.arange(25, dtype=np.int32).reshape(5, 5))
    kw = {"device": "cuda:0", "form": "tc", "use_metrics": ["energy_arr"]}
    pj, ks, off = solvers._encode_async(prob, kw).result(timeout=30)
    assert pj == prob.to_json() and ks == _json.encode(kw, indent=4) and off is None
    Q = prob.build_Q_matrix()
    assert solvers._encode_async(prob, kw, Q).result(timeout=30)[2] == prob.get_Q_Ising_offset(np, Q)
    import warnings
    with warnings.catch_warnings():  # forking a threaded process is the case under test
        warnings.simplefilter("ignore", DeprecationWarning)
        pid = os.fork()
    if pid == 0:  # child: no thread behind the inherited pool object
        try:
            ok = solvers._encode_async(prob, kw).result(timeout=10)[0] == pj
        except BaseException:  # noqa: BLE001
            ok = False
        os._exit(0 if ok else 1)
    _, status = os.waitpid(pid, 0)
    assert os.WIFEXITED(status) and os.WEXITSTATUS(status) == 0


def test_boundary_errors_without_gpu():
    with pytest.raises(ValueError):
        QBF().solve(Just_Q(np.eye(4, dtype=np.int32)), device="cpu")
    with pytest.raises(ValueError):
        QB_F1().solve(Just_Q(np.eye(20, dtype=np.int16)), device="cpu")
    with pytest.raises(ValueError):
        Parallel(base_solver=QBF, splits_cnt=3, devices=["cuda"])
    with pytest.raises(ValueError):
        Parallel(base_solver=QBF, splits_cnt=4, devices=["cpu", "cuda"])


def _declared_functions():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names += re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(qb_[a-z_0-9]+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_c_abi_exports_every_declared_symbol():
    names = _declared_functions()
    assert {"qb_solve", "qb_solve_begin", "qb_solve_finish", "qb_solve_noalloc", "qb_prefix_minima"} <= set(names)
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_c_abi_host_only_calls():
    L = _lib.load()
    assert L.qb_version() >= 100
    for s in range(9):
        assert L.qb_strerror(s)
    assert b"no-allocation" in L.qb_strerror(8)


def test_batch_descriptors():
    """qb_solve_batch's problem descriptors built on the host: sizes, dtype codes and the
    data address of each matrix (a contiguous copy for a non-contiguous input)."""
    rng = np.random.default_rng(3)
    ro = rng.normal(size=(21, 21))
    ro.flags.writeable = False
    Qs = [rng.normal(size=(20, 20)).astype(np.float32), ro,
          rng.integers(-9, 9, size=(24, 24)).astype(np.int16).T,  # non-contiguous
          np.zeros((0, 0), dtype=np.int32), rng.integers(-9, 9, size=(1, 1)).astype(np.int64)]
    probs, ns, keep = _lib.Handle._batch_problems(Qs)
    assert list(ns) == [20, 21, 24, 0, 1]
    for i, (p, Q) in enumerate(zip(probs, keep)):
        assert Q.flags.c_contiguous
        assert p.n == p.ldq == Q.shape[0]
        assert p.dtype == _lib._DTYPES[Q.dtype]
        assert (p.q or 0) == Q.__array_interface__["data"][0], i
        np.testing.assert_array_equal(Q, Qs[i])
    assert keep[0] is Qs[0] and keep[1] is Qs[1] and keep[2] is not Qs[2]
    assert len(_lib.Handle._batch_problems([])[0]) == 0
    with pytest.raises(ValueError):
        _lib.Handle._batch_problems([np.zeros((2, 3))])
    with pytest.raises(TypeError):
        _lib.Handle._batch_problems([np.zeros((2, 2), dtype=np.uint8)])


def test_config_generators_match_reference_inputs():
    from qubo_b200 import configs
    cfg = load_golden("configs.json")
    np.testing.assert_array_equal(configs.random_f32_n20(), dec_q(cfg["cfg1"]["Q"]))
    np.testing.assert_array_equal(configs.random_i16_n32(), dec_q(cfg["cfg2"]["Q"]))
    np.testing.assert_array_equal(configs.tsp6_int(), dec_q(cfg["cfg3"]["Q"]))
    np.testing.assert_array_equal(configs.maxcut_er(), dec_q(cfg["cfg4"]["Q"]))
    for b in cfg["cfg5_subset"]:
        np.testing.assert_array_equal(configs.batch_instance(b["index"], seed=1000), dec_q(b["Q"]))


def test_gray_group_identities():
    """The Gray-form and QB_F1 int16 kernels walk Gray steps in aligned groups of 32
    with constants in place of a per-step bit scan.  The identities they rely on: for ig a
    multiple of 32 and 0 <= l < 32, gray(ig + l) = gray(ig) ^ gray(l); step l > 0 flips bit
    ctz(l), which turns on unless bit ctz(l) + 1 of the step index is set (bit 5 of ig when
    ctz(l) = 4); and ctz5 in csrc/qb_common.cuh is ctz on 1..31."""
    def gray(i):
        return i ^ (i >> 1)

    def ctz5(l):  # restated from csrc/qb_common.cuh
        return 0 if l & 1 else 1 if l & 2 else 2 if l & 4 else 3 if l & 8 else 4

    rng = np.random.default_rng(3)
    for ig in [0, 32, 96, 4096] + [int(v) * 32 for v in rng.integers(0, 1 << 30, 200)]:
        for l in range(32):
            assert gray(ig + l) == gray(ig) ^ gray(l)
            if l:
                kb = ctz5(l)
                assert kb == (l & -l).bit_length() - 1
                turns_on = bool((gray(ig + l) >> kb) & 1)
                predicted = not ((l >> (kb + 1)) & 1) if kb < 4 else not ((ig >> 5) & 1)
                assert turns_on == predicted
