"""GPU parity: every search form against the oracle (which is pinned to the reference) on
seeded inputs, golden fixtures and edge cases.  Integer Q: bit-exact argmin and energy.
Float Q: the FP64 argmin, energy within 1e-9 relative of the oracle's FP64 value."""
import numpy as np
import pytest

import oracle
import qubo_b200  # noqa: F401
from conftest import bits_to_int, dec_q, load_golden
from qubo_b200 import _lib
from qubo_b200.problems import Just_Q, ReducedProblem
from qubo_b200.solvers import QBF, QB_F1, Parallel

pytestmark = pytest.mark.gpu

FLOAT_RTOL = 1e-9


def _x_int(sol) -> int:
    return bits_to_int("".join(map(str, sol.best_X)))


def _forms(n):
    f = ["exact", "auto"]
    if n >= 20:  # the Gray-code and tensor-core forms start at 20 variables
        f += ["gray", "tc"]
    return f


def _check(Q, sol, ref):
    if np.issubdtype(Q.dtype, np.integer):
        assert _x_int(sol) == ref["best_X_int"], (sol.search, ref)
        assert int(sol.best_E) == ref["best_E"]
    else:
        assert _x_int(sol) == ref["best_X_int"], (sol.search, ref)
        e64 = oracle.energy(Q, ref["best_X_int"])
        assert abs(float(sol.best_E) - e64) <= FLOAT_RTOL * max(1.0, abs(e64))


def _solve(Q, form, **kw):
    return QBF().solve(Just_Q(Q), device="cuda", form=form, **kw)


def _rand_cases():
    rng = np.random.default_rng(11)
    out = []
    for n in (1, 2, 3, 7, 12, 16, 19, 20, 21, 24, 26):
        for dt in (np.int8, np.int16, np.int32, np.int64, np.float32, np.float64):
            if np.issubdtype(dt, np.integer):
                hi = 3 if dt == np.int8 else 100
                U = rng.integers(-hi, hi + 1, (n, n)).astype(dt)
                Q = U if n % 2 else (np.triu(U) + np.triu(U, 1).T).astype(dt)
            else:
                Q = rng.standard_normal((n, n)).astype(dt)
            out.append((f"{np.dtype(dt).name}_n{n}", Q))
    return out


RAND = _rand_cases()


@pytest.mark.parametrize("name,Q", RAND, ids=[c[0] for c in RAND])
def test_random_all_forms(cuda_ok, name, Q):
    n = Q.shape[0]
    ref = oracle.qbf_port(Q)
    for form in _forms(n):
        _check(Q, _solve(Q, form), ref)


GOLD = [c for c in load_golden("qbf_small.json")["cases"] if "error" not in c]


@pytest.mark.parametrize("case", GOLD, ids=[c["name"] for c in GOLD])
def test_golden_qbf_cases(cuda_ok, case):
    Q = dec_q(case["Q"])
    n = Q.shape[0]
    kw = case["kwargs"]
    A = kw.get("A", n - kw["B"] if "B" in kw else n - min(n, 20))
    ref = oracle.qbf_port(Q, A=A)
    for form in _forms(n):
        _check(Q, _solve(Q, form, **kw), ref)


@pytest.mark.parametrize("A", [0, 3, 9, 17, 23])
def test_tie_rule_follows_split(cuda_ok, A):
    """Heavily tied problem (every optimum has many twins): the winner depends on A exactly
    as in the reference's prefix loop."""
    n = 24
    rng = np.random.default_rng(5)
    Q = np.zeros((n, n), np.int32)
    for i in range(0, n, 2):  # pairs (i, i+1) with E = -1 when exactly one of them is set
        Q[i, i] = -1
        Q[i + 1, i + 1] = -1
        Q[i, i + 1] = 2
    Q[rng.integers(0, n), rng.integers(0, n)] += 0
    ref = oracle.qbf_port(Q, A=A)
    for form in _forms(n):
        _check(Q, _solve(Q, form, A=A), ref)


def test_zero_and_positive_matrices(cuda_ok):
    for Q in (np.zeros((22, 22), np.int16), np.ones((21, 21), np.int32), np.eye(25, dtype=np.float32)):
        for form in _forms(Q.shape[0]):
            sol = _solve(Q, form)
            assert _x_int(sol) == 0 and float(sol.best_E) == 0.0


PAR = load_golden("parallel_small.json")["cases"]


@pytest.mark.parametrize("case", PAR, ids=[c["name"] for c in PAR])
def test_parallel_single_device(cuda_ok, case):
    Q = dec_q(case["Q"])
    k_splits = case["splits_cnt"]
    kw = {k: v for k, v in case["kwargs"].items()}
    ref = oracle.parallel_port(Q, k_splits, A_sub=kw.get("A", -1))
    sol = Parallel(base_solver=QBF, splits_cnt=k_splits, devices=["cuda"]).solve(Just_Q(Q), **kw)
    _check(Q, sol, ref)
    assert sol.epochs_cnt == k_splits and sol.solver_class == "QBF"
    if np.issubdtype(Q.dtype, np.integer):
        assert float(sol.best_E) == case["best_E"]


@pytest.mark.parametrize("n,seed", [(19, 0), (20, 1), (22, 2), (24, 3)])
def test_qb_f1_order(cuda_ok, n, seed):
    rng = np.random.default_rng(seed)
    U = rng.integers(-3, 4, (n, n)).astype(np.int16)
    Q = (np.triu(U) + np.triu(U, 1).T).astype(np.int16)
    ref = oracle.qbf1_numpy(Q)
    sol = QB_F1().solve(Just_Q(Q), device="cuda")
    assert _x_int(sol) == ref["best_X_int"] and sol.best_E == ref["best_E"]
    assert sol.solver_class == "QB_F1" and sol.epochs_cnt == 1 and isinstance(sol.best_E, int)


def test_solution_json_fields(cuda_ok):
    """QBF and QB_F1 solutions carry the problem's and the kwargs' JSON and the Ising offset
    (computed while the device search runs), equal to the direct computations, and the packed
    state vector of best_X; the solution round-trips."""
    from qubo_b200 import _json
    from qubo_b200.solution import Solution
    rng = np.random.default_rng(12)
    U = rng.integers(-5, 6, (22, 22)).astype(np.int16)
    prob = Just_Q((np.triu(U) + np.triu(U, 1).T).astype(np.int16))
    for solver, kw in ((QBF(), {"device": "cuda", "A": 3}), (QB_F1(), {"device": "cuda"})):
        sol = solver.solve(prob, **kw)
        assert sol.problem_instance_json == prob.to_json()
        assert sol.solver_params_json == _json.encode(kw, indent=4)
        assert sol.ising_offset == prob.get_Q_Ising_offset(np, prob.build_Q_matrix())
        np.testing.assert_array_equal(sol.state_vectors.get_wide_vectors()[0], sol.best_X)
        back = Solution.init_from_json(sol.to_json())
        assert float(back.best_E) == float(sol.best_E)
    for _ in range(20):  # back-to-back solves reuse the worker thread
        assert QBF().solve(prob, device="cuda").problem_instance_json == prob.to_json()


def test_qb_f1_rejects_non_int16(cuda_ok):
    with pytest.raises(TypeError):
        QB_F1().solve(Just_Q(np.zeros((20, 20), np.int32)), device="cuda")


def test_reduced_problem_prefix_energy(cuda_ok):
    rng = np.random.default_rng(9)
    U = rng.integers(-20, 21, (26, 26)).astype(np.int32)
    base = Just_Q(U)
    rp = ReducedProblem(base, np.array([1, 0, 1]))
    sol = QBF().solve(rp, device="cuda")
    Qr = rp.build_Q_matrix()
    ref = oracle.qbf_port(Qr)
    assert _x_int(sol) == ref["best_X_int"]
    assert sol.prefix_E == rp.prefix_E


def test_errors(cuda_ok):
    Q = np.zeros((8, 8), np.int32)
    with pytest.raises(ValueError):
        QBF().solve(Just_Q(Q), device="cpu")
    with pytest.raises(ValueError):
        QBF().solve(Just_Q(Q), use_gpu=True)
    with pytest.raises(ValueError):
        QBF().solve(Just_Q(Q), device="cuda", A=9)
    with pytest.raises(ValueError):
        Parallel(base_solver=QBF, splits_cnt=3, devices=["cuda"])
    with pytest.raises(ValueError):
        Parallel(base_solver=QBF, splits_cnt=2, devices=["cpu", "cuda"])


def test_c_abi_two_phase_matches_single_call(cuda_ok):
    """qb_solve_begin / qb_solve_finish over 3 shards reproduce qb_solve."""
    rng = np.random.default_rng(21)
    U = rng.integers(-50, 51, (27, 27)).astype(np.int32)
    Q = (np.triu(U) + np.triu(U, 1).T).astype(np.int32)
    h = _lib.handle(0)
    for form in ("gray", "exact", "auto"):
        whole = h.solve(Q, form=form)
        mins = []
        for s in range(3):
            mins.append(h.solve_begin(Q, form=form, shard_index=s, shard_count=3))
            h.solve_finish(mins[-1], 27)
        gmin = min(mins)
        outs = []
        for s in range(3):
            h.solve_begin(Q, form=form, shard_index=s, shard_count=3)
            outs.append(h.solve_finish(gmin, 27))
        found = [o for o in outs if o["found"]]
        best = min(found, key=lambda o: (o["best_E"], o["order_key"]))
        assert best["best_X_int"] == whole["best_X_int"] and best["best_E"] == whole["best_E"]
        assert sum(o["states"] for o in outs) == 2 ** 27


@pytest.mark.parametrize("n", [20, 21, 25, 29])
def test_tensor_core_pair_and_one_state_forms(cuda_ok, n):
    """Both tensor-core kernels (default: one state per accumulator; QB_FLAG_TC_PAIR: two)
    against the oracle, integer and float Q, whole problem and three shards."""
    rng = np.random.default_rng(400 + n)
    U = rng.integers(-60, 61, (n, n)).astype(np.int32)
    G = rng.standard_normal((n, n))
    h = _lib.handle(0)
    for Q in (U, (np.triu(U) + np.triu(U, 1).T).astype(np.int32), G, ((G + G.T) / 2).astype(np.float32)):
        ref = oracle.qbf_port(Q)
        for pair in (False, True):
            r = h.solve(Q, form="tc", tc_pair=pair)
            assert r["form"] == "tc"
            _check(Q, _as_sol(r), ref)
        for pair in (False, True):
            mins = []
            for s in range(3):  # one pending two-phase solve per handle: begin, then finish
                mins.append(h.solve_begin(Q, form="tc", shard_index=s, shard_count=3, tc_pair=pair))
                h.solve_finish(mins[-1], n)
            outs = []
            for s in range(3):
                h.solve_begin(Q, form="tc", shard_index=s, shard_count=3, tc_pair=pair)
                outs.append(h.solve_finish(min(mins), n))
            best = min((o for o in outs if o["found"]), key=lambda o: (o["best_E"], o["order_key"]))
            assert best["best_X_int"] == ref["best_X_int"]


class _as_sol:
    """A solve() result dict seen through the attributes _check reads."""

    def __init__(self, r):
        self.best_X = r["best_X"]
        self.best_E = r["best_E"]
        self.search = r


@pytest.mark.parametrize("n,hi,seed", [(20, 100, 1), (24, 100, 2), (29, 60, 3), (33, 40, 4), (36, 25, 5)])
def test_tensor_core_16bit_epilogue(cuda_ok, n, hi, seed):
    """Integer Q whose accumulator values span fewer than 2^16 integers runs the 16-bit
    epilogue (exact unsigned 16-bit minima over packed TMEM loads): the oracle's answer, the
    exact minimum as pass-1 minimum, and the same result as the fp32 minima (QB_FLAG_TC_NO16),
    whole problem and three shards."""
    rng = np.random.default_rng(900 + seed)
    Q = rng.integers(-hi, hi + 1, (n, n)).astype(np.int32)
    ref = oracle.qbf_port(Q)
    h = _lib.handle(0)
    rd = h.solve(Q, form="tc")
    r16 = h.solve(Q, form="tc", tc_one=True)
    r32 = h.solve(Q, form="tc", tc_no16=True)
    # the default is the 16-bit pair form wherever it applies, as here
    assert rd["plan"]["tc_kernel"] == "pair_u16"
    assert r16["plan"]["tc_kernel"] == "u16" and r32["plan"]["tc_kernel"] == "fp32"
    for r in (rd, r16, r32):
        assert (r["best_X_int"], r["best_E_int"]) == (ref["best_X_int"], ref["best_E"])
        assert r["pass1_min"] == ref["best_E"] or (ref["best_E"] == 0 and r["pass1_min"] >= 0)
    for kw in ({}, {"tc_one": True}):
        mins = []
        for s in range(3):
            mins.append(h.solve_begin(Q, form="tc", shard_index=s, shard_count=3, **kw))
            h.solve_finish(mins[-1], n)
        outs = []
        for s in range(3):
            h.solve_begin(Q, form="tc", shard_index=s, shard_count=3, **kw)
            outs.append(h.solve_finish(min(mins), n))
        best = min((o for o in outs if o["found"]), key=lambda o: (o["best_E"], o["order_key"]))
        assert best["best_X_int"] == ref["best_X_int"]


@pytest.mark.parametrize("n,hi,seed", [(24, 100, 11), (27, 70, 12), (31, 50, 13), (36, 25, 14)])
def test_tensor_core_pair_16bit_epilogue(cuda_ok, n, hi, seed):
    """The pair form's 16-bit epilogue (two states per packed accumulator: per-chunk minima
    for the MMA's tile, per-position minima over the chunks for the partner tile): the oracle's answer and exact pass-1 minimum,
    the same result as the pair form's fp32 minima, whole problem and five shards (shards start
    on either sign of the pair's shared variable)."""
    rng = np.random.default_rng(950 + seed)
    Q = rng.integers(-hi, hi + 1, (n, n)).astype(np.int32)
    Q[n - 16, n - 8:] = rng.integers(-hi, hi + 1, 8)  # couplings of the pair's variable with u
    ref = oracle.qbf_port(Q)
    h = _lib.handle(0)
    r16 = h.solve(Q, form="tc", tc_pair=True)
    r32 = h.solve(Q, form="tc", tc_pair=True, tc_no16=True)
    assert r16["plan"]["tc_kernel"] == "pair_u16" and r32["plan"]["tc_kernel"] == "pair"
    for r in (r16, r32):
        assert (r["best_X_int"], r["best_E_int"]) == (ref["best_X_int"], ref["best_E"])
        assert r["pass1_min"] == ref["best_E"] or (ref["best_E"] == 0 and r["pass1_min"] >= 0)
    mins = []
    for s in range(5):
        mins.append(h.solve_begin(Q, form="tc", tc_pair=True, shard_index=s, shard_count=5))
        h.solve_finish(mins[-1], n)
    assert min(mins) == r16["pass1_min"]
    outs = []
    for s in range(5):
        h.solve_begin(Q, form="tc", tc_pair=True, shard_index=s, shard_count=5)
        outs.append(h.solve_finish(min(mins), n))
    best = min((o for o in outs if o["found"]), key=lambda o: (o["best_E"], o["order_key"]))
    assert best["best_X_int"] == ref["best_X_int"]


def test_tensor_core_pair_16bit_shard_minima(cuda_ok):
    """The pass-1 minimum of every one of 16 shards of the 16-bit pair form equals the fp32
    pair form's and the one-state form's (all exact on integer Q)."""
    rng = np.random.default_rng(961)
    n = 30
    Q = rng.integers(-60, 61, (n, n)).astype(np.int32)
    h = _lib.handle(0)
    for s in range(16):
        got = []
        for kw in ({"tc_pair": True}, {"tc_pair": True, "tc_no16": True}, {}):
            got.append(h.solve_begin(Q, form="tc", shard_index=s, shard_count=16, **kw))
            h.solve_finish(got[-1], n)
        assert got[0] == got[1] == got[2], (s, got)


def test_tensor_core_pair_16bit_needs_room_for_chunk_shifts(cuda_ok):
    """Accumulator values that span fewer than 2^16 integers, but not with the pair's chunk
    offsets added (sum of |couplings| of the pair's variable with u bits 4..6, here 880 + 2 x
    1000 on a span of 63,720): the default is then the one-state 16-bit kernel, the pair form
    keeps fp32 minima, both exact; the pair and one-state flags together are refused."""
    n = 24
    rng = np.random.default_rng(962)
    Q = np.zeros((n, n), np.int32)
    for t in range(n - 15):
        Q[t, n - 8:] = 880  # t-u couplings: span 63,720
    Q[n - 16, n - 8:n - 5] = 1000  # the pair's variable with u bits 7, 6, 5: shifts of 3000
    Q[np.arange(n - 8), np.arange(n - 8)] = -rng.integers(0, 2000, n - 8)
    ref = oracle.qbf_port(Q)
    h = _lib.handle(0)
    d = h.solve(Q, form="tc")
    p = h.solve(Q, form="tc", tc_pair=True)
    assert d["plan"]["tc_kernel"] == "u16" and p["plan"]["tc_kernel"] == "pair"
    for r in (d, p):
        assert (r["best_X_int"], r["best_E_int"]) == (ref["best_X_int"], ref["best_E"])
    with pytest.raises(ValueError):
        h.solve(Q, form="tc", tc_pair=True, tc_one=True)


def test_tensor_core_16bit_epilogue_applies_only_in_range(cuda_ok):
    """On the exact integer path a coupling row beyond +-2048 or a value span of 2^16 or more
    keeps the fp32 minima; float Q takes the 16-bit pair form on rounded values."""
    rng = np.random.default_rng(77)
    n = 26
    h = _lib.handle(0)
    wide = rng.integers(-100, 101, (n, n)).astype(np.int32)
    wide[n - 9, n - 8:] = 400  # one coupling row of a y variable sums to 3200
    span = rng.integers(-2000, 2001, (n, n)).astype(np.int32)
    for Q in (wide, span):
        r = h.solve(Q, form="tc")
        assert r["plan"]["tc_kernel"] == "fp32"
        ref = oracle.qbf_port(Q)
        assert (r["best_X_int"], r["best_E_int"]) == (ref["best_X_int"], ref["best_E"])
    f = h.solve(rng.standard_normal((n, n)), form="tc")
    assert f["plan"]["tc_kernel"] == "pair_u16" and f["err_bound"] > 0


@pytest.mark.parametrize("n,seed", [(20, 1), (24, 2), (29, 3), (33, 4), (36, 5)])
def test_tensor_core_pair_16bit_float(cuda_ok, n, seed):
    """Float Q in the 16-bit pair form: values rounded to integers in units of a power of two,
    a stated error bound, every record within twice the bound re-walked in FP64.  The FP64
    argmin and energy of the oracle (float32 and float64 Q), the same state as the one-state
    fp32 kernel, whole problem and three shards."""
    rng = np.random.default_rng(990 + seed)
    G = rng.standard_normal((n, n))
    h = _lib.handle(0)
    for Q in (((G + G.T) / 2).astype(np.float32), G):
        ref = oracle.qbf_port(Q)
        r = h.solve(Q, form="tc")
        assert r["plan"]["tc_kernel"] == "pair_u16" and r["err_bound"] > 0
        _check(Q, _as_sol(r), ref)
        one = h.solve(Q, form="tc", tc_one=True)
        assert one["plan"]["tc_kernel"] == "fp32" and one["best_X_int"] == r["best_X_int"]
        mins = []
        for s in range(3):
            mins.append(h.solve_begin(Q, form="tc", shard_index=s, shard_count=3))
            h.solve_finish(mins[-1], n)
        outs = []
        for s in range(3):
            h.solve_begin(Q, form="tc", shard_index=s, shard_count=3)
            outs.append(h.solve_finish(min(mins), n))
        best = min((o for o in outs if o["found"]), key=lambda o: (o["best_E"], o["order_key"]))
        assert best["best_X_int"] == ref["best_X_int"]


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_float_near_ties_below_the_error_bound(cuda_ok, seed):
    """A 5-city TSP QUBO (its optimal tours tie: every tour in both directions) plus symmetric
    float noise of 1e-6: the optima differ by far less than the pass-1 error bound of the
    rounded 16-bit pair form, so every record holding one must become a candidate and the
    FP64 re-walk must pick the oracle's state, in every form."""
    from qubo_b200.problems import TSP
    rng = np.random.default_rng(seed)
    w = rng.integers(1, 101, (5, 5))
    w = np.triu(w, 1)
    w = w + w.T
    noise = rng.standard_normal((25, 25)) * 1e-6
    Q = TSP.qubo_from_distances(w.astype(np.float64)) + (noise + noise.T) / 2
    ref = oracle.qbf_port(Q)
    h = _lib.handle(0)
    r = h.solve(Q, form="tc")
    assert r["plan"]["tc_kernel"] == "pair_u16" and r["err_bound"] > 1e-3
    assert r["candidate_records"] >= 2
    _check(Q, _as_sol(r), ref)
    for form in ("gray", "exact", "auto"):
        _check(Q, _as_sol(h.solve(Q, form=form)), ref)


def test_tensor_core_pair_16bit_rounded_integers(cuda_ok):
    """Integer Q beyond the exact-digit range (sum|Q| > 2^22) takes the 16-bit pair form on
    rounded values with a nonzero error bound; pass 2 makes the answer bit-exact.  A problem
    whose u variables have no couplings (a zero value span) keeps one state per accumulator."""
    rng = np.random.default_rng(995)
    n = 26
    Q = rng.integers(-300000, 300001, (n, n)).astype(np.int64)
    ref = oracle.qbf_port(Q)
    h = _lib.handle(0)
    r = h.solve(Q, form="tc")
    assert r["plan"]["tc_kernel"] == "pair_u16" and r["err_bound"] > 0
    assert (r["best_X_int"], r["best_E_int"]) == (ref["best_X_int"], ref["best_E"])
    Z = rng.standard_normal((n, n))
    Z[:, n - 8:] = 0.0
    Z[n - 8:, :] = 0.0
    z = h.solve(Z, form="tc")
    assert z["plan"]["tc_kernel"] == "fp32"
    _check(Z, _as_sol(z), oracle.qbf_port(Z))
