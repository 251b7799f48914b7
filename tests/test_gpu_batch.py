"""qb_solve_batch (QBF.solve_batch): many problems of uneven size in one batched search,
each answer equal to the single-problem answer and to the oracle's (bit-exact for integer
Q, FP64 argmin within 1e-9 relative for float Q)."""
import numpy as np
import pytest

import oracle
import qubo_b200  # noqa: F401
from conftest import bits_to_int, dec_q, load_golden
from qubo_b200 import _lib, configs
from qubo_b200.problems import Just_Q
from qubo_b200.solvers import QBF

pytestmark = pytest.mark.gpu


def _mixed(seed, count):
    rng = np.random.default_rng(seed)
    Qs = []
    for i in range(count):
        n = int(rng.integers(1, 27))
        kind = i % 4
        if kind == 0:
            U = rng.integers(-60, 61, (n, n)).astype(np.int32)
            Qs.append((np.triu(U) + np.triu(U, 1).T).astype(np.int32))
        elif kind == 1:
            Qs.append(rng.integers(-9, 10, (n, n)).astype(np.int16))
        elif kind == 2:
            Qs.append(rng.standard_normal((n, n)).astype(np.float32))
        else:
            G = rng.standard_normal((n, n))
            Qs.append((G + G.T) / 2)
    return Qs


def _check(Q, r):
    ref = oracle.qbf_port(Q)
    assert r["best_X_int"] == ref["best_X_int"], (Q.shape, Q.dtype, r, ref)
    if np.issubdtype(Q.dtype, np.integer):
        assert r["best_E"] == ref["best_E"]
    else:
        assert abs(r["best_E"] - ref["best_E"]) <= 1e-9 * max(1.0, abs(ref["best_E"]))


def test_batch_mixed_sizes_and_dtypes(cuda_ok):
    Qs = _mixed(3, 96)
    res = _lib.handle(0).solve_batch(Qs)
    assert len(res) == len(Qs)
    for Q, r in zip(Qs, res):
        _check(Q, r)


def test_batch_twice_and_matches_single_calls(cuda_ok):
    h = _lib.handle(0)
    Qs = _mixed(4, 40)
    a = h.solve_batch(Qs)
    b = h.solve_batch(Qs[::-1])[::-1]
    for Q, ra, rb in zip(Qs, a, b):
        rs = h.solve(Q, form="auto")
        assert ra["best_X_int"] == rb["best_X_int"] == rs["best_X_int"]
        assert ra["best_E"] == rb["best_E"]
        assert abs(ra["best_E"] - rs["best_E"]) <= 1e-9 * max(1.0, abs(rs["best_E"]))


def test_batch_read_only_and_strided_matrices(cuda_ok):
    """Members passed as read-only arrays and as non-contiguous views (the descriptors then
    point at a contiguous copy or come from the array interface) give the answers of their
    writable contiguous copies and of the oracle."""
    Qs = _mixed(11, 24)
    given = []
    for i, Q in enumerate(Qs):
        if i % 3 == 0:
            R = Q.copy()
            R.flags.writeable = False
            given.append(R)
        elif i % 3 == 1:
            given.append(np.asfortranarray(Q).T.T)  # same values, Fortran order
        else:
            given.append(np.ascontiguousarray(Q.T).T)  # a transposed view of Q's transpose
    h = _lib.handle(0)
    a = h.solve_batch(given)
    b = h.solve_batch(Qs)
    for Q, ra, rb in zip(Qs, a, b):
        assert (ra["best_X_int"], ra["best_E"]) == (rb["best_X_int"], rb["best_E"])
        _check(Q, ra)


def test_batch_ties_follow_the_split(cuda_ok):
    rng = np.random.default_rng(8)
    Qs = [rng.integers(-2, 3, (n, n)).astype(np.int32) for n in (12, 18, 22, 25)]
    for A in (0, 5, 9):
        res = _lib.handle(0).solve_batch(Qs, prefix_bits=A)
        for Q, r in zip(Qs, res):
            ref = oracle.qbf_port(Q, A=A)
            assert (r["best_X_int"], r["best_E"]) == (ref["best_X_int"], ref["best_E"])


def test_batch_natural_rule_and_large_member(cuda_ok):
    rng = np.random.default_rng(9)
    Qs = [rng.integers(-3, 4, (n, n)).astype(np.int32) for n in (10, 21, 25, 37)]
    res = _lib.handle(0).solve_batch(Qs, tie_rule="natural")
    for Q, r in zip(Qs, res):
        single = _lib.handle(0).solve(Q, tie_rule="natural")
        assert (r["best_X_int"], r["best_E"]) == (single["best_X_int"], single["best_E"])


def test_batch_empty_and_zero_matrices(cuda_ok):
    assert _lib.handle(0).solve_batch([]) == []
    res = _lib.handle(0).solve_batch([np.zeros((n, n), np.int32) for n in (3, 20, 26)])
    for r in res:
        assert r["best_E"] == 0 and r["best_X_int"] == 0


def test_solver_batch_cfg5_subset_against_reference(cuda_ok):
    cases = load_golden("configs.json")["cfg5_subset"]
    probs = [Just_Q(dec_q(c["Q"])) for c in cases]
    sols = QBF().solve_batch(probs, device="cuda")
    for c, p, sol in zip(cases, probs, sols):
        Q = p.build_Q_matrix()
        x = bits_to_int("".join(map(str, sol.best_X)))
        ref = oracle.qbf_port(Q)
        assert x == ref["best_X_int"]
        assert abs(float(sol.best_E) - ref["best_E"]) <= 1e-9 * max(1.0, abs(ref["best_E"]))
        assert sol.solver_class == "QBF" and sol.epochs_cnt == 2 ** sol_A(p.N)


def sol_A(n):
    return n - min(n, 20)


def test_batch_cfg5_sample_of_4096(cuda_ok):
    Qs = [configs.batch_instance(i) for i in range(0, 4096, 128)]
    res = _lib.handle(0).solve_batch(Qs)
    for Q, r in zip(Qs, res):
        _check(Q, r)


def test_batch_tensor_core_members_beyond_exact_digits(cuda_ok):
    """n >= 24 members take the tensor-core form; integers with sum |Q| > 2^22 use its
    float digits and an error bound, the answers stay exact after re-evaluation."""
    rng = np.random.default_rng(21)
    Qs = [rng.integers(-100000, 100001, (n, n)).astype(np.int64) for n in (24, 25, 26)]
    Qs += [rng.integers(-40, 41, (n, n)).astype(np.int16) for n in (24, 26)]
    res = _lib.handle(0).solve_batch(Qs)
    for Q, r in zip(Qs, res):
        assert r["form"] == "tc"
        _check(Q, r)


def test_batch_tensor_core_members_take_the_16bit_pair_kernel(cuda_ok):
    """When every tensor-core member (n >= 24) fits it, the batch runs the batched 16-bit pair
    kernel: float members on values rounded to a power-of-two unit with an error bound,
    integer members on exact digits; the oracle's answers, and the same states as the
    one-state kernel (QB_FLAG_TC_ONE); an integer member whose values span more than 2^16
    takes rounded values too and stays exact."""
    rng = np.random.default_rng(31)
    Qs = [configs.batch_instance(i) for i in range(0, 4096, 97)]
    Qs += [rng.integers(-40, 41, (n, n)).astype(np.int32) for n in (24, 27, 29)]
    h = _lib.handle(0)
    res = h.solve_batch(Qs)
    one = h.solve_batch(Qs, tc_one=True)
    for Q, r, r1 in zip(Qs, res, one):
        _check(Q, r)
        assert r1["best_X_int"] == r["best_X_int"]
        if r["form"] == "tc":
            assert r["plan"]["tc_kernel"] == "pair_u16" and r1["plan"]["tc_kernel"] == "fp32"
            assert (r["err_bound"] > 0) == (not np.issubdtype(Q.dtype, np.integer))
    assert sum(r["form"] == "tc" for r in res) >= 10
    wide = rng.integers(-2000, 2001, (26, 26)).astype(np.int32)  # exact digits, span beyond 2^16
    mix = h.solve_batch([Qs[0], wide])
    for Q, r in zip([Qs[0], wide], mix):
        _check(Q, r)


def test_batch_falls_back_to_one_state_when_a_member_does_not_fit(cuda_ok):
    """A tensor-core member the 16-bit pair kernel cannot take (float Q whose u variables have
    no couplings: a zero value span) keeps the whole batch on the one-state kernel, and every
    member keeps its own plan: an integer member on exact digits whose values span more than
    2^16 (which alone would take rounded values) stays exact, a float member keeps its bound."""
    rng = np.random.default_rng(41)
    n = 26
    wide = rng.integers(-2000, 2001, (n, n)).astype(np.int32)
    Z = rng.standard_normal((n, n))
    Z[:, n - 8:] = 0.0
    Z[n - 8:, :] = 0.0
    F = rng.standard_normal((n, n))
    Qs = [wide, Z, F]
    res = _lib.handle(0).solve_batch(Qs)
    for Q, r in zip(Qs, res):
        assert r["form"] == "tc" and r["plan"]["tc_kernel"] == "fp32", r["plan"]
        _check(Q, r)
    assert res[0]["err_bound"] == 0.0


def _same_shapes(Qs, seed):
    """New matrices with the sizes and dtypes of Qs (the same batch shape, other values)."""
    rng = np.random.default_rng(seed)
    out = []
    for Q in Qs:
        n = Q.shape[0]
        if np.issubdtype(Q.dtype, np.integer):
            out.append(rng.integers(-9, 10, (n, n)).astype(Q.dtype))
        else:
            out.append(rng.standard_normal((n, n)).astype(Q.dtype))
    return out


def test_batch_as_one_graph_launch(cuda_ok):
    """QB_FLAG_GRAPH: the first batch is captured, a batch of the same shape with other values
    replays the graph (its new inputs are uploaded by the replay), another shape is captured
    anew; every answer equals the oracle's and the launch-by-launch run's."""
    h = _lib.handle(0)
    Qa = _mixed(31, 48)
    Qb = _same_shapes(Qa, 32)
    Qc = _mixed(33, 20)
    for Qs in (Qa, Qb, Qb, Qc, Qa):
        g = h.solve_batch(Qs, graph=True)
        plain = h.solve_batch(Qs)
        for Q, rg, rp in zip(Qs, g, plain):
            _check(Q, rg)
            assert (rg["best_X_int"], rg["best_E"]) == (rp["best_X_int"], rp["best_E"])
        assert g[0]["kernels"] == plain[0]["kernels"] and g[0]["pass2_ms"] == 0.0
