"""The benchmark configurations on the GPU against the reference's own answers
(tests/golden/configs.json, recorded by running the reference QBF / Parallel on CPU):

  cfg1  RandomQUBO n=20 fp32 symmetrised (seed 0), every form
  cfg2  RandomQUBO n=32 int16 symmetric (seed 0), split A=12, every form
  cfg3  6-city TSP, integer distances (seed 0), n=36: QBF and Parallel(16 splits)
  cfg4  max-cut ER n=40 p=0.5 (seed 0): the reference's 2^30 slice exactly, and the full
        2^40 search (tensor-core and Gray forms agree; the full minimum bounds the slice's)
  cfg5  batch instances (seeds 1000+i) that the reference solved, against the FP64 oracle
"""
import numpy as np
import pytest

import oracle
import qubo_b200  # noqa: F401
from conftest import bits_to_int, dec_q, load_golden
from qubo_b200 import _lib, configs
from qubo_b200.problems import Just_Q, ReducedProblem
from qubo_b200.solvers import QBF, Parallel

pytestmark = pytest.mark.gpu
CFG = load_golden("configs.json")


def _xint(sol):
    return bits_to_int("".join(map(str, sol.best_X)))


@pytest.mark.parametrize("form", ["auto", "gray", "tc", "exact"])
def test_cfg1_n20_f32(cuda_ok, form):
    Q = configs.random_f32_n20()
    ref = CFG["cfg1"]["ref"]
    sol = QBF().solve(Just_Q(Q), device="cuda", form=form)
    assert _xint(sol) == bits_to_int(ref["best_X"])
    e64 = oracle.energy(Q, _xint(sol))
    assert abs(float(sol.best_E) - e64) <= 1e-9 * max(1.0, abs(e64))
    assert float(sol.best_E) == pytest.approx(ref["best_E"], rel=1e-5)  # the reference sums in fp32


@pytest.mark.parametrize("form", ["auto", "gray", "tc", "exact"])
def test_cfg2_n32_i16(cuda_ok, form):
    Q = configs.random_i16_n32()
    ref = CFG["cfg2"]["ref"]
    sol = QBF().solve(Just_Q(Q), device="cuda", A=12, form=form)
    assert _xint(sol) == bits_to_int(ref["best_X"])
    assert int(sol.best_E) == int(ref["best_E"])


@pytest.mark.parametrize("form", ["tc", "gray"])
def test_cfg3_tsp36(cuda_ok, form):
    Q = configs.tsp6_int()
    ref = CFG["cfg3"]["ref"]
    sol = Parallel(base_solver=QBF, splits_cnt=16, devices=["cuda"]).solve(Just_Q(Q), form=form)
    assert int(sol.best_E) == int(ref["best_E"]) == -991
    assert _xint(sol) == bits_to_int(ref["best_X"])
    x = np.array(sol.best_X).reshape(6, 6)
    assert (x.sum(axis=0) == 1).all() and (x.sum(axis=1) == 1).all()  # a valid tour
    sol1 = QBF().solve(Just_Q(Q), device="cuda", form=form)
    assert int(sol1.best_E) == -991


def test_cfg4_maxcut40(cuda_ok):
    Q = configs.maxcut_er()
    ref = CFG["cfg4"]["ref_slice"]
    rp = ReducedProblem(Just_Q(Q), np.zeros(10, dtype=np.int64))
    sl = QBF().solve(rp, device="cuda")
    assert _xint(sl) == bits_to_int(ref["best_X"])
    assert int(sl.best_E) == int(ref["best_E"])
    full = {f: _lib.handle(0).solve(Q, form=f) for f in ("tc", "gray")}
    assert full["tc"]["best_E"] == full["gray"]["best_E"] <= ref["best_E"]
    assert full["tc"]["best_X_int"] == full["gray"]["best_X_int"]
    assert oracle.energy(Q, full["tc"]["best_X_int"]) == full["tc"]["best_E"]
    assert full["tc"]["states"] == 1 << 40


@pytest.mark.parametrize("case", CFG["cfg5_subset"], ids=[f"i{c['index']}_n{c['Q']['n']}" for c in CFG["cfg5_subset"]])
def test_cfg5_instances(cuda_ok, case):
    Q = dec_q(case["Q"])
    assert np.array_equal(Q, configs.batch_instance(case["index"], seed=1000))
    sol = QBF().solve(Just_Q(Q), device="cuda")
    ref = oracle.qbf_port(Q)
    assert _xint(sol) == ref["best_X_int"]
    assert abs(float(sol.best_E) - ref["best_E"]) <= 1e-9 * max(1.0, abs(ref["best_E"]))
    # the reference compares fp32 sums: its state agrees unless two minima are that close
    rx = bits_to_int(case["ref"]["best_X"])
    if rx != _xint(sol):
        assert abs(oracle.energy(Q, rx) - ref["best_E"]) <= 1e-5 * max(1.0, abs(ref["best_E"]))
