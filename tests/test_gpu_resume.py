"""Resumable search (qubo_b200.resume): a run stopped after some shares and restarted from
its checkpoint gives the answer of one call over the whole space."""
import json

import numpy as np
import pytest

import qubo_b200  # noqa: F401
from qubo_b200 import _lib
from qubo_b200.resume import solve_resumable

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype,form", [(np.int32, "tc"), (np.float64, "gray"), (np.int16, "auto")])
def test_stop_and_resume_matches_one_call(cuda_ok, tmp_path, dtype, form):
    rng = np.random.default_rng(4)
    n = 28
    Q = (rng.integers(-5, 6, (n, n)) if dtype != np.float64 else rng.standard_normal((n, n))).astype(dtype)
    path = str(tmp_path / "ckpt.json")
    first = solve_resumable(Q, 8, path, form=form, max_chunks_this_call=3)
    assert not first["done"] and first["next"] == 3
    assert json.load(open(path))["next"] == 3
    last = solve_resumable(Q, 8, path, form=form)
    assert last["done"] and last["states"] == 1 << n
    ref = _lib.handle(0).solve(Q, form=form)
    assert (last["best_X_int"], last["best_E"]) == (ref["best_X_int"], ref["best_E"])
    assert last["order_key"] == ref["order_key"]
    with pytest.raises(ValueError):
        solve_resumable(Q, 4, path, form=form)
