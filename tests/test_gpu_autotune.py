"""qb_autotune: times the Gray-code and tensor-core forms on the device, caches the faster
one per n in the handle, and QB_FORM_AUTO then uses it (answers unchanged)."""
import numpy as np
import pytest

import oracle
import qubo_b200  # noqa: F401
from qubo_b200 import _lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,dtype", [(12, np.int32), (26, np.int16), (30, np.float32)])
def test_autotune_choice_is_used(cuda_ok, n, dtype):
    h = _lib.Handle(0)
    try:
        form = h.autotune(n, dtype)
        assert form in (("exact",) if n < 20 else ("gray", "tc"))
        rng = np.random.default_rng(n)
        Q = (rng.integers(-50, 51, (n, n)) if np.issubdtype(dtype, np.integer)
             else rng.standard_normal((n, n))).astype(dtype)
        r = h.solve(Q, form="auto")
        assert r["form"] == form
        ref = oracle.qbf_port(Q)
        assert r["best_X_int"] == ref["best_X_int"]
        assert abs(r["best_E"] - ref["best_E"]) <= 1e-9 * max(1.0, abs(ref["best_E"]))
    finally:
        h.close()
