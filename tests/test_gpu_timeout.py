"""The search kernel's failure path, without a GPU fault: with QB_FLAG_TEST_STALL the tile
walk publishes nothing, every other role's bounded wait (2 s) runs out, the kernel drains
and frees its tensor memory, and the call reports QB_ETIMEOUT.  The same handle then solves
normally."""
import numpy as np
import pytest

import oracle
import qubo_b200  # noqa: F401
from qubo_b200 import _lib

pytestmark = pytest.mark.gpu


def test_bounded_waits_report_timeout_and_context_survives(cuda_ok):
    h = _lib.Handle(0)
    try:
        Q = np.random.default_rng(3).integers(-50, 51, (24, 24)).astype(np.int32)
        with pytest.raises(_lib.QbError) as ei:
            h.solve(Q, form="tc", flags=_lib.QB_FLAG_TEST_STALL)
        assert ei.value.status == _lib.QB_ETIMEOUT
        r = h.solve(Q, form="tc")
        ref = oracle.qbf_port(Q)
        assert (r["best_X_int"], r["best_E"]) == (ref["best_X_int"], ref["best_E"])
    finally:
        h.close()
