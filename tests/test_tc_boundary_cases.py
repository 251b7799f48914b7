"""The boundary cases of tests/test_gpu_tc_boundary.py hit the limits they are built for
(checked on the CPU, so a GPU run cannot pass on cases that miss the edge)."""
import numpy as np
import pytest

import tc_boundary_cases as tcb


@pytest.mark.parametrize("n", [24, 32, 36])
def test_cases_sit_at_the_limit(n):
    for kind in tcb.KINDS:
        Q = tcb.make_case(n, kind)
        want = {"at_limit": tcb.LIMIT, "over_limit": tcb.LIMIT + 1}.get(kind, tcb.LIMIT - 1)
        assert tcb.abs_sum(Q) == want
        assert np.array_equal(Q, np.triu(Q))
        assert np.abs(Q).max() < 2 ** 31  # fits the int32 the GPU tests pass
    # one contraction row near -2^22: its high base-2048 digit is -2048
    v = -int(tcb.coupling_sums(tcb.make_case(n, "v_row")).max())
    assert v // 2048 == -2048
    assert tcb.coupling_sums(tcb.make_case(n, "v_spread")).min() > 2 ** 18
    assert tcb.coupling_sums(tcb.make_case(n, "cancel")).max() > 2 ** 20
