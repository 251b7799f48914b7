"""qb_solve_noalloc (the entry point that allocates nothing) against qb_solve and the oracle.

Q and the result live in device memory owned by the caller (torch tensors here); the call
goes through the C ABI with ctypes.  Each case runs two different problems back to back
and compares both with qb_solve's Gray form on the same inputs and with the oracle (the C
restatement of the reference's QBF loop): bit-exact for integer Q, the FP64 argmin with the
energy within 1e-9 relative for float Q.  The status cases cover rejected input (NaN,
fractional entries with is_integer set), too many candidate records and the 2^53 range.
"""
import ctypes

import numpy as np
import pytest

import oracle
from qubo_b200 import _lib

pytestmark = pytest.mark.gpu

RESULT_BYTES = ctypes.sizeof(_lib.QbNoAllocResult)


def _noalloc(torch, Q: np.ndarray, is_integer: bool, prefix_bits: int = -1, out=None):
    q = torch.as_tensor(np.ascontiguousarray(Q, dtype=np.float64), device="cuda:0")
    if out is None:
        out = torch.zeros(RESULT_BYTES, dtype=torch.uint8, device="cuda:0")
    stream = torch.cuda.current_stream(0).cuda_stream
    rc = _lib.load().qb_solve_noalloc(0, q.data_ptr(), Q.shape[0], int(is_integer), int(prefix_bits),
                                      out.data_ptr(), stream)
    return rc, q, out


def _read(torch, out) -> _lib.QbNoAllocResult:
    torch.cuda.synchronize()
    raw = out.cpu().numpy().tobytes()
    return _lib.QbNoAllocResult.from_buffer_copy(raw)


def _reference(Q, prefix_bits=-1):
    return _lib.handle(0).solve(Q, form="gray", prefix_bits=prefix_bits)


@pytest.fixture
def torch_cuda(cuda_ok):
    import torch
    return torch


def _int_problem(n, seed, lo=-100, hi=100):
    rng = np.random.default_rng(seed)
    return rng.integers(lo, hi, size=(n, n)).astype(np.int16)


def _float_problem(n, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n, n)).astype(np.float64)


@pytest.mark.parametrize("n", [20, 27, 36])
def test_integer_two_calls_match_qb_solve(torch_cuda, n):
    torch = torch_cuda
    Qa, Qb = _int_problem(n, 100 + n), _int_problem(n, 200 + n)
    rca, qa, outa = _noalloc(torch, Qa.astype(np.float64), True)
    rcb, qb, outb = _noalloc(torch, Qb.astype(np.float64), True)
    assert rca == 0 and rcb == 0
    ra, rb = _read(torch, outa), _read(torch, outb)
    for Q, r in ((Qa, ra), (Qb, rb)):
        ref = _reference(Q)
        assert r.status == 0
        assert r.best_e == ref["best_E"]  # integer energies: exact
        assert r.best_x == ref["best_X_int"]
        assert r.order_key == ref["order_key"]
        orc = oracle.qbf_port(Q)
        assert (r.best_x, r.best_e) == (orc["best_X_int"], orc["best_E"])


@pytest.mark.parametrize("n", [22, 31])
def test_float_two_calls_match_qb_solve(torch_cuda, n):
    torch = torch_cuda
    Qa, Qb = _float_problem(n, 300 + n), _float_problem(n, 400 + n)
    _, _, outa = _noalloc(torch, Qa, False)
    _, _, outb = _noalloc(torch, Qb, False)
    ra, rb = _read(torch, outa), _read(torch, outb)
    for Q, r in ((Qa, ra), (Qb, rb)):
        ref = _reference(Q)
        assert r.status == 0
        # both are FP64 re-evaluations of the same state: tolerance 1e-9 relative
        assert abs(r.best_e - ref["best_E"]) <= 1e-9 * max(1.0, abs(ref["best_E"]))
        assert r.best_x == ref["best_X_int"]
        orc = oracle.qbf_port(Q)
        assert r.best_x == orc["best_X_int"]
        assert abs(r.best_e - orc["best_E"]) <= 1e-9 * max(1.0, abs(orc["best_E"]))


def test_prefix_bits_and_repeat(torch_cuda):
    """A non-default Gray prefix and the same call twice give qb_solve's answer both times."""
    torch = torch_cuda
    Q = _int_problem(24, 7, -3, 3)  # many ties: the order key decides
    ref = _reference(Q, prefix_bits=9)
    out = torch.zeros(RESULT_BYTES, dtype=torch.uint8, device="cuda:0")
    for _ in range(2):
        rc, _, _ = _noalloc(torch, Q.astype(np.float64), True, prefix_bits=9, out=out)
        assert rc == 0
        r = _read(torch, out)
        assert r.status == 0
        assert (r.best_e, r.best_x, r.order_key) == (ref["best_E"], ref["best_X_int"], ref["order_key"])
    orc = oracle.qbf_port(Q, A=9)
    assert (r.best_x, r.best_e) == (orc["best_X_int"], orc["best_E"])


def test_no_device_memory_taken_after_setup(torch_cuda):
    torch = torch_cuda
    Q = _int_problem(32, 11).astype(np.float64)
    q = torch.as_tensor(Q, device="cuda:0")
    out = torch.zeros(RESULT_BYTES, dtype=torch.uint8, device="cuda:0")
    stream = torch.cuda.current_stream(0).cuda_stream
    L = _lib.load()
    assert L.qb_solve_noalloc(0, q.data_ptr(), 32, 1, -1, out.data_ptr(), stream) == 0  # set-up call
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for _ in range(3):
        assert L.qb_solve_noalloc(0, q.data_ptr(), 32, 1, -1, out.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0
    assert _read(torch, out).status == 0


def test_sizes_outside_the_scratch_are_rejected(torch_cuda):
    torch = torch_cuda
    for n in (19, 37):
        rc, _, _ = _noalloc(torch, np.zeros((n, n)), True)
        assert rc == _lib.QB_ETOOBIG
    assert "no-allocation" in _lib.strerror(_lib.QB_ETOOBIG)


def _status(torch, Q, is_integer):
    rc, _, out = _noalloc(torch, Q, is_integer)
    assert rc == 0  # the problem is queued; its status is in the device result
    return _read(torch, out)


def test_rejected_input(torch_cuda):
    """NaN / infinity anywhere, or a fractional entry when the caller says Q is integer."""
    torch = torch_cuda
    base = _int_problem(24, 31).astype(np.float64)
    for bad in (np.nan, np.inf, -np.inf):
        Q = base.copy()
        Q[3, 17] = bad
        for is_int in (True, False):
            assert _status(torch, Q, is_int).status == _lib.QB_EINVAL
    Q = base.copy()
    Q[5, 5] = 0.5
    assert _status(torch, Q, True).status == _lib.QB_EINVAL
    r = _status(torch, Q, False)  # the same matrix as float input is fine
    orc = oracle.qbf_port(Q)
    assert r.status == 0 and r.best_x == orc["best_X_int"]
    assert abs(r.best_e - orc["best_E"]) <= 1e-9 * max(1.0, abs(orc["best_E"]))


def test_too_many_candidates(torch_cuda):
    """Float Q = 0 at n = 28: every one of the 8192 records ties with the minimum, more than
    the 4096 that fit."""
    r = _status(torch_cuda, np.zeros((28, 28)), False)
    assert r.status == _lib.QB_EOVERFLOW and r.candidates > 4096


def test_integer_range_limit(torch_cuda):
    Q = np.zeros((22, 22))
    Q[0, 0] = -2.0 ** 53
    assert _status(torch_cuda, Q, True).status == _lib.QB_ERANGE


def test_zero_answer_needs_no_candidates(torch_cuda):
    """Exact integer Q with no negative energy: X = 0 is the answer and nothing is re-walked."""
    r = _status(torch_cuda, np.ones((26, 26)), True)
    assert (r.status, r.best_x, r.best_e, r.order_key, r.candidates) == (0, 0, 0.0, 0, 0)
