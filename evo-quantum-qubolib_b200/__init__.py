"""qubo_b200 -- B200-native exhaustive QUBO search, a drop-in for qubo_lib's brute-force
solvers (QBF, QB_F1 and Parallel over them).

Host code is Python; the search runs in hand-written sm_100a CUDA kernels reached through
the C ABI of ``libqubo_b200.so`` (declared in include/qubo_b200.h).  There is no CPU
fallback: solving needs a CUDA device and the built library.
"""
import logging as _logging

__version__ = "0.1.0"

_logging.getLogger(__name__).addHandler(_logging.NullHandler())
