"""Import shim: makes the package directory ``evo-quantum-qubolib_b200/`` importable as
``qubo_b200`` (a directory name with hyphens is not a Python identifier).

    import qubo_b200
    from qubo_b200.solvers import QBF, QB_F1, Parallel
    from qubo_b200.problems import RandomQUBO, Just_Q, TSP, MaxCut, ReducedProblem
"""
import importlib.util as _ilu
import os as _os
import sys as _sys

_PKG_DIR = _os.path.join(_os.path.dirname(_os.path.abspath(__file__)), "evo-quantum-qubolib_b200")
_spec = _ilu.spec_from_file_location(__name__, _os.path.join(_PKG_DIR, "__init__.py"),
                                     submodule_search_locations=[_PKG_DIR])
_mod = _ilu.module_from_spec(_spec)
_sys.modules[__name__] = _mod
_spec.loader.exec_module(_mod)
