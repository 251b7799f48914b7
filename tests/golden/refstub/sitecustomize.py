"""Test-only import stubs that let the reference library run in this container.

The reference (cloud-ru-tech/evo-quantum-qubolib) imports ``jsonpickle`` to serialise
kwargs and problems, and ``ortools`` for the TSP ground-state helper; neither is on the
exhaustive-search arithmetic path and neither is installed here.  This file is placed on
PYTHONPATH by tests/golden/make_golden.py only, so that spawned ``Parallel`` workers load
the same stubs.
"""
import json
import sys
import types


def _encode(obj, indent=None, **_kw):
    def default(o):
        d = getattr(o, "__dict__", None)
        return {"py/object": type(o).__name__, **d} if d is not None else repr(o)
    return json.dumps(obj, indent=indent, default=default)


_jp = types.ModuleType("jsonpickle")
_jp.encode = _encode
_jp.decode = json.loads
sys.modules.setdefault("jsonpickle", _jp)

for _name in ("ortools", "ortools.constraint_solver", "ortools.constraint_solver.routing_enums_pb2",
              "ortools.constraint_solver.pywrapcp"):
    sys.modules.setdefault(_name, types.ModuleType(_name))
