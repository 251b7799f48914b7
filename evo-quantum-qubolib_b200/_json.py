"""JSON round trip for problems, solver kwargs and solutions.

The reference serialises with ``jsonpickle`` (src/qubo_lib/solution.py:64-69,
src/qubo_lib/abc/solver_abc.py:50).  When jsonpickle is importable the same encoder is
used, so ``solver_params_json`` and ``to_json`` strings keep the reference's format.
Otherwise a small self-describing encoder with the same object-tag convention
(``{"py/object": "module.Class", ...}``) is used; it round-trips every field this package
stores (numpy arrays, numpy scalars, nested objects, tuples, sets).
"""
from __future__ import annotations

import base64
import importlib
import json

import numpy as np

try:  # pragma: no cover - depends on the environment
    import jsonpickle as _jsonpickle
except Exception:  # noqa: BLE001
    _jsonpickle = None


def _enc(o):
    if isinstance(o, np.ndarray):
        return {"py/numpy.ndarray": {"dtype": o.dtype.str, "shape": list(o.shape),
                                     "b64": base64.b64encode(np.ascontiguousarray(o).tobytes()).decode()}}
    if isinstance(o, np.generic):
        return {"py/numpy.scalar": {"dtype": o.dtype.str, "value": o.item()}}
    if isinstance(o, type):
        return {"py/type": f"{o.__module__}.{o.__qualname__}"}
    if isinstance(o, tuple):
        return {"py/tuple": [_enc(v) for v in o]}
    if isinstance(o, (set, frozenset)):
        return {"py/set": [_enc(v) for v in sorted(o, key=repr)]}
    if isinstance(o, dict):
        return {str(k): _enc(v) for k, v in o.items()}
    if isinstance(o, list):
        return [_enc(v) for v in o]
    if isinstance(o, (str, int, float, bool)) or o is None:
        return o
    d = getattr(o, "__dict__", None)
    if d is not None:
        out = {"py/object": f"{type(o).__module__}.{type(o).__qualname__}"}
        out.update({k: _enc(v) for k, v in d.items()})
        return out
    return repr(o)


def _resolve(path: str):
    mod, _, name = path.rpartition(".")
    return getattr(importlib.import_module(mod), name)


def _dec(o):
    if isinstance(o, list):
        return [_dec(v) for v in o]
    if not isinstance(o, dict):
        return o
    if "py/numpy.ndarray" in o:
        a = o["py/numpy.ndarray"]
        return np.frombuffer(base64.b64decode(a["b64"]), dtype=np.dtype(a["dtype"])).reshape(a["shape"]).copy()
    if "py/numpy.scalar" in o:
        a = o["py/numpy.scalar"]
        return np.dtype(a["dtype"]).type(a["value"])
    if "py/type" in o:
        return _resolve(o["py/type"])
    if "py/tuple" in o:
        return tuple(_dec(v) for v in o["py/tuple"])
    if "py/set" in o:
        return set(_dec(v) for v in o["py/set"])
    if "py/object" in o:
        cls = _resolve(o["py/object"])
        obj = cls.__new__(cls)
        obj.__dict__.update({k: _dec(v) for k, v in o.items() if k != "py/object"})
        return obj
    return {k: _dec(v) for k, v in o.items()}


def encode(obj, indent: int | None = 4) -> str:
    if _jsonpickle is not None:
        return _jsonpickle.encode(obj, indent=indent)
    return json.dumps(_enc(obj), indent=indent)


def decode(s: str):
    if _jsonpickle is not None:
        return _jsonpickle.decode(s)
    return _dec(json.loads(s))
