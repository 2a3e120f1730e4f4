"""Loading of the in-tree shared libraries (fails loudly when missing)."""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "lib")

_cache: dict[str, ctypes.CDLL] = {}


def load(name: str) -> ctypes.CDLL:
    """Load ``programs_b200/lib/<name>``; raise if it has not been built."""
    if name in _cache:
        return _cache[name]
    path = os.path.join(LIB, name)
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is missing: build it with `python -m programs_b200.build` "
            "(there is no CPU fallback for the solver path)")
    lib = ctypes.CDLL(path)
    _cache[name] = lib
    return lib
