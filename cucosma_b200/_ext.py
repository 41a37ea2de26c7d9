"""ctypes bindings of the optional entry points (grouped GEMM, sigmoid
forward/backward, tuner).  Each binding is attached only if the symbol is
exported by the loaded libcucosma.so."""
from __future__ import annotations

import ctypes as C


def bind(L):
    vp, sz = C.c_void_p, C.c_size_t
    table = {}
    for name, (argtypes, restype) in table.items():
        f = getattr(L, name, None)
        if f is not None:
            f.argtypes = argtypes
            f.restype = restype
