"""tioga_b200: TIOGA's overset-connectivity C API on a B200 GPU.

The product is the shared library ``libtioga_b200.so`` (built in-tree by
``python -m tioga_b200.build``), which exports TIOGA's C/Fortran interface.
This package adds:

* ``capi``  -- a ctypes mirror of that interface (works with any library that
  exports it, e.g. the CPU oracle in ``oracle/`` for comparisons);
* ``cases`` -- the seeded synthetic overset systems used by tests and bench;
* ``library_path()`` / ``extras()`` -- locate the GPU library and its
  ``tioga_b200_*`` additions (statistics, timings, precision mode).

There is no CPU fallback: ``library_path()`` raises when the CUDA library has
not been built.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_NAME = "libtioga_b200.so"


def library_path() -> str:
    p = os.path.join(_HERE, LIB_NAME)
    if not os.path.exists(p):
        raise RuntimeError(
            f"{LIB_NAME} is not built (run `python -m tioga_b200.build`); the GPU path has no fallback")
    return p


def extras(lib: C.CDLL):
    """Bind the tioga_b200_* additions on an already loaded library."""
    lib.tioga_b200_last_error.restype = C.c_int
    lib.tioga_b200_device_ok.restype = C.c_int
    return lib


def stats(lib: C.CDLL) -> dict:
    out = (C.c_longlong * 16)()
    lib.tioga_b200_stats_(out)
    keys = ["nquery", "ndonor", "nties", "ncand", "nrefine", "nreceptor", "nhole", "nrecords",
            "error", "npairs", "launches", "cand_verts", "nleaf", "nmerged"]
    return {k: int(out[i]) for i, k in enumerate(keys)}


def timing(lib: C.CDLL) -> dict:
    out = (C.c_float * 16)()
    lib.tioga_b200_timing_(out)
    keys = ["upload", "holemap", "boxes_refit", "query", "search", "donors", "celliblank",
            "download", "total", "search_traverse", "search_candidates", "search_refine", "cell_pass",
            "cell_boxes"]
    return {k: float(out[i]) for i, k in enumerate(keys)}


def set_int(lib: C.CDLL, fn: str, v: int):
    getattr(lib, fn)(C.byref(C.c_int(int(v))))
