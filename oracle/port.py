"""ctypes access to the C restatement oracle (oracle/_ref/libldl_oracle.so).

Test infrastructure only: the numeric multifrontal LDL^T restated in plain C
from the reference's sparse_ldl.h, driven by the symbolic structure the
reference computes (or any structure with the same layout). Used by tests/
and bench.py's CPU-baseline leg; the product package never imports it.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "_ref", "libldl_oracle.so")
_i32p = ctypes.POINTER(ctypes.c_int)
_f64p = ctypes.POINTER(ctypes.c_double)
_lib = None


def load():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(LIB)
        lib.ldlo_create.restype = ctypes.c_void_p
        lib.ldlo_create.argtypes = [ctypes.c_int, _i32p, _i32p, ctypes.c_int] + [_i32p] * 7 + [
            ctypes.c_double, ctypes.c_double]
        lib.ldlo_destroy.argtypes = [ctypes.c_void_p]
        lib.ldlo_factor.argtypes = [ctypes.c_void_p, _f64p, _f64p]
        lib.ldlo_solve.argtypes = [ctypes.c_void_p, ctypes.c_int, _f64p, ctypes.c_int]
        lib.ldlo_inertia.argtypes = [ctypes.c_void_p, _i32p, _i32p]
        lib.ldlo_pivot_record.restype = ctypes.c_longlong
        lib.ldlo_pivot_record.argtypes = [ctypes.c_void_p, _i32p, _i32p, _i32p, _i32p]
        _lib = lib
    return _lib


class PortLDL:
    """Numeric restatement on a given symbolic structure (dict with the keys
    of ``oracle.ref.RefLDL.symbolic()``)."""

    def __init__(self, rowp, cols, sym: dict, ustab=0.01, pivot_tol=1e-14):
        self._lib = load()
        self.rowp = np.ascontiguousarray(rowp, np.int32)
        self.cols = np.ascontiguousarray(cols, np.int32)
        self.n = len(self.rowp) - 1
        self._sym = {k: np.ascontiguousarray(v, np.int32) for k, v in sym.items()}
        s = self._sym
        nn = len(s["node_ptr"]) - 1
        ip = lambda a: a.ctypes.data_as(_i32p)  # noqa: E731
        self._h = self._lib.ldlo_create(
            self.n, ip(self.rowp), ip(self.cols), nn, ip(s["node_ptr"]), ip(s["node_to_var"]),
            ip(s["children_ptr"]), ip(s["children"]), ip(s["contrib_ptr"]),
            ip(s["contrib_rows"]), ip(s["invperm"]), ustab, pivot_tol)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ldlo_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def factor(self, vals, diag=None):
        self._vals = np.ascontiguousarray(vals, np.float64)
        self._diag = None if diag is None else np.ascontiguousarray(diag, np.float64)
        return self._lib.ldlo_factor(self._h, self._vals.ctypes.data_as(_f64p),
                                     self._diag.ctypes.data_as(_f64p)
                                     if self._diag is not None else None)

    def solve(self, b):
        x = np.array(b, dtype=np.float64, order="F", copy=True)
        nrhs = 1 if x.ndim == 1 else x.shape[1]
        self._lib.ldlo_solve(self._h, nrhs, x.ctypes.data_as(_f64p), self.n)
        return x

    def pivot_record(self) -> dict:
        """Per supernode: front size, pivots, delayed candidates, and the
        front variables after pivoting, in the layout of
        ``amigo_b200.sparse_ldl.SparseLDL.pivot_record``."""
        nn = len(self._sym["node_ptr"]) - 1
        total = self._lib.ldlo_pivot_record(self._h, None, None, None, None)
        rec = {k: np.empty(max(nn, 1), np.int32) for k in ("f", "npiv", "ndel")}
        rec["fv"] = np.empty(max(total, 1), np.int32)
        self._lib.ldlo_pivot_record(self._h, *[rec[k].ctypes.data_as(_i32p)
                                               for k in ("f", "npiv", "ndel", "fv")])
        return {"f": rec["f"][:nn], "npiv": rec["npiv"][:nn], "ndel": rec["ndel"][:nn],
                "fv": rec["fv"][:total]}

    def inertia(self):
        p = ctypes.c_int()
        q = ctypes.c_int()
        self._lib.ldlo_inertia(self._h, ctypes.byref(p), ctypes.byref(q))
        return (p.value, q.value)
