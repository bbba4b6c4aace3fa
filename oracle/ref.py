"""ctypes access to the compiled reference oracle (oracle/_ref/liboracle_ref.so).

Test infrastructure only: the reference's own ``SparseLDL`` (Mersoltane/amigo
include/sparse_ldl.h, compiled unchanged by oracle/Makefile) used as the
checker for the GPU path and as the timed CPU baseline. The product package
never imports this module.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS: dict[str, ctypes.CDLL] = {}

ORDER_ND, ORDER_AMD, ORDER_MULTICOLOR, ORDER_NATURAL = 0, 1, 2, 3

_i32p = ctypes.POINTER(ctypes.c_int)
_f64p = ctypes.POINTER(ctypes.c_double)


def lib_path(openmp: bool = False) -> str:
    name = "liboracle_ref_omp.so" if openmp else "liboracle_ref.so"
    return os.path.join(_HERE, "_ref", name)


def available(openmp: bool = False) -> bool:
    return os.path.exists(lib_path(openmp))


def load(openmp: bool = False) -> ctypes.CDLL:
    key = "omp" if openmp else "serial"
    if key in _LIBS:
        return _LIBS[key]
    path = lib_path(openmp)
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
    lib = ctypes.CDLL(path)
    lib.oref_create.restype = ctypes.c_void_p
    lib.oref_create.argtypes = [
        ctypes.c_int, ctypes.c_int, _i32p, _i32p, ctypes.c_int, ctypes.c_int,
        ctypes.c_double, ctypes.c_double, ctypes.c_double,
    ]
    lib.oref_destroy.argtypes = [ctypes.c_void_p]
    lib.oref_num_nodes.argtypes = [ctypes.c_void_p]
    lib.oref_num_contrib.argtypes = [ctypes.c_void_p]
    lib.oref_get_symbolic.argtypes = [ctypes.c_void_p] + [_i32p] * 7
    lib.oref_etree.argtypes = [ctypes.c_void_p, _i32p, _i32p, _i32p]
    lib.oref_order.argtypes = [ctypes.c_int, _i32p, _i32p, ctypes.c_int, _i32p, _i32p]
    lib.oref_factor.argtypes = [ctypes.c_void_p, _f64p, _f64p]
    lib.oref_solve.argtypes = [ctypes.c_void_p, ctypes.c_int, _f64p, ctypes.c_int]
    lib.oref_inertia.argtypes = [ctypes.c_void_p, _i32p, _i32p]
    lib.oref_node_pivots.argtypes = [ctypes.c_void_p, _i32p, _i32p]
    lib.oref_csr_assemble.argtypes = [ctypes.c_int, ctypes.c_int, _i32p, _i32p, ctypes.c_int,
                                      _i32p, _i32p, _i32p, _f64p, _f64p]
    lib.oref_chol_create.restype = ctypes.c_void_p
    lib.oref_chol_create.argtypes = [ctypes.c_int, ctypes.c_int, _i32p, _i32p, ctypes.c_int]
    lib.oref_chol_destroy.argtypes = [ctypes.c_void_p]
    lib.oref_chol_factor.argtypes = [ctypes.c_void_p, _f64p]
    lib.oref_chol_solve.argtypes = [ctypes.c_void_p, _f64p]
    _LIBS[key] = lib
    return lib


def _ip(a: np.ndarray):
    return a.ctypes.data_as(_i32p)


def _fp(a: np.ndarray):
    return a.ctypes.data_as(_f64p)


def order(rowp, cols, kind: int = ORDER_AMD):
    """The reference's ordering (copy_for_reorder + reorder): (perm, iperm)."""
    lib = load()
    rowp = np.ascontiguousarray(rowp, dtype=np.int32)
    cols = np.ascontiguousarray(cols, dtype=np.int32)
    n = len(rowp) - 1
    perm = np.empty(n, np.int32)
    iperm = np.empty(n, np.int32)
    lib.oref_order(n, _ip(rowp), _ip(cols), kind, _ip(perm), _ip(iperm))
    return perm, iperm


class RefLDL:
    """The reference SparseLDL<double> on the host."""

    def __init__(self, rowp, cols, order: int = ORDER_AMD, cholesky: bool = False,
                 ustab: float = 0.01, pivot_tol: float = 1e-14,
                 delay_growth: float = 2.0, openmp: bool = False):
        self._lib = load(openmp)
        self.rowp = np.ascontiguousarray(rowp, dtype=np.int32)
        self.cols = np.ascontiguousarray(cols, dtype=np.int32)
        self.n = len(self.rowp) - 1
        self.nnz = int(self.rowp[-1])
        self._h = self._lib.oref_create(
            self.n, self.nnz, _ip(self.rowp), _ip(self.cols), order,
            1 if cholesky else 0, ustab, pivot_tol, delay_growth)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.oref_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    @property
    def num_nodes(self) -> int:
        return self._lib.oref_num_nodes(self._h)

    def symbolic(self) -> dict:
        nn = self.num_nodes
        nc = self._lib.oref_num_contrib(self._h)
        out = {
            "invperm": np.empty(self.n, np.int32),
            "node_ptr": np.empty(nn + 1, np.int32),
            "node_to_var": np.empty(self.n, np.int32),
            "children_ptr": np.empty(nn + 2, np.int32),
            "children": np.empty(max(nn, 1), np.int32),
            "contrib_ptr": np.empty(nn + 1, np.int32),
            "contrib_rows": np.empty(max(nc, 1), np.int32),
        }
        self._lib.oref_get_symbolic(
            self._h, *[_ip(out[k]) for k in (
                "invperm", "node_ptr", "node_to_var", "children_ptr",
                "children", "contrib_ptr", "contrib_rows")])
        out["children"] = out["children"][:nn]
        out["contrib_rows"] = out["contrib_rows"][:nc]
        return out

    def etree(self):
        parent = np.empty(self.n, np.int32)
        post = np.empty(self.n, np.int32)
        colcount = np.empty(self.n, np.int32)
        self._lib.oref_etree(self._h, _ip(parent), _ip(post), _ip(colcount))
        return parent, post, colcount

    def factor(self, vals, diag=None) -> int:
        vals = np.ascontiguousarray(vals, dtype=np.float64)
        if diag is not None:
            diag = np.ascontiguousarray(diag, dtype=np.float64)
            return self._lib.oref_factor(self._h, _fp(vals), _fp(diag))
        return self._lib.oref_factor(self._h, _fp(vals), None)

    def solve(self, b: np.ndarray) -> np.ndarray:
        x = np.array(b, dtype=np.float64, order="F", copy=True)
        nrhs = 1 if x.ndim == 1 else x.shape[1]
        self._lib.oref_solve(self._h, nrhs, _fp(x), self.n)
        return x

    def inertia(self) -> tuple[int, int]:
        p = ctypes.c_int(0)
        q = ctypes.c_int(0)
        self._lib.oref_inertia(self._h, ctypes.byref(p), ctypes.byref(q))
        return (p.value, q.value)

    def node_pivots(self):
        nn = self.num_nodes
        npiv = np.empty(nn, np.int32)
        ndel = np.empty(nn, np.int32)
        self._lib.oref_node_pivots(self._h, _ip(npiv), _ip(ndel))
        return npiv, ndel


class RefCholesky:
    """The reference's SparseCholesky (include/sparse_cholesky.h:64-375):
    a symmetric quasi-definite matrix factored in natural order, the first
    ``sqdef_index`` rows forming the positive definite block (-1: all)."""

    def __init__(self, rowp, cols, sqdef_index: int = -1, openmp: bool = False):
        self._lib = load(openmp)
        self.rowp = np.ascontiguousarray(rowp, dtype=np.int32)
        self.cols = np.ascontiguousarray(cols, dtype=np.int32)
        self.n = len(self.rowp) - 1
        self._h = self._lib.oref_chol_create(self.n, int(self.rowp[-1]), _ip(self.rowp),
                                             _ip(self.cols), int(sqdef_index))

    def close(self):
        if getattr(self, "_h", None):
            self._lib.oref_chol_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def factor(self, vals) -> int:
        vals = np.ascontiguousarray(vals, dtype=np.float64)
        return self._lib.oref_chol_factor(self._h, _fp(vals))

    def solve(self, b: np.ndarray) -> np.ndarray:
        """K^{-1} b for one right-hand side (1-D) or each column of a 2-D b."""
        b = np.asarray(b, dtype=np.float64)
        if b.ndim == 1:
            x = np.array(b, copy=True)
            self._lib.oref_chol_solve(self._h, _fp(x))
            return x
        return np.stack([self.solve(b[:, j]) for j in range(b.shape[1])], axis=1)


def csr_assemble(rowp, cols, groups, blocks) -> np.ndarray:
    """The reference's Hessian assembly (add_row per element column, in
    order) of the element blocks into the CSR values. groups: list of
    [nelem, ncomp] int arrays of global indices; blocks: list of
    [nelem, ncomp, ncomp] arrays, block[e, j, i] = column j, row i."""
    lib = load()
    rowp = np.ascontiguousarray(rowp, dtype=np.int32)
    cols = np.ascontiguousarray(cols, dtype=np.int32)
    n = len(rowp) - 1
    nelems = np.array([g.shape[0] for g in groups], dtype=np.int32)
    ncomp = np.array([g.shape[1] for g in groups], dtype=np.int32)
    conn = np.ascontiguousarray(np.concatenate([np.asarray(g, np.int32).ravel() for g in groups])
                                if groups else np.zeros(1, np.int32), dtype=np.int32)
    vals = np.ascontiguousarray(np.concatenate([np.asarray(b, np.float64).ravel()
                                                for b in blocks]) if blocks
                                else np.zeros(1), dtype=np.float64)
    out = np.zeros(int(rowp[-1]), dtype=np.float64)
    lib.oref_csr_assemble(n, int(rowp[-1]), _ip(rowp), _ip(cols), len(groups), _ip(nelems),
                          _ip(ncomp), _ip(conn), _fp(vals), _fp(out))
    return out
