"""Host-side mirror of the reference's SparseLDL interface, running on the GPU.

``SparseLDL(mat, solver_type, ustab, pivot_tol, delay_growth, order)`` with
``factor(diagonal=None)``, ``solve(x)`` and ``get_inertia()`` behaves like the
pybind class of the same name (amigo/amigo.cpp:648-732 over
include/sparse_ldl.h:65-213): the symbolic phase runs on the host when the
object is built, ``factor`` returns 0, ``solve`` overwrites its argument,
``get_inertia`` returns ``(npos, nneg)``. The numeric work runs in the
sm_100a kernels of libb200ldl.so; there is no CPU path.

Accepted value containers: numpy arrays (host; copied to the device inside
the call) and torch CUDA tensors (used in place on the device).
"""

from __future__ import annotations

import ctypes
import enum

import numpy as np

from . import _native

__all__ = ["SolverType", "OrderingType", "CSRMat", "Vector", "SparseLDL", "SparseLDLBatch",
           "SparseCholesky"]


class SolverType(enum.IntEnum):
    LDL = 0
    CHOLESKY = 1


class OrderingType(enum.IntEnum):
    NESTED_DISSECTION = 0
    AMD = 1
    MULTI_COLOR = 2
    NATURAL = 3
    # our nested dissection without METIS (the reference's needs METIS and
    # is the identity without it); not one of the reference's values
    GRAPH_ND = 4
    # the reference's DEFAULT without METIS (amigo/amigo.cpp:329-333)
    DEFAULT = 1


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


class CSRMat:
    """Symmetric CSR matrix (full pattern), as amigo.CSRMat's constructor
    ``CSRMat(nrows, ncols, rowp, cols, vals)`` (amigo/amigo.cpp:346-381).
    ``vals`` may be a numpy array or a torch CUDA tensor."""

    def __init__(self, nrows, ncols, rowp, cols, vals=None):
        self.nrows = int(nrows)
        self.ncols = int(ncols)
        self.rowp = np.ascontiguousarray(rowp, dtype=np.int32)
        self.cols = np.ascontiguousarray(cols, dtype=np.int32)
        if self.rowp.shape != (self.nrows + 1,):
            raise RuntimeError("rowp must have length nrows + 1")
        nnz = int(self.rowp[-1])
        if vals is None:
            vals = np.zeros(nnz)
        if not _is_torch(vals):
            vals = np.ascontiguousarray(vals, dtype=np.float64)
        if len(self.cols) != nnz or vals.shape[0] != nnz:
            raise RuntimeError("cols and vals must have the same length")
        self.vals = vals

    @property
    def nnz(self) -> int:
        return int(self.rowp[-1])

    def get_nonzero_structure(self):
        return self.nrows, self.ncols, self.nnz, self.rowp.copy(), self.cols.copy()

    def get_data(self):
        return self.vals


class Vector:
    """Minimal stand-in for amigo.Vector: a length-n float64 array (numpy or a
    torch CUDA tensor) with item access."""

    def __init__(self, n_or_array):
        if isinstance(n_or_array, (int, np.integer)):
            self.array = np.zeros(int(n_or_array))
        else:
            self.array = n_or_array

    def get_size(self) -> int:
        return int(self.array.shape[0])

    def get_array(self):
        return self.array

    def __getitem__(self, i):
        return self.array[i]

    def __setitem__(self, i, v):
        self.array[i] = v


def _values_of(obj):
    """numpy/torch array behind a CSRMat, Vector, amigo object or array."""
    if obj is None:
        return None
    if isinstance(obj, CSRMat):
        return obj.vals
    if isinstance(obj, Vector):
        return obj.array
    if hasattr(obj, "get_data") and not isinstance(obj, np.ndarray) and not _is_torch(obj):
        return np.asarray(obj.get_data())  # amigo.CSRMat (host view)
    if hasattr(obj, "get_size") and hasattr(obj, "__getitem__") and not _is_torch(obj) \
            and not isinstance(obj, np.ndarray):
        return np.asarray(obj[:], dtype=np.float64)  # amigo.Vector
    return obj


class SparseLDL:
    """GPU multifrontal LDL^T with the reference SparseLDL's interface."""

    def __init__(self, mat, solver_type=SolverType.LDL, ustab: float = 0.01,
                 pivot_tol: float = 1e-14, delay_growth: float = 2.0,
                 order=OrderingType.NATURAL):
        self._lib = _native.load()
        if isinstance(mat, CSRMat):
            rowp, cols = mat.rowp, mat.cols
            n = mat.nrows
        else:  # an amigo.CSRMat
            n, _, _, rowp, cols = mat.get_nonzero_structure()
        self.mat = mat
        self.n = int(n)
        self.rowp = np.ascontiguousarray(rowp, dtype=np.int32)
        self.cols = np.ascontiguousarray(cols, dtype=np.int32)
        self.nnz = int(self.rowp[-1])
        self.solver_type = SolverType(int(solver_type))
        self.order = int(order)
        h = ctypes.c_void_p()
        st = self._lib.b200ldl_create(
            ctypes.byref(h), self.n, self.nnz,
            self.rowp.ctypes.data_as(_native._i32p), self.cols.ctypes.data_as(_native._i32p),
            int(self.solver_type), float(ustab), float(pivot_tol), float(delay_growth),
            self.order)
        if st != 0:
            raise _native.NativeError(f"b200ldl_create failed with status {st}", st)
        self._h = h
        self._keep = []

    # -- lifetime -----------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._lib.b200ldl_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- numeric phase -------------------------------------------------------
    def factor(self, diagonal=None) -> int:
        vals = _values_of(self.mat)
        diag = _values_of(diagonal)
        if _is_torch(vals):
            import torch

            if not vals.is_cuda:
                vals = vals.numpy()
            else:
                vals = vals.contiguous().to(torch.float64)
                if diag is not None:
                    if not _is_torch(diag):
                        diag = torch.as_tensor(np.asarray(diag, np.float64), device=vals.device)
                    diag = diag.contiguous().to(device=vals.device, dtype=torch.float64)
                self._keep = [vals, diag]
                self._sync_stream(vals)
                st = self._lib.b200ldl_factor(
                    self._h, ctypes.c_void_p(vals.data_ptr()),
                    ctypes.c_void_p(diag.data_ptr()) if diag is not None else None)
                return _native.check(self._h, st, "factor")
        v = np.ascontiguousarray(vals, dtype=np.float64)
        d = None if diag is None else np.ascontiguousarray(
            diag.cpu().numpy() if _is_torch(diag) else diag, dtype=np.float64)
        st = self._lib.b200ldl_factor_host(
            self._h, v.ctypes.data_as(_native._f64p),
            d.ctypes.data_as(_native._f64p) if d is not None else None)
        return _native.check(self._h, st, "factor")

    def factor_elements(self, assembly, blocks, diagonal=None) -> int:
        """Factor from the element Hessian blocks through ``assembly`` (an
        amigo_b200.assembly.CSRAssembly of this pattern) without forming the
        CSR values: each front reads its entries as sums of their element
        contributions, in the order CSRAssembly.values sums them, so the
        factorization is the one of ``factor`` after ``values``. ``blocks``
        as CSRAssembly.values takes them; CUDA tensors."""
        import torch

        if isinstance(blocks, (list, tuple)):
            blocks = torch.cat([b.reshape(-1) for b in blocks])
        if not (torch.is_tensor(blocks) and blocks.is_cuda and blocks.dtype == torch.float64):
            raise TypeError("blocks must be a float64 CUDA tensor")
        blocks = blocks.contiguous().reshape(-1)
        if blocks.numel() != assembly.nvals:
            raise ValueError(f"expected {assembly.nvals} block values, got {blocks.numel()}")
        diag = _values_of(diagonal)
        if diag is not None:
            if not _is_torch(diag):
                diag = torch.as_tensor(np.asarray(diag, np.float64), device=blocks.device)
            diag = diag.contiguous().to(device=blocks.device, dtype=torch.float64)
        self._keep = [blocks, diag]
        self._sync_stream(blocks)
        st = self._lib.b200ldl_factor_elements(
            self._h, assembly._h, ctypes.c_void_p(blocks.data_ptr()),
            ctypes.c_void_p(diag.data_ptr()) if diag is not None else None)
        return _native.check(self._h, st, "factor_elements")

    def _sync_stream(self, t):
        import torch

        stream = torch.cuda.current_stream(t.device)
        self._lib.b200ldl_set_stream(self._h, ctypes.c_void_p(stream.cuda_stream))

    def solve(self, x):
        """Overwrite x (Vector, numpy 1D/2D, or torch CUDA tensor 1D/2D with
        the n rows first) with K^{-1} x."""
        arr = _values_of(x)
        if _is_torch(arr) and arr.is_cuda:
            import torch

            if arr.dtype != torch.float64:
                raise TypeError("solve needs float64")
            nrhs = 1 if arr.dim() == 1 else arr.shape[1]
            if arr.dim() == 1:
                work = arr if arr.is_contiguous() else arr.contiguous()
                ldx = self.n
            else:
                # column-major n x nrhs == row-major nrhs x n
                if arr.stride(0) == 1 and arr.stride(1) >= self.n:
                    work = arr
                    ldx = arr.stride(1)
                else:
                    work = arr.t().contiguous().t()
                    ldx = self.n
            self._sync_stream(work)
            st = self._lib.b200ldl_solve(self._h, nrhs, ctypes.c_void_p(work.data_ptr()), ldx)
            _native.check(self._h, st, "solve")
            if work.data_ptr() != arr.data_ptr():
                arr.copy_(work)
            return None
        a = np.asarray(arr)
        if a.dtype != np.float64:
            raise TypeError("NumPy array must have dtype=float64")
        nrhs = 1 if a.ndim == 1 else a.shape[1]
        f = np.asfortranarray(a)
        st = self._lib.b200ldl_solve_host(self._h, nrhs, f.ctypes.data_as(_native._f64p),
                                          self.n)
        _native.check(self._h, st, "solve")
        if not np.shares_memory(f, a):
            a[...] = f
        if isinstance(x, Vector) and x.array is not a:
            x.array[...] = a
        elif not isinstance(x, (np.ndarray, Vector)) and hasattr(x, "__setitem__"):
            x[:] = a
        return None

    def solve_refine(self, b, max_iter: int = 5, tol: float = 1e-12, diagonal=None):
        """x = K^-1 b with FP64 iterative refinement against the CSR values
        (device path: ``b`` a torch CUDA tensor, [n] or [n, k] with the n
        rows first). Returns (x, berr per column, corrections used)."""
        import torch

        vals = _values_of(self.mat)
        diag = _values_of(diagonal)
        if not (_is_torch(vals) and vals.is_cuda):
            raise TypeError("solve_refine needs the CSR values on the GPU (torch CUDA tensor)")
        dev = vals.device
        bb = b if b.dim() == 2 else b.unsqueeze(1)
        bcm = bb.t().contiguous().t()  # column-major copy
        x = torch.empty_like(bcm)
        x = x.t().contiguous().t()
        nrhs = bcm.shape[1]
        d = None
        if diag is not None:
            d = diag if _is_torch(diag) else torch.as_tensor(np.asarray(diag), device=dev)
            d = d.contiguous().to(device=dev, dtype=torch.float64)
        berr = np.zeros(nrhs)
        iters = ctypes.c_int()
        self._sync_stream(vals)
        st = self._lib.b200ldl_solve_refine(
            self._h, ctypes.c_void_p(vals.data_ptr()),
            ctypes.c_void_p(d.data_ptr()) if d is not None else None, nrhs,
            ctypes.c_void_p(bcm.data_ptr()), bcm.stride(1), ctypes.c_void_p(x.data_ptr()),
            x.stride(1), int(max_iter), float(tol), berr.ctypes.data_as(_native._f64p),
            ctypes.byref(iters))
        _native.check(self._h, st, "solve_refine")
        out = x if b.dim() == 2 else x[:, 0]
        return out, berr, iters.value

    def value_gradient(self, lam, x):
        """Derivatives of a scalar loss through x = K^{-1} b, given the
        solution ``x`` and the adjoint ``lam = K^{-1} dloss/dx`` (torch CUDA
        float64 tensors, [n] or [n, k] with k <= 8): returns ``(gvals,
        gdiag)`` with gvals[e] = -sum_r lam[i, r] x[j, r] for each stored
        entry e = (i, j) and gdiag[i] = -sum_r lam[i, r] x[i, r]."""
        import torch

        lam2 = lam if lam.dim() == 2 else lam.unsqueeze(1)
        x2 = x if x.dim() == 2 else x.unsqueeze(1)
        lcm = lam2.t().contiguous()  # rows of the transposed copy: column-major n x k
        xcm = x2.t().contiguous()
        k = lcm.shape[0]
        gvals = torch.empty(self.nnz, dtype=torch.float64, device=lam.device)
        gdiag = torch.empty(self.n, dtype=torch.float64, device=lam.device)
        self._sync_stream(lcm)
        st = self._lib.b200ldl_value_gradient(
            self._h, k, ctypes.c_void_p(lcm.data_ptr()), self.n, ctypes.c_void_p(xcm.data_ptr()),
            self.n, ctypes.c_void_p(gvals.data_ptr()), ctypes.c_void_p(gdiag.data_ptr()))
        _native.check(self._h, st, "value_gradient")
        return gvals, gdiag

    # -- inertia correction -----------------------------------------------------
    def set_perturbation_rows(self, primal, dual):
        """Rows that take +delta_x (primal) and -delta_c (constraints) in
        :meth:`factor_perturbed`: the index sets of
        problem.get_primal_indices / get_constraint_indices
        (amigo/algorithm/solvers/inertia_correction.py:280-293)."""
        p = np.ascontiguousarray(np.asarray(primal).ravel(), dtype=np.int32)
        d = np.ascontiguousarray(np.asarray(dual).ravel(), dtype=np.int32)
        st = self._lib.b200ldl_set_perturbation_rows(
            self._h, len(p), p.ctypes.data_as(_native._i32p), len(d),
            d.ctypes.data_as(_native._i32p))
        _native.check(self._h, st, "set_perturbation_rows")

    def device_values(self, diagonal=None):
        """The CSR values and the diagonal as float64 CUDA tensors (uploaded
        when they are host arrays), for repeated :meth:`factor_perturbed`
        attempts on one system."""
        import torch

        vals = _values_of(self.mat)
        diag = _values_of(diagonal)
        dev = vals.device if _is_torch(vals) and vals.is_cuda else torch.device("cuda")
        v = torch.as_tensor(np.asarray(vals) if not _is_torch(vals) else vals, device=dev)
        v = v.to(torch.float64).contiguous()
        d = None
        if diag is not None:
            d = torch.as_tensor(np.asarray(diag) if not _is_torch(diag) else diag, device=dev)
            d = d.to(torch.float64).contiguous()
        return v, d

    def factor_perturbed(self, delta_x: float, delta_c: float, vals=None, diag=None):
        """One inertia-correction attempt: factor K + diag(diag + delta_x on
        the primal rows - delta_c on the constraint rows), the perturbed
        diagonal formed on the device, and return the inertia (npos, nneg).
        ``vals``/``diag`` are CUDA tensors from :meth:`device_values` (by
        default the matrix's own values and no diagonal)."""
        if vals is None:
            vals, diag = self.device_values(diag)
        self._keep = [vals, diag]
        self._sync_stream(vals)
        p = ctypes.c_int()
        q = ctypes.c_int()
        st = self._lib.b200ldl_factor_perturbed(
            self._h, ctypes.c_void_p(vals.data_ptr()),
            ctypes.c_void_p(diag.data_ptr()) if diag is not None else None,
            float(delta_x), float(delta_c), ctypes.byref(p), ctypes.byref(q))
        _native.check(self._h, st, "factor_perturbed")
        return p.value, q.value

    def perturbed_diagonal(self):
        """The diagonal of the last :meth:`factor_perturbed` (a CUDA tensor)."""
        import torch

        out = torch.empty(self.n, dtype=torch.float64, device="cuda")
        if self._keep and self._keep[0] is not None:
            out = out.to(self._keep[0].device)
            self._sync_stream(out)
        st = self._lib.b200ldl_copy_perturbed_diagonal(self._h, ctypes.c_void_p(out.data_ptr()))
        _native.check(self._h, st, "perturbed_diagonal")
        return out

    def get_inertia(self):
        p = ctypes.c_int()
        q = ctypes.c_int()
        st = self._lib.b200ldl_get_inertia(self._h, ctypes.byref(p), ctypes.byref(q))
        _native.check(self._h, st, "get_inertia")
        if self.solver_type == SolverType.CHOLESKY:
            return (0, 0)
        return (p.value, q.value)

    # -- introspection used by the parity tests --------------------------------
    def symbolic(self) -> dict:
        nn = ctypes.c_int()
        nc = ctypes.c_int()
        self._lib.b200ldl_symbolic_sizes(self._h, ctypes.byref(nn), ctypes.byref(nc))
        nn, nc = nn.value, nc.value
        out = {
            "invperm": np.empty(self.n, np.int32),
            "node_ptr": np.empty(nn + 1, np.int32),
            "node_to_var": np.empty(self.n, np.int32),
            "children_ptr": np.empty(nn + 2, np.int32),
            "children": np.empty(max(nn, 1), np.int32),
            "contrib_ptr": np.empty(nn + 1, np.int32),
            "contrib_rows": np.empty(max(nc, 1), np.int32),
        }
        keys = ("invperm", "node_ptr", "node_to_var", "children_ptr", "children",
                "contrib_ptr", "contrib_rows")
        self._lib.b200ldl_get_symbolic(self._h, *[out[k].ctypes.data_as(_native._i32p)
                                                  for k in keys])
        out["children"] = out["children"][:nn]
        out["contrib_rows"] = out["contrib_rows"][:nc]
        return out

    def node_pivots(self):
        nn = len(self.symbolic()["node_ptr"]) - 1
        a = np.empty(nn, np.int32)
        b = np.empty(nn, np.int32)
        st = self._lib.b200ldl_node_pivots(self._h, a.ctypes.data_as(_native._i32p),
                                           b.ctypes.data_as(_native._i32p))
        _native.check(self._h, st, "node_pivots")
        return a, b

    # -- precision -------------------------------------------------------------------
    def set_precision(self, mode: str = "fp64", refine_iters: int = 5, refine_tol: float = 1e-12):
        """``"fp64"`` (the default) or ``"mixed"``: after pivot-order reuse, the
        contribution-block tiles of the big fronts' trailing updates run on
        the tensor cores with about FP32 accuracy, and every solve is refined
        in FP64 against the factored matrix (at most ``refine_iters``
        corrections, until the backward error is <= ``refine_tol``)."""
        code = {"fp64": 0, "mixed": 1}[mode]
        _native.check(self._h, self._lib.b200ldl_set_precision(self._h, code), "set_precision")
        _native.check(self._h, self._lib.b200ldl_set_refinement(self._h, int(refine_iters),
                                                                float(refine_tol)),
                      "set_refinement")

    def last_refinement(self) -> dict:
        """Corrections and largest backward error of the last refined solve,
        whether the factor in use ran mixed-precision tiles, and how many
        factorizations the mixed-precision checks redid in FP64."""
        it = ctypes.c_int()
        be = ctypes.c_double()
        mx = ctypes.c_int()
        fb = ctypes.c_int()
        self._lib.b200ldl_last_refinement(self._h, ctypes.byref(it), ctypes.byref(be),
                                          ctypes.byref(mx), ctypes.byref(fb))
        return {"iterations": it.value, "backward_error": be.value, "mixed": bool(mx.value),
                "fp64_redos": fb.value}

    # -- pivot-order reuse --------------------------------------------------------
    def pivot_record(self) -> dict:
        """The last factorization's pivot record: per supernode the front size
        ``f``, pivots ``npiv`` and delayed candidates ``ndel``, and ``fv``,
        each front's variables after pivoting (pivots in elimination order
        with 2x2 pairs encoded -(v+1), delayed, contribution rows)."""
        nn = len(self.symbolic()["node_ptr"]) - 1
        total = ctypes.c_longlong()
        st = self._lib.b200ldl_get_pivot_record(self._h, None, None, None, None,
                                                ctypes.byref(total))
        _native.check(self._h, st, "get_pivot_record")
        rec = {k: np.empty(max(nn, 1), np.int32) for k in ("f", "npiv", "ndel")}
        rec["fv"] = np.empty(max(total.value, 1), np.int32)
        st = self._lib.b200ldl_get_pivot_record(
            self._h, *[rec[k].ctypes.data_as(_native._i32p) for k in ("f", "npiv", "ndel", "fv")],
            ctypes.byref(total))
        _native.check(self._h, st, "get_pivot_record")
        return {"f": rec["f"][:nn], "npiv": rec["npiv"][:nn], "ndel": rec["ndel"][:nn],
                "fv": rec["fv"][:total.value]}

    def set_pivot_record(self, rec=None):
        """Re-plan the fronts from a pivot record (``pivot_record()`` of any
        factorization of this pattern): each candidate is then tested first
        in the front that accepted it. ``None`` returns to the reference's
        symbolic structure. Factor again before solving."""
        if rec is None:
            st = self._lib.b200ldl_set_pivot_record(self._h, None, None, None, None)
        else:
            arrs = [np.ascontiguousarray(rec[k], np.int32) for k in ("f", "npiv", "ndel", "fv")]
            st = self._lib.b200ldl_set_pivot_record(
                self._h, *[a.ctypes.data_as(_native._i32p) for a in arrs])
        _native.check(self._h, st, "set_pivot_record")

    def reuse_pivot_order(self):
        """Re-plan the fronts from the last factorization's own pivot record
        (the pattern's next factorizations, e.g. the next interior-point
        iterations, then test each candidate where it was accepted)."""
        st = self._lib.b200ldl_reuse_pivot_order(self._h)
        _native.check(self._h, st, "reuse_pivot_order")

    # -- profiling ---------------------------------------------------------------
    PHASES =("fronts", "big_assembly", "big_panel", "big_update", "solve_forward",
              "solve_backward", "cluster_fronts")

    def set_profiling(self, on: bool):
        self._lib.b200ldl_set_profiling(self._h, 1 if on else 0)

    def reset_profile(self):
        self._lib.b200ldl_reset_profile(self._h)

    def launch_count(self) -> int:
        return int(self._lib.b200ldl_launch_count(self._h))

    def work(self) -> dict:
        v = np.zeros(8)
        self._lib.b200ldl_work(self._h, v.ctypes.data_as(_native._f64p), 8)
        return {"flops": v[0], "panel_flops": v[1], "update_flops": v[2], "update_bytes": v[3],
                "cluster_flops": v[4], "app_panels": int(v[5]), "app_rejected": int(v[6]),
                "app_block_delays": int(v[7])}

    def profile(self) -> list:
        """Per kernel class: device milliseconds (CUDA events), launches, and
        the algorithmic work used for its roofline: flops for the front and
        panel kernels (compute), bytes for the update and solve kernels."""
        v = np.zeros(2 * len(self.PHASES))
        self._lib.b200ldl_profile(self._h, v.ctypes.data_as(_native._f64p), len(v))
        return [{"name": nm, "ms": float(v[2 * i]), "launches": int(v[2 * i + 1])}
                for i, nm in enumerate(self.PHASES)]

    def stats(self) -> dict:
        v = np.zeros(6)
        st = self._lib.b200ldl_stats(self._h, v.ctypes.data_as(_native._f64p), 6)
        _native.check(self._h, st, "stats")
        return {"flops": v[0], "L_bytes": v[1], "cb_bytes": v[2], "max_front": int(v[3]),
                "delayed": int(v[4]), "levels": int(v[5])}


class SparseCholesky:
    """The reference's SparseCholesky interface (include/sparse_cholesky.h:
    64-375, bound at amigo/amigo.cpp:641-646) on the GPU factorization.

    The reference factors a symmetric quasi-definite matrix
    [[A, B^T], [B, -C]] (A, C positive definite; the first ``sqdef_index``
    rows are A's) in natural order as L L^T over A and -F F^T over the
    Schur complement of C. A quasi-definite matrix has an LDL^T
    factorization with 1x1 pivots under every symmetric permutation, so
    here the threshold test is off (ustab = 0: every pivot is accepted where
    it stands, so nothing is delayed; fronts without contribution rows keep
    Bunch-Kaufman) and the rows are ordered by AMD for less fill. The solution is
    the same; the factor differs from the reference's only by that
    ordering and the scaling of L by sqrt|D|.

    ``factor()`` returns 0, or 1 when the signs of the pivots do not match
    the quasi-definite structure (the reference returns the failing
    Cholesky factorization's flag there). ``solve(x)`` overwrites x with
    K^{-1} x.
    """

    def __init__(self, mat, sqdef_index: int | None = None, order=OrderingType.AMD,
                 pivot_tol: float = 1e-14):
        if sqdef_index is None and hasattr(mat, "get_sqdef_index"):
            sqdef_index = mat.get_sqdef_index()
        self.ldl = SparseLDL(mat, SolverType.LDL, ustab=0.0, pivot_tol=pivot_tol, order=order)
        n = self.ldl.n
        self.sqdef_index = n if sqdef_index is None or not 0 <= sqdef_index <= n \
            else int(sqdef_index)

    def factor(self) -> int:
        self.ldl.factor(None)
        npos, nneg = self.ldl.get_inertia()
        return 0 if (npos, nneg) == (self.sqdef_index, self.ldl.n - self.sqdef_index) else 1

    def solve(self, x):
        self.ldl.solve(x)

    def get_inertia(self):
        return self.ldl.get_inertia()


class SparseLDLBatch(SparseLDL):
    """Many independent symmetric systems factored and solved together.

    ``SparseLDLBatch(mats, ...)`` takes a list of CSRMat (each with its own
    pattern, size and values). Every system gets the symbolic phase it would
    get alone in ``SparseLDL``; the numeric factorization and the solves run
    all systems' supernodes level by level in the same launches. Vectors
    (diagonals, right-hand sides, solutions) are the systems' vectors
    concatenated in order; ``offsets[s]:offsets[s+1]`` is system s.
    """

    def __init__(self, mats, solver_type=SolverType.LDL, ustab: float = 0.01,
                 pivot_tol: float = 1e-14, delay_growth: float = 2.0,
                 order=OrderingType.NATURAL):
        self._lib = _native.load()
        self.mats = list(mats)
        if not self.mats:
            raise ValueError("no systems")
        sys_n = np.array([m.nrows for m in self.mats], dtype=np.int32)
        sys_nnz = np.array([int(m.rowp[-1]) for m in self.mats], dtype=np.int32)
        rowp_cat = np.ascontiguousarray(np.concatenate([m.rowp for m in self.mats]),
                                        dtype=np.int32)
        cols_cat = np.ascontiguousarray(np.concatenate([m.cols for m in self.mats]),
                                        dtype=np.int32)
        self.offsets = np.concatenate([[0], np.cumsum(sys_n)]).astype(np.int64)
        self.val_offsets = np.concatenate([[0], np.cumsum(sys_nnz)]).astype(np.int64)
        self.n = int(self.offsets[-1])
        self.nnz = int(self.val_offsets[-1])
        self.solver_type = SolverType(int(solver_type))
        self.order = int(order)
        h = ctypes.c_void_p()
        st = self._lib.b200ldl_create_batch(
            ctypes.byref(h), len(self.mats), sys_n.ctypes.data_as(_native._i32p),
            sys_nnz.ctypes.data_as(_native._i32p), rowp_cat.ctypes.data_as(_native._i32p),
            cols_cat.ctypes.data_as(_native._i32p), int(self.solver_type), float(ustab),
            float(pivot_tol), float(delay_growth), self.order)
        if st != 0:
            raise _native.NativeError(f"b200ldl_create_batch failed with status {st}", st)
        self._h = h
        self._keep = []
        # the block-diagonal pattern, as one CSRMat for the inherited methods
        rowp_all = np.zeros(self.n + 1, dtype=np.int32)
        cols_all = np.empty(self.nnz, dtype=np.int32)
        for i, m in enumerate(self.mats):
            o, vo = int(self.offsets[i]), int(self.val_offsets[i])
            rowp_all[o + 1:o + m.nrows + 1] = vo + m.rowp[1:]
            cols_all[vo:vo + int(m.rowp[-1])] = o + m.cols
        self.rowp, self.cols = rowp_all, cols_all
        self.mat = CSRMat(self.n, self.n, rowp_all, cols_all, self._gather_values())

    @property
    def num_systems(self) -> int:
        return len(self.mats)

    def _gather_values(self):
        vals = [_values_of(m) for m in self.mats]
        if any(_is_torch(v) and v.is_cuda for v in vals):
            import torch

            dev = next(v.device for v in vals if _is_torch(v) and v.is_cuda)
            return torch.cat([torch.as_tensor(v, dtype=torch.float64, device=dev) for v in vals])
        return np.concatenate([np.asarray(v.cpu().numpy() if _is_torch(v) else v, np.float64)
                               for v in vals])

    def factor(self, diagonal=None, values=None) -> int:
        """Factor every system with its current values, or with ``values``
        (the systems' values concatenated) when given; ``diagonal`` is the
        concatenated diagonal vector (or a list of per-system vectors)."""
        self.mat.vals = self._gather_values() if values is None else values
        if isinstance(diagonal, (list, tuple)):
            parts = [_values_of(d) for d in diagonal]
            if any(_is_torch(d) for d in parts):
                import torch

                diagonal = torch.cat([torch.as_tensor(d, dtype=torch.float64) for d in parts])
            else:
                diagonal = np.concatenate([np.asarray(d, np.float64) for d in parts])
        return super().factor(diagonal)

    def system_inertia(self) -> list:
        ns = len(self.mats)
        p = np.zeros(ns, np.int32)
        q = np.zeros(ns, np.int32)
        st = self._lib.b200ldl_system_inertia(self._h, p.ctypes.data_as(_native._i32p),
                                              q.ctypes.data_as(_native._i32p))
        _native.check(self._h, st, "system_inertia")
        return [(int(a), int(b)) for a, b in zip(p, q)]

    def split(self, x):
        """Per-system views of a concatenated vector or [n, k] array."""
        return [x[int(self.offsets[i]):int(self.offsets[i + 1])] for i in range(len(self.mats))]
