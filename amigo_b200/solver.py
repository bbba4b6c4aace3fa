"""The Amigo linear-solver plugin backed by the B200 factorization.

``LinearSolver`` restates the reference's abstract base
(amigo/algorithm/solvers/linear_solver.py:5-35) so that this package does not
need Amigo importable. ``B200LdlSolver`` has AmigoSolver's constructor and
methods (amigo/algorithm/solvers/amigo_solver.py:11-64), so
``options["solver"] = B200LdlSolver(options, state)`` drops it into
``make_solver`` (amigo/algorithm/solvers/__init__.py:16-19) unchanged. It
works with Amigo's own CSRMat/Vector objects (host views through
``get_nonzero_structure``/``get_data``/``[:]``) and with this package's
CSRMat/Vector holding numpy arrays or torch CUDA tensors.
"""

from __future__ import annotations

from abc import ABC, abstractmethod

import numpy as np

from .sparse_ldl import OrderingType, SolverType, SparseLDL, _is_torch, _values_of

__all__ = ["LinearSolver", "B200LdlSolver"]


class LinearSolver(ABC):
    @abstractmethod
    def factor(self, hess, diag):
        return

    @abstractmethod
    def solve(self, b, x):
        return

    def inertia_enabled(self):
        return False

    def get_inertia(self):
        return None

    def set_pivot_tolerance(self, pivtol):
        pass

    @staticmethod
    def find_diag_indices(rowp, cols, nrows):
        """CSR data index of each diagonal entry (the reference helper of the
        same name, linear_solver.py:24-35)."""
        diag_idx = np.empty(nrows, dtype=np.intp)
        for i in range(nrows):
            start, end = rowp[i], rowp[i + 1]
            pos = np.searchsorted(cols[start:end], i)
            if pos < end - start and cols[start + pos] == i:
                diag_idx[i] = start + pos
            else:
                diag_idx[i] = start
        return diag_idx


class B200LdlSolver(LinearSolver):
    """AmigoSolver's contract on the GPU: symbolic analysis once for the
    Hessian's pattern (AMD, ustab 0.01, pivot_tol 1e-14), numeric
    factorization and inertia on every ``factor``, solve on the stored
    factor.

    ``reuse_pivot_order=True`` makes the factorizations after the first one
    test each candidate in the front that accepted it in a recent
    factorization (SparseLDL.reuse_pivot_order). The structure is re-planned
    before the second factorization, and again before the factorization that
    follows one which delayed more than ``refresh_delays * n`` candidates
    (the iterates moved away from the record). Every threshold test still
    applies, so the inertia is the same; the values differ in rounding.
    Off by default: every factorization then replays the reference's pivot
    sequence."""

    def __init__(self, options=None, state=None, hessian=None, ustab: float = 0.01,
                 pivot_tol: float = 1e-14, order=OrderingType.DEFAULT,
                 reuse_pivot_order: bool = False, refresh_delays: float = 0.01):
        self.options = options
        self.hessian = hessian if hessian is not None else state.hessian
        self.ldl = SparseLDL(self.hessian, SolverType.LDL, ustab=ustab, pivot_tol=pivot_tol,
                             order=order)
        self.reuse_pivot_order = bool(reuse_pivot_order)
        self.refresh_delays = float(refresh_delays)
        self._replan = False  # re-plan from the last record before the next factorization
        self._planned = False

    def _before_factor(self):
        if self._replan:
            self.ldl.reuse_pivot_order()  # drops the last factor: only right before factoring
            self._replan = False
            self._planned = True

    def _after_factor(self):
        if self.reuse_pivot_order:
            delayed = self.ldl.stats()["delayed"]
            self._replan = (not self._planned) or delayed > self.refresh_delays * self.ldl.n

    def factor(self, hessian, diagonal):
        if hessian is not self.hessian and hessian != self.hessian:
            raise ValueError("Hessian instance must be the same")
        # Amigo objects may keep the current values on the device; bring the
        # host view up to date exactly as AmigoSolver does
        if hasattr(diagonal, "copy_device_to_host"):
            diagonal.copy_device_to_host()
        if hasattr(self.hessian, "copy_data_device_to_host"):
            self.hessian.copy_data_device_to_host()
        self._before_factor()
        flag = self.ldl.factor(diagonal)
        if flag != 0:
            raise RuntimeError(f"B200LdlSolver factorization failed with flag = {flag}")
        self._after_factor()
        return flag

    def solve(self, b, x):
        bv = _values_of(b)
        if _is_torch(bv) and bv.is_cuda:
            xv = _values_of(x)
            xv.copy_(bv)
            self.ldl.solve(xv)
            return
        rhs = np.array(bv[:] if not isinstance(bv, np.ndarray) else bv, dtype=np.float64)
        self.ldl.solve(rhs)
        if hasattr(x, "copy_host_to_device") and hasattr(x, "__setitem__"):
            x[:] = rhs
            x.copy_host_to_device()
        else:
            xv = _values_of(x)
            xv[...] = rhs

    def inertia_enabled(self):
        return True

    def get_inertia(self):
        return self.ldl.get_inertia()

    def set_pivot_tolerance(self, pivtol):
        pass

    # the pivot tolerance of the threshold test is fixed at construction, as
    # in AmigoSolver (amigo_solver.py:63-64)
    uses_pivot_tolerance = False

    # -- inertia correction on the device (amigo_b200.inertia_correction) -------
    def set_perturbation_rows(self, primal, dual):
        self.ldl.set_perturbation_rows(primal, dual)

    def load_system(self, hessian, diagonal):
        """Bring the Hessian values and the diagonal to the device once for
        the attempts that follow."""
        if hessian is not self.hessian and hessian != self.hessian:
            raise ValueError("Hessian instance must be the same")
        if hasattr(diagonal, "copy_device_to_host"):
            diagonal.copy_device_to_host()
        if hasattr(self.hessian, "copy_data_device_to_host"):
            self.hessian.copy_data_device_to_host()
        self._dev = self.ldl.device_values(diagonal)

    def factor_perturbed(self, delta_x, delta_c):
        """One attempt on the loaded system; returns (npos, nneg)."""
        vals, diag = self._dev
        self._before_factor()
        out = self.ldl.factor_perturbed(delta_x, delta_c, vals, diag)
        self._after_factor()
        return out
