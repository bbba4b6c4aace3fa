"""Inertia correction of the KKT system on the B200 factorization.

The interior-point loop needs ``n_primal`` positive and ``n_dual`` negative
eigenvalues. When the factorization reports another inertia it refactors
with a larger primal shift ``delta_w`` and/or a constraint shift
``delta_c``. These are Algorithm IC of Waechter and Biegler (2006, Table 3)
and its degeneracy detection, as amigo's ``InertiaCorrector`` implements
them (amigo/algorithm/solvers/inertia_correction.py:11-395). The sequence of
shifts is the contract: the interior-point step depends on which shift
succeeds. So this class takes the same decisions in the same order. It has
the same constructor, ``factor_for_inertia`` and ``last_delta_w`` /
``last_delta_c``, so it drops in where the reference's class is used.

With a solver that has ``factor_perturbed`` (``B200LdlSolver``), an attempt
never leaves the device. The Hessian values and the diagonal are uploaded
once per system. The shifted diagonal is formed by a kernel, and only the
two inertia counts come back. An attempt whose shifts equal those of the
previous attempt is not refactored when the solver ignores the pivot
tolerance (as AmigoSolver does, amigo_solver.py:63-64). The factorization is
deterministic, so the counts are the same. Any other solver is driven
through ``solver.factor(hessian, perturbed_diagonal)``, as the reference
drives it.
"""

from __future__ import annotations

import enum

import numpy as np

__all__ = ["InertiaCorrector"]


class _Degen(enum.IntEnum):
    """Structural degeneracy of the Hessian or the Jacobian."""

    UNKNOWN = 0
    NO = 1
    YES = 2


class _Trial(enum.IntEnum):
    """Which shifts the current system has tried during the degeneracy test
    (dc: constraint shift on/off, dx: primal shift on/off)."""

    NONE = 0
    DC0_DX0 = 1
    DC1_DX0 = 2
    DC0_DX1 = 3
    DC1_DX1 = 4


def _index_array(obj) -> np.ndarray:
    if isinstance(obj, np.ndarray):
        return obj.astype(np.int32, copy=False)
    if hasattr(obj, "cpu"):  # torch
        return obj.cpu().numpy().astype(np.int32)
    if hasattr(obj, "get_size"):  # amigo.Vector<int>
        return np.asarray(obj[:], dtype=np.int32)
    return np.asarray(obj, dtype=np.int32)


class InertiaCorrector:
    """Algorithm IC with structural-degeneracy detection. The constants are
    the paper's Table 3 values the reference uses (inertia_correction.py:
    66-75, 85-86)."""

    # Table 3 of Waechter & Biegler
    DW_FIRST = 1e-4       # first primal shift
    DW_MIN = 1e-20        # smallest primal shift
    DW_MAX = 1e20         # largest primal shift
    INC = 8.0             # growth of the primal shift
    INC_FIRST = 100.0     # growth while far from the last successful shift
    DEC = 1.0 / 3         # decay from the last successful shift
    DC_VALUE = 1e-8       # constraint shift = DC_VALUE * mu ** DC_EXPONENT
    DC_EXPONENT = 0.25
    DEGEN_ITERS = 3       # systems before declaring structural degeneracy
    PIVTOL_MAX = 0.1

    def __init__(self, options, problem, optimizer):
        self.options = options
        self.problem = problem
        self.optimizer = optimizer
        self.num_primal = optimizer.get_num_primals()
        self.num_dual = optimizer.get_num_constraints()
        self.perturbed_diagonal = problem.create_vector()
        self.max_corrections = 10
        self.numerical_eps = 1e-12
        # shifts: current attempt and last successful system
        self._dw = 0.0
        self._dc = 0.0
        self._dw_prev = 0.0
        self._dc_prev = 0.0
        self.last_delta_w = 0.0
        self.last_delta_c = 0.0
        self._hess = _Degen.UNKNOWN
        self._jac = _Degen.UNKNOWN
        self._degen_count = 0
        self._trial = _Trial.NONE
        self._pivtol = 1e-6
        self.verbose = options["verbose_barrier"]
        self._rows_set_for = None  # solver whose perturbation rows are set
        self.attempts = 0  # attempts taken by the last factor_for_inertia
        self.factorizations = 0  # of which refactored

    # -- the shift schedule ---------------------------------------------------
    def _dc_for(self, state) -> float:
        return self.DC_VALUE * state.mu**self.DC_EXPONENT

    def _raise_dw(self) -> bool:
        """Next primal shift. False (and the shift left unchanged) when it
        would exceed DW_MAX; the remembered shift is then forgotten."""
        old = self._dw
        if old == 0.0:
            new = self.DW_FIRST if self._dw_prev == 0.0 else max(self.DW_MIN,
                                                                 self._dw_prev * self.DEC)
        elif self._dw_prev == 0.0 or 1e5 * self._dw_prev < old:
            new = old * self.INC_FIRST
        else:
            new = old * self.INC
        if new > self.DW_MAX:
            self._dw = old
            self._dw_prev = 0.0
            return False
        self._dw = new
        return True

    # -- degeneracy bookkeeping --------------------------------------------------
    def _close_trial(self):
        """A system factored with the right inertia (or a new system begins):
        conclude what the trial shows about degeneracy."""
        t = self._trial
        if t == _Trial.NONE:
            return
        if t == _Trial.DC0_DX0:
            # no shift was needed: neither block is degenerate
            if self._hess == _Degen.UNKNOWN:
                self._hess = _Degen.NO
            if self._jac == _Degen.UNKNOWN:
                self._jac = _Degen.NO
        elif t == _Trial.DC1_DX0:
            # the constraint shift alone was enough
            if self._hess == _Degen.UNKNOWN:
                self._hess = _Degen.NO
            if self._jac == _Degen.UNKNOWN:
                self._degen_count += 1
                if self._degen_count >= self.DEGEN_ITERS:
                    self._jac = _Degen.YES
        elif t == _Trial.DC0_DX1:
            # the primal shift alone was enough
            if self._jac == _Degen.UNKNOWN:
                self._jac = _Degen.NO
            if self._hess == _Degen.UNKNOWN:
                self._degen_count += 1
                if self._degen_count >= self.DEGEN_ITERS:
                    self._hess = _Degen.YES
        else:  # both shifts
            self._degen_count += 1
            if self._degen_count >= self.DEGEN_ITERS:
                self._hess = _Degen.YES
                self._jac = _Degen.YES
        self._trial = _Trial.NONE

    def _new_system(self, state):
        self._close_trial()
        if self._dw > 0.0:
            self._dw_prev = self._dw
        if self._dc > 0.0:
            self._dc_prev = self._dc
        testing = self._hess == _Degen.UNKNOWN or self._jac == _Degen.UNKNOWN
        self._trial = _Trial.DC0_DX0 if testing else _Trial.NONE
        self._dc = self._dc_for(state) if self._jac == _Degen.YES else 0.0
        self._dw = 0.0
        if self._hess == _Degen.YES:
            self._raise_dw()

    # -- responses to a wrong inertia ----------------------------------------------
    def _too_many_negative(self, state) -> bool:
        self._close_trial()
        if self._raise_dw():
            return True
        if self._dc != 0.0:
            return False
        # the primal shift ran out: add the constraint shift and start over
        self._dc = self._dc_for(state)
        self._dw = 0.0
        if self._hess == _Degen.YES:
            self._hess = _Degen.UNKNOWN
        self._trial = _Trial.NONE
        return self._raise_dw()

    def _too_few_negative(self, state) -> bool:
        """Treat the system as singular."""
        if self._hess != _Degen.UNKNOWN and self._jac != _Degen.UNKNOWN:
            if self._dc > 0.0:
                return self._raise_dw()
            self._dc = self._dc_for(state)
            return True
        t = self._trial
        if t == _Trial.DC0_DX0:
            if self._jac == _Degen.UNKNOWN:
                self._dc = self._dc_for(state)
                self._trial = _Trial.DC1_DX0
                return True
            if not self._raise_dw():
                return False
            self._trial = _Trial.DC0_DX1
        elif t == _Trial.DC1_DX0:
            self._dc = 0.0
            if not self._raise_dw():
                return False
            self._trial = _Trial.DC0_DX1
        elif t == _Trial.DC0_DX1:
            self._dc = self._dc_for(state)
            if not self._raise_dw():
                return False
            self._trial = _Trial.DC1_DX1
        elif t == _Trial.DC1_DX1:
            if not self._raise_dw():
                return False
        return True

    def _sharpen_pivoting(self, solver) -> bool:
        if self._pivtol >= self.PIVTOL_MAX:
            return False
        self._pivtol = min(self.PIVTOL_MAX, self._pivtol**0.5)
        solver.set_pivot_tolerance(self._pivtol)
        return True

    # -- factorization ------------------------------------------------------------
    def _inertia_ok(self, npos: int, nneg: int) -> bool:
        tol = self.options["inertia_tolerance"]
        return (abs(npos - self.num_primal) <= tol and abs(nneg - self.num_dual) <= tol
                and npos + nneg >= self.num_primal + self.num_dual - tol)

    def _shifted_host_diagonal(self, diagonal, out):
        """out = diagonal + (eps + delta_w) on primal rows - delta_c on
        constraint rows, with the reference's Vector operations."""
        primal = self.problem.get_primal_indices()
        dual = self.problem.get_constraint_indices()
        dx = self.numerical_eps + self._dw
        if hasattr(out, "add_scalar_at"):
            out.copy(diagonal)
            if dx > 0:
                out.add_scalar_at(primal, dx)
            if self._dc > 0:
                out.add_scalar_at(dual, -self._dc)
            return out
        arr = np.array(np.asarray(diagonal), dtype=np.float64)
        if dx > 0:
            arr[_index_array(primal)] += dx
        if self._dc > 0:
            arr[_index_array(dual)] += -self._dc
        return arr

    def _device_solver(self, solver) -> bool:
        return hasattr(solver, "factor_perturbed")

    def factor_for_inertia(self, solver, evaluator, state) -> bool:
        evaluator.evaluate_hessian(state)
        evaluator.evaluate_diagonal(state)
        device = self._device_solver(solver)
        if device and self._rows_set_for is not solver:
            solver.set_perturbation_rows(_index_array(self.problem.get_primal_indices()),
                                         _index_array(self.problem.get_constraint_indices()))
            self._rows_set_for = solver
        if device:
            solver.load_system(state.hessian, state.diagonal)

        def attempt():
            dx = self.numerical_eps + self._dw
            if device:
                return solver.factor_perturbed(dx, self._dc)
            d = self._shifted_host_diagonal(state.diagonal, self.perturbed_diagonal)
            solver.factor(state.hessian, d)
            return solver.get_inertia()

        self.attempts = 0
        self.factorizations = 0
        if not solver.inertia_enabled():
            attempt()
            self.attempts = self.factorizations = 1
            return True

        self._new_system(state)
        solver.set_pivot_tolerance(self._pivtol)
        sharpened = False
        reuse = device and not getattr(solver, "uses_pivot_tolerance", True)
        last = None  # (shifts, inertia) of the previous attempt
        for _ in range(self.max_corrections + 1):
            shifts = (self._dw, self._dc)
            self.attempts += 1
            if reuse and last is not None and last[0] == shifts:
                npos, nneg = last[1]
            else:
                npos, nneg = attempt()
                self.factorizations += 1
            last = (shifts, (npos, nneg))
            if self._inertia_ok(npos, nneg):
                self.last_delta_w = self._dw
                self.last_delta_c = self._dc
                if self._dw > 0 and state.comm_rank == 0 and self.verbose:
                    print(f"  Inertia correction: delta_w={self._dw:.2e}, "
                          f"delta_c={self._dc:.2e}, attempts={self.attempts}")
                return True
            if state.comm_rank == 0 and self.verbose:
                print(f"  Inertia: expected ({self.num_primal}+, {self.num_dual}-), "
                      f"got ({npos}+, {nneg}-), dw={self._dw:.1e}, pivtol={self._pivtol:.1e}")
            if nneg < self.num_dual:
                # too few negative eigenvalues: first sharpen the pivoting,
                # then treat the system as singular
                if not sharpened:
                    sharpened = self._sharpen_pivoting(solver)
                    if sharpened:
                        continue
                if not self._too_few_negative(state):
                    break
            elif not self._too_many_negative(state):
                if state.comm_rank == 0:
                    print(f"  Inertia: delta_w={self._dw:.2e} > max, aborting correction")
                break
        self.last_delta_w = self._dw
        self.last_delta_c = self._dc
        return False

    def add_log_info(self, info):
        info["inertia_delta"] = self.last_delta_w
