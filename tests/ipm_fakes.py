"""Stand-ins for the interior-point objects that an inertia corrector talks
to (options, problem, optimizer, evaluator, state, solver), and a scripted
inertia model. They let the reference's InertiaCorrector and
amigo_b200.inertia_correction.InertiaCorrector run on the same sequence of
systems, so that their attempts (shifts and counts) can be compared."""

from __future__ import annotations

import numpy as np

N_PRIMAL = 4
N_DUAL = 2
PRIMAL = np.arange(N_PRIMAL, dtype=np.int32)
DUAL = np.arange(N_PRIMAL, N_PRIMAL + N_DUAL, dtype=np.int32)
BASE_DIAG = np.array([1.0, 2.0, 0.5, 3.0, -1e-8, -1e-8])


class FakeVec:
    """amigo.Vector's operations that the corrector uses."""

    def __init__(self, n):
        self.a = np.zeros(n)

    def copy(self, src):
        self.a[...] = src.a if isinstance(src, FakeVec) else np.asarray(src)

    def add_scalar_at(self, idx, value):
        self.a[np.asarray(idx)] += value

    def get_size(self):
        return len(self.a)

    def __getitem__(self, k):
        return self.a[k]

    def __array__(self, dtype=None, copy=None):
        return self.a if dtype is None else self.a.astype(dtype)


class FakeProblem:
    def create_vector(self):
        return FakeVec(N_PRIMAL + N_DUAL)

    def get_primal_indices(self):
        return PRIMAL

    def get_constraint_indices(self):
        return DUAL


class FakeOptimizer:
    def get_num_primals(self):
        return N_PRIMAL

    def get_num_constraints(self):
        return N_DUAL


class FakeEvaluator:
    def evaluate_hessian(self, state):
        pass

    def evaluate_diagonal(self, state):
        pass


class FakeState:
    def __init__(self, mu):
        self.mu = mu
        self.comm_rank = 0
        self.hessian = "H"
        self.diagonal = FakeVec(N_PRIMAL + N_DUAL)
        self.diagonal.a[...] = BASE_DIAG


def model_inertia(rule, dw, dc):
    """Inertia of a scripted system under primal shift dw and constraint
    shift dc. rule["singular"]: None, "jac" (short of negative eigenvalues
    unless dc > 0), "hess" (unless dw > 0) or "both" (unless both); then
    rule["tx"]: one eigenvalue has the wrong sign until dw >= tx."""
    sing = rule.get("singular")
    short = ((sing == "jac" and dc == 0.0) or (sing == "hess" and dw == 0.0)
             or (sing == "both" and (dc == 0.0 or dw == 0.0)))
    if short:
        return N_PRIMAL, N_DUAL - 1
    if dw < rule.get("tx", 0.0):
        return N_PRIMAL - 1, N_DUAL + 1
    return N_PRIMAL, N_DUAL


class ScriptedSolver:
    """A solver whose inertia follows model_inertia. ``shifts()`` reads the
    corrector's current (dw, dc). Records every factorization."""

    def __init__(self, shifts, device=False):
        self.shifts = shifts
        self.rule = {}
        self.log = []
        self.pivtols = []
        self._inertia = (0, 0)
        if device:
            self.factor_perturbed = self._factor_perturbed
            self.uses_pivot_tolerance = False

    def inertia_enabled(self):
        return True

    def set_pivot_tolerance(self, pivtol):
        self.pivtols.append(pivtol)

    def factor(self, hessian, diag):
        dw, dc = self.shifts()
        self._inertia = model_inertia(self.rule, dw, dc)
        self.log.append((dw, dc, *self._inertia, np.array(np.asarray(diag), dtype=float)))
        return 0

    def get_inertia(self):
        return self._inertia

    # device-style attempts (B200LdlSolver's interface)
    def set_perturbation_rows(self, primal, dual):
        self.rows = (np.asarray(primal), np.asarray(dual))

    def load_system(self, hessian, diagonal):
        self.loaded = np.array(np.asarray(diagonal), dtype=float)

    def _factor_perturbed(self, delta_x, delta_c):
        dw, dc = self.shifts()
        d = self.loaded.copy()
        d[self.rows[0]] += delta_x
        if delta_c > 0:
            d[self.rows[1]] += -delta_c
        self._inertia = model_inertia(self.rule, dw, dc)
        self.log.append((dw, dc, *self._inertia, d))
        return self._inertia


def scenarios():
    """Sequences of systems (rule, mu) covering each branch of Algorithm IC."""
    rng = np.random.default_rng(0)
    mus = [0.1 * 0.2**k for k in range(40)]
    out = {
        "no_shift": [{"tx": 0.0}] * 3,
        "primal_shift_schedule": [{"tx": t} for t in
                                  (1e-3, 0.5, 1e3, 1e-30, 5e-4, 2e-4, 7.0, 1e-6, 1e-12)],
        "primal_shift_overflow": [{"tx": 1e30}, {"tx": 1e-2}, {"tx": 1e30}, {"tx": 1e-2},
                                  {"singular": "hess", "tx": 1e30}, {"tx": 0.0}],
        "jacobian_degenerate": [{"singular": "jac"}] * 5 + [{"singular": "jac", "tx": 1e-2}],
        "hessian_degenerate": [{"singular": "hess", "tx": 1e-2}] * 5,
        "both_degenerate": [{"singular": "both", "tx": 1e-3}] * 5,
    }
    mixed = []
    for _ in range(30):
        sing = [None, None, "jac", "hess", "both"][rng.integers(5)]
        tx = [0.0, 1e-5, 1e-2, 3.0, 1e4][rng.integers(5)]
        mixed.append({"singular": sing, "tx": tx})
    out["mixed"] = mixed
    return {k: [(r, mus[i]) for i, r in enumerate(v)] for k, v in out.items()}


def run_scenario(corrector_cls, shifts_of, systems, device=False):
    """Drive a corrector through the systems; per system: its attempts
    [(dw, dc, npos, nneg, diagonal)], the result and last shifts."""
    options = {"verbose_barrier": False, "inertia_tolerance": 0}
    corr = corrector_cls(options, FakeProblem(), FakeOptimizer())
    solver = ScriptedSolver(lambda: shifts_of(corr), device=device)
    out = []
    for rule, mu in systems:
        solver.rule = rule
        solver.log = []
        ok = corr.factor_for_inertia(solver, FakeEvaluator(), FakeState(mu))
        out.append({"attempts": list(solver.log), "ok": bool(ok),
                    "last_delta_w": corr.last_delta_w, "last_delta_c": corr.last_delta_c,
                    "pivtols": list(solver.pivtols)})
        solver.pivtols = []
    return out
