"""GPU inertia correction: the corrector driving the device attempts
(b200ldl_factor_perturbed through B200LdlSolver) takes the same steps as the
same corrector driving the compiled reference SparseLDL with the perturbed
diagonal formed on the host (the reference's own route,
inertia_correction.py:293-316). The corrector itself is pinned to the
reference's class on CPU (test_inertia_correction.py)."""

import numpy as np
import pytest

from amigo_b200.inertia_correction import InertiaCorrector
from amigo_b200.solver import B200LdlSolver
from amigo_b200.sparse_ldl import CSRMat, OrderingType
from amigo_b200.workloads import optimal_control_kkt
from oracle import ref
from tests.conftest import backward_error

pytestmark = pytest.mark.gpu


class _Vec:
    def __init__(self, a):
        self.a = np.array(a, dtype=np.float64)

    def copy(self, src):
        self.a[...] = src.a

    def add_scalar_at(self, idx, value):
        self.a[np.asarray(idx)] += value

    def get_size(self):
        return len(self.a)

    def __getitem__(self, k):
        return self.a[k]

    def __array__(self, dtype=None, copy=None):
        return self.a


class _Problem:
    def __init__(self, n, nprim):
        self.n = n
        self.nprim = nprim

    def create_vector(self):
        return _Vec(np.zeros(self.n))

    def get_primal_indices(self):
        return np.arange(self.nprim, dtype=np.int32)

    def get_constraint_indices(self):
        return np.arange(self.nprim, self.n, dtype=np.int32)


class _Optimizer:
    def __init__(self, nprim, ncon):
        self.nprim, self.ncon = nprim, ncon

    def get_num_primals(self):
        return self.nprim

    def get_num_constraints(self):
        return self.ncon


class _Evaluator:
    def evaluate_hessian(self, state):
        pass

    def evaluate_diagonal(self, state):
        pass


class _State:
    def __init__(self, hessian, diag, mu):
        self.hessian = hessian
        self.diagonal = _Vec(diag)
        self.mu = mu
        self.comm_rank = 0


class _RefSolver:
    """The compiled reference SparseLDL behind the plugin interface,
    recording each factorization's inertia."""

    def __init__(self, mat):
        self.mat = mat
        self.r = ref.RefLDL(mat.rowp, mat.cols, order=int(OrderingType.AMD))
        self.log = []

    def inertia_enabled(self):
        return True

    def set_pivot_tolerance(self, pivtol):
        pass

    def factor(self, hessian, diag):
        self.r.factor(np.asarray(hessian.vals), np.asarray(diag, dtype=np.float64))
        self.log.append((self.corr._dw, self.corr._dc) + tuple(self.r.inertia()))

    def get_inertia(self):
        return tuple(self.r.inertia())


class _Recorder(B200LdlSolver):
    def factor_perturbed(self, delta_x, delta_c):
        out = super().factor_perturbed(delta_x, delta_c)
        self.log.append((self.corr._dw, self.corr._dc) + tuple(out))
        return out


def _systems(s):
    """IPM-like sequence on one pattern: plain; indefinite Hessian block
    (wrong inertia until delta_w is large enough); a zero constraint row (too
    few negative eigenvalues until delta_c > 0); plain again."""
    r = np.repeat(np.arange(s.n), np.diff(s.rowp))
    out = [(s.vals.copy(), s.diag.copy())]
    d = s.diag.copy()
    d[: s.n_primal: 97] = -30.0
    out.append((s.vals.copy(), d))
    v = s.vals.copy()
    c = s.n_primal + 5
    v[(r == c) | (s.cols == c)] = 0.0
    d = s.diag.copy()
    d[c] = 0.0
    out.append((v, d))
    out.append((s.vals.copy(), s.diag.copy()))
    return out


def test_device_attempts_follow_reference_factorizations():
    s = optimal_control_kkt(N=200, nrhs=1, seed=3)
    opts = {"verbose_barrier": False, "inertia_tolerance": 0}
    mat_g = CSRMat(s.n, s.n, s.rowp, s.cols, s.vals.copy())
    mat_r = CSRMat(s.n, s.n, s.rowp, s.cols, s.vals.copy())
    gsolver = _Recorder(opts, hessian=mat_g, order=OrderingType.AMD)
    gsolver.log = []
    rsolver = _RefSolver(mat_r)
    prob = _Problem(s.n, s.n_primal)
    optim = _Optimizer(s.n_primal, s.n_con)
    cg = InertiaCorrector(opts, prob, optim)
    cr = InertiaCorrector(opts, prob, optim)
    gsolver.corr, rsolver.corr = cg, cr
    for k, (vals, diag) in enumerate(_systems(s)):
        mu = 0.1 * 0.2**k
        mat_g.vals = vals.copy()
        mat_r.vals = vals.copy()
        gsolver.log, rsolver.log = [], []
        ok_g = cg.factor_for_inertia(gsolver, _Evaluator(), _State(mat_g, diag, mu))
        ok_r = cr.factor_for_inertia(rsolver, _Evaluator(), _State(mat_r, diag, mu))
        assert ok_g == ok_r, k
        assert (cg.last_delta_w, cg.last_delta_c) == (cr.last_delta_w, cr.last_delta_c), k
        assert cg.attempts == cr.attempts, k
        # same shifts and inertia at every attempt; the device skips only an
        # attempt that repeats the previous one's shifts
        want = [a for i, a in enumerate(rsolver.log)
                if i == 0 or a[:2] != rsolver.log[i - 1][:2]]
        assert gsolver.log == want, (k, gsolver.log, rsolver.log)
        assert cg.factorizations == len(want) and cr.factorizations == len(rsolver.log)
        if k == 1:
            assert cg.last_delta_w > 0 and cg.attempts > 1
        if k == 2:
            assert cg.last_delta_c > 0 and cg.factorizations < cr.factorizations
        # the stored factor solves the perturbed system to FP64 accuracy
        pd = gsolver.ldl.perturbed_diagonal().cpu().numpy()
        sys_k = optimal_control_kkt(N=200, nrhs=1, seed=3)
        sys_k.vals, sys_k.diag = vals, pd
        b = s.rhs[:, 0].copy()
        x = b.copy()
        gsolver.ldl.solve(x)
        assert backward_error(sys_k, x, b) <= 1e-12, k
        # the perturbed diagonal is bit-identical to the host-formed one
        want_d = np.array(diag)
        want_d[: s.n_primal] += cg.numerical_eps + cg.last_delta_w
        if cg.last_delta_c > 0:
            want_d[s.n_primal:] += -cg.last_delta_c
        assert np.array_equal(pd, want_d), k

