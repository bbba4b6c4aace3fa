"""GPU parity of pivot-order reuse: fronts re-planned from a factorization's
own pivot record, factored again on the device. Inertia must equal the
compiled reference's and the backward error stay at the FP64 level, both for
the values the record came from and for other values of the same pattern."""

import dataclasses

import numpy as np
import pytest

from amigo_b200.sparse_ldl import CSRMat, OrderingType, SparseLDL, SparseLDLBatch, Vector
from amigo_b200.workloads import batched_optimal_control, optimal_control_kkt, plane_stress_kkt
from oracle import ref
from tests.conftest import backward_error

pytestmark = pytest.mark.gpu

BERR_TOL = 1e-12


def _factor_solve(ldl, s):
    ldl.mat.vals = s.vals
    assert ldl.factor(Vector(s.diag)) == 0
    x = np.asfortranarray(s.rhs.copy())
    ldl.solve(x)
    return x


@pytest.mark.parametrize("nel", [32, 96])
def test_plane_stress_reuse(nel):
    s0, s1 = plane_stress_kkt(nel, seed=0), plane_stress_kkt(nel, seed=1)
    ldl = SparseLDL(CSRMat(s0.n, s0.n, s0.rowp, s0.cols, s0.vals), order=OrderingType.AMD)
    _factor_solve(ldl, s0)
    delayed_ref_structure = ldl.stats()["delayed"]
    ldl.reuse_pivot_order()
    r = ref.RefLDL(s0.rowp, s0.cols, order=ref.ORDER_AMD)
    for s in (s0, s1):
        x = _factor_solve(ldl, s)
        r.factor(s.vals, s.diag)
        assert tuple(ldl.get_inertia()) == tuple(r.inertia()) == s.expected_inertia
        assert backward_error(s, x, s.rhs) <= BERR_TOL
        xr = r.solve(s.rhs)
        assert np.abs(x - xr).max() / np.abs(xr).max() < 1e-6
        if s is s0:
            # the same values: every candidate is accepted where it now stands
            # (rounding may flip a borderline test)
            assert ldl.stats()["delayed"] <= max(8, delayed_ref_structure // 200)


def test_optimal_control_and_batch_reuse():
    s = optimal_control_kkt(N=400, seed=4)
    ldl = SparseLDL(CSRMat(s.n, s.n, s.rowp, s.cols, s.vals), order=OrderingType.AMD)
    _factor_solve(ldl, s)
    ldl.reuse_pivot_order()
    x = _factor_solve(ldl, s)
    assert tuple(ldl.get_inertia()) == s.expected_inertia
    assert backward_error(s, x, s.rhs) <= BERR_TOL
    systems = batched_optimal_control(num_systems=12, seed=9)
    mats = [CSRMat(q.n, q.n, q.rowp, q.cols, q.vals) for q in systems]
    batch = SparseLDLBatch(mats, order=OrderingType.AMD)
    d = Vector(np.concatenate([q.diag for q in systems]))
    batch.factor(d)
    batch.reuse_pivot_order()
    batch.factor(d)
    bh = np.concatenate([q.rhs[:, 0] for q in systems])
    xb = bh.copy()
    batch.solve(xb)
    for q, xs, inert in zip(systems, batch.split(xb), batch.system_inertia()):
        assert tuple(int(v) for v in inert) == q.expected_inertia
        assert backward_error(q, xs.reshape(-1, 1), q.rhs[:, :1]) <= BERR_TOL


def test_plugin_reuses_and_refreshes_the_pivot_order():
    """B200LdlSolver with reuse_pivot_order: the second factorization runs on
    the structure re-planned from the first, and with refresh_delays = 0
    every factorization that delays a candidate re-plans the next one from
    its own record (a record taken on a re-planned structure). Inertia as
    the compiled reference gives it and FP64-level backward errors on the
    benchmark values, a neighbouring iterate's values, and back."""
    from amigo_b200.solver import B200LdlSolver
    from tests.test_gpu_configs import _perturbed_values

    s = plane_stress_kkt(48)
    mat = CSRMat(s.n, s.n, s.rowp, s.cols, s.vals.copy())
    solver = B200LdlSolver(hessian=mat, order=OrderingType.AMD, reuse_pivot_order=True,
                           refresh_delays=0.0)
    pv, pd = _perturbed_values(s)
    b = s.rhs[:, 0].copy()
    for vals, diag in ((s.vals, s.diag), (pv, pd), (s.vals, s.diag), (pv, pd)):
        mat.vals[:] = vals
        solver.factor(mat, diag)
        r = ref.RefLDL(s.rowp, s.cols, order=ref.ORDER_AMD)
        r.factor(vals, diag)
        assert tuple(solver.get_inertia()) == tuple(r.inertia())
        x = np.empty(s.n)
        solver.solve(b, x)
        sys_ = dataclasses.replace(s, vals=np.asarray(vals), diag=np.asarray(diag))
        assert backward_error(sys_, x.reshape(-1, 1), b.reshape(-1, 1)) <= 1e-12
    assert solver._planned
