"""GPU parity of the mixed-precision factorization: after pivot-order reuse,
the contribution-block tiles of the big fronts' trailing updates run on the
tensor cores (about FP32 accuracy) and every solve is refined in FP64
against the factored matrix. A mixed factorization whose inertia differs
from the handle's last FP64 factorization, or whose refinement stalls, is
redone in FP64 (on these KKT systems FP32-level rounding flips the sign of
pivots that cancellation makes tiny). Whatever the path, inertia must equal
the compiled reference's, the backward error must be at the FP64 level, and
the solution must agree with the reference's FP64 solve as the FP64 path
does."""

import numpy as np
import pytest

from amigo_b200.sparse_ldl import CSRMat, OrderingType, SparseLDL, Vector
from amigo_b200.workloads import hex_elasticity_kkt, plane_stress_kkt
from oracle import ref
from tests.conftest import backward_error

pytestmark = pytest.mark.gpu

BERR_TOL = 1e-12


def _mixed(s, reuse_from=None):
    ldl = SparseLDL(CSRMat(s.n, s.n, s.rowp, s.cols, s.vals), order=OrderingType.AMD)
    src = s if reuse_from is None else reuse_from
    ldl.mat.vals = src.vals
    assert ldl.factor(Vector(src.diag)) == 0
    ldl.reuse_pivot_order()
    ldl.set_precision("mixed")
    ldl.mat.vals = s.vals
    assert ldl.factor(Vector(s.diag)) == 0
    return ldl


@pytest.mark.parametrize("make", [lambda: plane_stress_kkt(48), lambda: plane_stress_kkt(128),
                                  lambda: hex_elasticity_kkt(8)],
                         ids=["plane_stress_48", "plane_stress_128", "hex_8"])
def test_mixed_precision_matches_reference(make):
    s = make()
    ldl = _mixed(s)
    r = ref.RefLDL(s.rowp, s.cols, order=ref.ORDER_AMD)
    r.factor(s.vals, s.diag)
    assert tuple(ldl.get_inertia()) == tuple(r.inertia()) == s.expected_inertia
    x = np.asfortranarray(s.rhs.copy())
    ldl.solve(x)
    info = ldl.last_refinement()
    assert info["mixed"] or info["fp64_redos"] > 0
    assert backward_error(s, x, s.rhs) <= BERR_TOL
    xr = r.solve(s.rhs)
    tol = 1e-4 if s.name.startswith("hex") else 1e-6
    assert np.abs(x - xr).max() / np.abs(xr).max() < tol


def test_mixed_precision_with_record_from_other_values():
    s0, s1 = plane_stress_kkt(64, seed=0), plane_stress_kkt(64, seed=1)
    ldl = _mixed(s1, reuse_from=s0)
    r = ref.RefLDL(s1.rowp, s1.cols, order=ref.ORDER_AMD)
    r.factor(s1.vals, s1.diag)
    assert tuple(ldl.get_inertia()) == tuple(r.inertia())
    x = np.asfortranarray(s1.rhs.copy())
    ldl.solve(x)
    assert backward_error(s1, x, s1.rhs) <= BERR_TOL
