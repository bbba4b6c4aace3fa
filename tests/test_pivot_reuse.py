"""CPU tests of pivot-order reuse: the fronts re-planned from a pivot record.

The record comes from the C restatement oracle factoring the reference's
symbolic structure; the library re-plans the fronts on the host (no GPU
needed) and the oracle then factors the re-planned structure. With the same
values every candidate must be accepted where it now stands (no delays) with
the reference's inertia; with other values of the same pattern the threshold
tests still decide, so the inertia and the accuracy stay the reference's.
"""

import numpy as np
import pytest

from amigo_b200 import _native
from amigo_b200.sparse_ldl import CSRMat, OrderingType, SparseLDL
from amigo_b200.workloads import optimal_control_kkt, plane_stress_kkt
from oracle import port, ref
from tests.conftest import backward_error


def _replanned(system):
    ldl = SparseLDL(CSRMat(system.n, system.n, system.rowp, system.cols), order=OrderingType.AMD)
    sym_ref = ldl.symbolic()
    p = port.PortLDL(system.rowp, system.cols, sym_ref)
    p.factor(system.vals, system.diag)
    rec = p.pivot_record()
    ldl.set_pivot_record(rec)
    return ldl, sym_ref, rec


@pytest.mark.parametrize("make", [lambda s: optimal_control_kkt(N=200, seed=s),
                                  lambda s: plane_stress_kkt(24, seed=s)],
                         ids=["optimal_control", "plane_stress"])
def test_replanned_fronts_accept_every_pivot(make):
    s0 = make(0)
    ldl, sym_ref, rec = _replanned(s0)
    new = ldl.symbolic()
    nn = len(sym_ref["node_ptr"]) - 1
    # same tree; each supernode's pivots are the variables it eliminated
    assert np.array_equal(new["children_ptr"], sym_ref["children_ptr"])
    assert np.array_equal(new["children"], sym_ref["children"])
    assert np.array_equal(np.diff(new["node_ptr"]), rec["npiv"])
    assert np.array_equal(np.sort(new["node_to_var"]), np.arange(s0.n))
    assert np.array_equal(new["invperm"][new["node_to_var"]], np.arange(s0.n))
    assert len(new["contrib_rows"]) == int((rec["f"] - rec["npiv"]).sum())

    r = ref.RefLDL(s0.rowp, s0.cols, order=ref.ORDER_AMD)
    r.factor(s0.vals, s0.diag)
    q = port.PortLDL(s0.rowp, s0.cols, new)
    q.factor(s0.vals, s0.diag)
    rq = q.pivot_record()
    assert int(rq["ndel"].sum()) == 0
    assert np.array_equal(rq["f"], rec["f"])
    assert q.inertia() == r.inertia() == s0.expected_inertia
    x = q.solve(s0.rhs)
    assert backward_error(s0, x, s0.rhs) < 1e-14
    xr = r.solve(s0.rhs)
    assert np.abs(x - xr).max() / np.abs(xr).max() < 1e-6

    # other values of the same pattern (the next interior-point iterate):
    # threshold tests and delays still decide, and fewer candidates move
    s1 = make(1)
    r.factor(s1.vals, s1.diag)
    p1 = port.PortLDL(s1.rowp, s1.cols, sym_ref)
    p1.factor(s1.vals, s1.diag)
    q.factor(s1.vals, s1.diag)
    assert q.inertia() == r.inertia() == s1.expected_inertia
    assert backward_error(s1, q.solve(s1.rhs), s1.rhs) < 1e-14
    assert q.pivot_record()["ndel"].sum() <= p1.pivot_record()["ndel"].sum()
    assert nn == len(new["node_ptr"]) - 1


def test_reset_returns_to_reference_structure():
    s = plane_stress_kkt(12, seed=3)
    ldl, sym_ref, rec = _replanned(s)
    assert not np.array_equal(ldl.symbolic()["node_to_var"], sym_ref["node_to_var"])
    ldl.set_pivot_record(None)
    back = ldl.symbolic()
    theirs = ref.RefLDL(s.rowp, s.cols, order=ref.ORDER_AMD).symbolic()
    for key in theirs:
        assert np.array_equal(back[key], theirs[key]), key


def test_invalid_record_is_rejected_and_structure_kept():
    s = plane_stress_kkt(10, seed=2)
    ldl, sym_ref, rec = _replanned(s)
    planned = ldl.symbolic()
    bad = {k: v.copy() for k, v in rec.items()}
    # a variable eliminated twice (and another never)
    first = int(np.argmax(bad["npiv"] > 1))
    o = int(bad["f"][:first].sum())
    v0 = bad["fv"][o]
    bad["fv"][o + 1] = v0
    with pytest.raises(_native.NativeError) as e:
        ldl.set_pivot_record(bad)
    assert e.value.status == -4
    # a contribution row missing from its parent front
    bad = {k: v.copy() for k, v in rec.items()}
    k = int(np.argmax(bad["f"] > bad["npiv"] + 1))
    o = int(bad["f"][:k].sum())
    bad["fv"][o + bad["f"][k] - 1] = bad["fv"][o]  # duplicate row within one front
    with pytest.raises(_native.NativeError):
        ldl.set_pivot_record(bad)
    after = ldl.symbolic()
    for key in planned:
        assert np.array_equal(after[key], planned[key]), key
