"""CPU tests: the oracle pinned against the reference's golden cases, the
C-ABI library's exported symbols, and the host symbolic phase compared
bit-for-bit with the reference's (ordering, supernode partition, children,
contribution rows)."""

import os
import re

import numpy as np
import pytest

from amigo_b200 import _native
from amigo_b200.sparse_ldl import CSRMat, OrderingType, SparseLDL
from amigo_b200.workloads import (batched_optimal_control, csr_from_coo,
                                  optimal_control_kkt, plane_stress_kkt, poisson_2d)
from oracle import ref

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    header = open(os.path.join(ROOT, "include", "b200ldl.h")).read()
    declared = set(re.findall(r"\b(b200ldl_[a-z_]+)\s*\(", header))
    assert declared, "no declarations found"
    lib = _native.load()
    for name in declared:
        assert hasattr(lib, name), name
    assert declared == set(_native.SIGNATURES)


@pytest.mark.parametrize("order", ["natural", "amd"])
def test_oracle_matches_reference_golden(golden, order):
    """The compiled reference reproduces the reference tests' assertions
    (tests/unit/test_ldl.py: exact inertia, 7-RHS solutions of A x = A 1 to
    1e-11) and the stored fixture."""
    code = ref.ORDER_NATURAL if order == "natural" else ref.ORDER_AMD
    for name in golden["names"]:
        rowp = golden[f"{name}/rowp"]
        cols = golden[f"{name}/cols"]
        vals = golden[f"{name}/vals"]
        r = ref.RefLDL(rowp, cols, order=code, ustab=0.4)
        assert r.factor(vals) == 0
        assert tuple(r.inertia()) == tuple(golden[f"{name}/inertia"]), name
        assert tuple(r.inertia()) == tuple(golden[f"{name}/{order}/inertia"]), name
        X = np.tile(golden[f"{name}/rhs"][:, None], (1, 7))
        x = r.solve(X)
        assert np.abs(x - golden[f"{name}/x"][:, None]).max() < 1e-11, name
        assert np.abs(x - golden[f"{name}/{order}/solution"]).max() < 1e-13, name


def _compare_symbolic(rowp, cols, order):
    n = len(rowp) - 1
    mine = SparseLDL(CSRMat(n, n, rowp, cols), order=order)
    theirs = ref.RefLDL(rowp, cols, order=int(order))
    a = mine.symbolic()
    b = theirs.symbolic()
    for key in a:
        assert a[key].shape == b[key].shape, key
        assert np.array_equal(a[key], b[key]), key


@pytest.mark.parametrize("order", [OrderingType.AMD, OrderingType.NATURAL,
                                   OrderingType.NESTED_DISSECTION])
def test_symbolic_matches_reference_golden_cases(golden, order):
    for name in golden["names"]:
        _compare_symbolic(golden[f"{name}/rowp"], golden[f"{name}/cols"], order)


@pytest.mark.parametrize("order", [OrderingType.AMD, OrderingType.NATURAL])
def test_symbolic_matches_reference_kkt(order):
    s = optimal_control_kkt()
    _compare_symbolic(s.rowp, s.cols, order)
    for s in batched_optimal_control(num_systems=6, seed=3):
        _compare_symbolic(s.rowp, s.cols, order)
    for nel in (4, 16, 48):
        s = plane_stress_kkt(nel)
        _compare_symbolic(s.rowp, s.cols, order)


def test_symbolic_matches_reference_random_patterns():
    rng = np.random.default_rng(7)
    for _ in range(40):
        n = int(rng.integers(1, 250))
        dens = rng.random() * 0.08
        a = rng.random((n, n)) < dens
        a = a | a.T
        r, c = np.nonzero(a)
        rowp, cols, _ = csr_from_coo(n, r, c, np.ones(len(r)))
        _compare_symbolic(rowp, cols, OrderingType.AMD)


def test_symbolic_handles_disconnected_and_trivial():
    # n = 1, diagonal only, and a block-diagonal (forest) pattern
    for n, r, c in ((1, [0], [0]), (5, list(range(5)), list(range(5))),
                    (6, [0, 1, 3, 4], [1, 0, 4, 3])):
        rowp, cols, _ = csr_from_coo(n, r, c, np.ones(len(r)))
        _compare_symbolic(rowp, cols, OrderingType.AMD)
        _compare_symbolic(rowp, cols, OrderingType.NATURAL)


@pytest.mark.slow
def test_symbolic_matches_reference_plane_stress_256():
    s = plane_stress_kkt(256)
    _compare_symbolic(s.rowp, s.cols, OrderingType.AMD)


def test_create_rejects_bad_input():
    with pytest.raises(_native.NativeError):
        SparseLDL(CSRMat(2, 2, [0, 1, 2], [0, 5], [1.0, 1.0]))
    with pytest.raises(_native.NativeError):
        SparseLDL(CSRMat(2, 2, [0, 1, 2], [0, 1], [1.0, 1.0]), order=OrderingType.MULTI_COLOR)


def test_poisson_generator_matches_reference_matrix(golden):
    for n in (10, 20, 50):
        rowp, cols, vals = poisson_2d(n)
        m = (n - 1) ** 2
        a = np.zeros((m, m))
        r = np.repeat(np.arange(m), np.diff(rowp))
        a[r, cols] = vals
        g = np.zeros((m, m))
        gr = golden[f"poisson{n}/rowp"]
        g[np.repeat(np.arange(m), np.diff(gr)), golden[f"poisson{n}/cols"]] = \
            golden[f"poisson{n}/vals"]
        assert np.array_equal(a, g)


def test_reference_cholesky_oracle_on_golden_cases(golden):
    """The compiled reference SparseCholesky solves the golden positive
    definite cases and refuses the indefinite ones."""
    for name in golden["names"]:
        rowp, cols, vals = (golden[f"{name}/{k}"] for k in ("rowp", "cols", "vals"))
        c = ref.RefCholesky(rowp, cols)
        flag = c.factor(vals)
        spd = tuple(golden[f"{name}/natural/inertia"])[1] == 0
        assert (flag == 0) == spd, name
        if spd:
            x = c.solve(golden[f"{name}/rhs"])
            assert np.abs(x - golden[f"{name}/x"]).max() < 1e-11, name


def test_batch_symbolic_is_each_systems_own():
    """A batch handle's merged forest is every system's own symbolic phase,
    shifted by the system's variable and supernode offsets (host only)."""
    from amigo_b200.sparse_ldl import SparseLDLBatch

    systems = batched_optimal_control(num_systems=5, seed=11)
    mats = [CSRMat(q.n, q.n, q.rowp, q.cols, q.vals) for q in systems]
    batch = SparseLDLBatch(mats, order=OrderingType.AMD)
    m = batch.symbolic()
    voff = noff = 0
    roots = []
    for q in systems:
        one = SparseLDL(CSRMat(q.n, q.n, q.rowp, q.cols, q.vals), order=OrderingType.AMD)
        s = one.symbolic()
        nn = len(s["node_ptr"]) - 1
        assert np.array_equal(m["invperm"][voff:voff + q.n], s["invperm"] + voff)
        assert np.array_equal(m["node_to_var"][voff:voff + q.n], s["node_to_var"] + voff)
        assert np.array_equal(m["node_ptr"][noff:noff + nn + 1], s["node_ptr"] + voff)
        for k in range(nn):
            a0, a1 = m["contrib_ptr"][noff + k], m["contrib_ptr"][noff + k + 1]
            b0, b1 = s["contrib_ptr"][k], s["contrib_ptr"][k + 1]
            assert np.array_equal(m["contrib_rows"][a0:a1], s["contrib_rows"][b0:b1] + voff)
            c0, c1 = m["children_ptr"][noff + k], m["children_ptr"][noff + k + 1]
            d0, d1 = s["children_ptr"][k], s["children_ptr"][k + 1]
            assert np.array_equal(m["children"][c0:c1], s["children"][d0:d1] + noff)
        r0, r1 = s["children_ptr"][nn], s["children_ptr"][nn + 1]
        roots.extend((s["children"][r0:r1] + noff).tolist())
        voff += q.n
        noff += nn
    total = len(m["node_ptr"]) - 1
    assert total == noff
    # every system's roots, in system order, in the merged roots slot
    assert m["children"][m["children_ptr"][total]:m["children_ptr"][total + 1]].tolist() == roots


def test_hex_element_stiffness_has_the_rigid_modes():
    from amigo_b200.workloads import _q1_hex_ke

    ke = _q1_hex_ke()
    assert np.abs(ke - ke.T).max() < 1e-15
    assert np.linalg.matrix_rank(ke) == 18
    # node coordinates of the unit cube in the element's node order
    xyz = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                    [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], dtype=float)
    for d in range(3):
        t = np.zeros(24)
        t[d::3] = 1.0
        assert np.abs(ke @ t).max() < 1e-14
    for a, b in ((0, 1), (1, 2), (2, 0)):  # small rotations about each axis
        w = np.zeros(24)
        w[a::3] = -xyz[:, b]
        w[b::3] = xyz[:, a]
        assert np.abs(ke @ w).max() < 1e-14


@pytest.mark.parametrize("order", [OrderingType.AMD, OrderingType.NATURAL])
def test_symbolic_matches_reference_hex_with_dense_row(order):
    """The 3D workload with its dense volume-constraint row, at small sizes."""
    from amigo_b200.workloads import hex_elasticity_kkt

    for nel in (2, 4, 6, 10):
        s = hex_elasticity_kkt(nel)
        _compare_symbolic(s.rowp, s.cols, order)


def test_hex_workload_has_the_designed_inertia():
    """The compiled reference factors the 3D workload with the inertia the
    generator promises (n_primal positive, n_con negative) and a FP64
    backward error."""
    from amigo_b200.workloads import hex_elasticity_kkt

    for nel in (3, 5):
        s = hex_elasticity_kkt(nel)
        r = ref.RefLDL(s.rowp, s.cols, order=ref.ORDER_AMD)
        r.factor(s.vals, s.diag)
        assert tuple(r.inertia()) == s.expected_inertia
        x = r.solve(s.rhs)
        berr = np.abs(s.matvec(x) - s.rhs).max() / (
            s.inf_norm() * np.abs(x).max() + np.abs(s.rhs).max())
        assert berr < 1e-14


def test_symbolic_matches_reference_cliques_and_dense_rows():
    """Patterns that reach the ordering's long-list paths: many small
    cliques (repeated ones make indistinguishable variables) and a few dense
    rows."""
    rng = np.random.default_rng(123)
    for _ in range(30):
        n = int(rng.integers(200, 1500))
        rows, cols = [], []
        for _ in range(int(rng.integers(n // 8, n // 2))):
            m = int(rng.integers(2, 12))
            vs = rng.choice(n, size=m, replace=False)
            rows.extend(np.repeat(vs, m))
            cols.extend(np.tile(vs, m))
        for _ in range(int(rng.integers(0, 4))):
            d = int(rng.integers(n))
            others = rng.choice(n, size=int(rng.integers(n // 3, n)), replace=False)
            rows.extend([d] * len(others) + list(others))
            cols.extend(list(others) + [d] * len(others))
        rowp, colsp, _ = csr_from_coo(n, np.array(rows), np.array(cols), np.ones(len(rows)))
        _compare_symbolic(rowp, colsp, OrderingType.AMD)


def test_generated_kkt_systems_are_symmetric_with_diagonals():
    """Every workload's CSR holds the full symmetric pattern with exactly
    symmetric values, a diagonal entry in every row and sorted columns."""
    from amigo_b200.workloads import hex_elasticity_kkt

    for s in (optimal_control_kkt(N=50), plane_stress_kkt(6), hex_elasticity_kkt(3),
              *batched_optimal_control(num_systems=2, seed=1)):
        n = s.n
        r = np.repeat(np.arange(n), np.diff(s.rowp))
        a = {(int(i), int(j)): v for i, j, v in zip(r, s.cols, s.vals)}
        assert all(a.get((j, i)) == v for (i, j), v in a.items()), s.name
        assert all((i, i) in a for i in range(n)), s.name
        for i in range(n):
            c = s.cols[s.rowp[i]:s.rowp[i + 1]]
            assert np.all(np.diff(c) > 0), s.name


def _permuted_csr(rowp, cols, iperm):
    n = len(rowp) - 1
    r = np.repeat(np.arange(n), np.diff(rowp))
    rp, cp, _ = csr_from_coo(n, iperm[r], iperm[cols], np.ones(len(r)))
    return rp, cp


def test_graph_nd_gives_a_permutation_on_awkward_patterns():
    rng = np.random.default_rng(5)
    cases = [(1, [0], [0]), (6, [0, 1, 3, 4], [1, 0, 4, 3])]
    for _ in range(20):
        n = int(rng.integers(50, 1500))
        a = rng.random((n, n)) < rng.random() * 0.02
        a = a | a.T
        if rng.random() < 0.5:  # a dense row
            d = int(rng.integers(n))
            a[d, :] = a[:, d] = True
        r, c = np.nonzero(a)
        cases.append((n, r, c))
    for n, r, c in cases:
        rowp, cols, _ = csr_from_coo(n, np.asarray(r), np.asarray(c), np.ones(len(r)))
        inv = SparseLDL(CSRMat(n, n, rowp, cols), order=OrderingType.GRAPH_ND).symbolic()["invperm"]
        assert sorted(inv.tolist()) == list(range(n))


def test_symbolic_under_graph_nd_is_the_references_on_the_permuted_matrix():
    """With our nested dissection, the supernodes, children and contribution
    rows equal the reference's symbolic phase run on the symmetrically
    permuted matrix in natural order (mapped back through the permutation);
    and the reference factors that matrix with the designed inertia."""
    from amigo_b200.workloads import hex_elasticity_kkt

    for s in (plane_stress_kkt(16), hex_elasticity_kkt(6)):
        a = SparseLDL(CSRMat(s.n, s.n, s.rowp, s.cols), order=OrderingType.GRAPH_ND).symbolic()
        inv = a["invperm"]
        perm = np.argsort(inv)
        rp, cp = _permuted_csr(s.rowp, s.cols, inv)
        b = ref.RefLDL(rp, cp, order=ref.ORDER_NATURAL).symbolic()
        assert np.array_equal(a["node_ptr"], b["node_ptr"])
        assert np.array_equal(a["node_to_var"], perm[b["node_to_var"]])
        assert np.array_equal(a["children_ptr"], b["children_ptr"])
        assert np.array_equal(a["children"], b["children"])
        assert np.array_equal(a["contrib_ptr"], b["contrib_ptr"])
        assert np.array_equal(a["contrib_rows"], perm[b["contrib_rows"]])
        # the permuted system itself
        r_ = np.repeat(np.arange(s.n), np.diff(s.rowp))
        key = inv[r_].astype(np.int64) * s.n + inv[s.cols]
        vals = np.empty(len(key))
        order_ = np.argsort(key)
        vals[:] = s.vals[order_]  # CSR of P A P^T lists entries in sorted key order
        r = ref.RefLDL(rp, cp, order=ref.ORDER_NATURAL)
        r.factor(vals, s.diag[perm])
        assert tuple(r.inertia()) == s.expected_inertia
