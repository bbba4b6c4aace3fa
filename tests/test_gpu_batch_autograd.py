"""GPU checks of the batched factorization of many independent systems and
of the differentiable solve.

Batched: systems of uneven size in one handle must give every system the
inertia the compiled reference gives it alone, and FP64-level backward
errors per system.

Differentiation: parameters that scale groups of the A_k blocks of an
optimal-control KKT system (the entries of A_k and their mirrors together,
so K stays symmetric) and shift the right-hand side; loss = 1/2 ||x_primal||^2.
The gradient from ``kkt_solve``'s backward pass (adjoint solve on the stored
factor + the value-gradient kernel) must match FP64 central differences of
the same loss computed with the compiled reference solver.
"""

import numpy as np
import pytest

from amigo_b200.sparse_ldl import CSRMat, OrderingType, SparseLDL, SparseLDLBatch
from amigo_b200.workloads import batched_optimal_control, optimal_control_kkt
from oracle import ref
from tests.conftest import backward_error

pytestmark = pytest.mark.gpu

BERR_TOL = 1e-12


def test_batch_of_uneven_systems():
    systems = batched_optimal_control(num_systems=24, nmin=20, nmax=160, nx=6, nu=3, seed=3)
    mats = [CSRMat(s.n, s.n, s.rowp, s.cols, s.vals) for s in systems]
    batch = SparseLDLBatch(mats, order=OrderingType.AMD)
    assert batch.num_systems == len(systems)
    assert batch.factor([s.diag for s in systems]) == 0
    inertia = batch.system_inertia()
    for s, got in zip(systems, inertia):
        r = ref.RefLDL(s.rowp, s.cols, order=int(OrderingType.AMD))
        r.factor(s.vals, s.diag)
        assert got == tuple(r.inertia()) == s.expected_inertia
    assert tuple(batch.get_inertia()) == (sum(p for p, _ in inertia), sum(q for _, q in inertia))
    b = np.concatenate([s.rhs[:, 0] for s in systems])
    x = b.copy()
    batch.solve(x)
    for s, xs, bs in zip(systems, batch.split(x), batch.split(b)):
        assert backward_error(s, xs, bs) <= BERR_TOL
    # the same systems one at a time give the same solutions (up to the
    # summation order of the two factorizations)
    for s, xs in list(zip(systems, batch.split(x)))[:4]:
        g = SparseLDL(CSRMat(s.n, s.n, s.rowp, s.cols, s.vals), order=OrderingType.AMD)
        g.factor(s.diag)
        x1 = s.rhs[:, 0].copy()
        g.solve(x1)
        assert np.abs(x1 - xs).max() <= 1e-6 * np.abs(x1).max()


def _a_groups(s, N, nx, nu, ngroups):
    """Group index of every CSR entry that belongs to an A_k block or its
    mirror (-1 otherwise): stage k -> group floor(ngroups k / (N - 1))."""
    m = nx + nu
    rows = np.repeat(np.arange(s.n), np.diff(s.rowp))
    cols = s.cols.astype(np.int64)
    grp = np.full(s.nnz, -1)
    for r_, c_, flip in ((rows, cols, False), (cols, rows, True)):
        is_con = r_ >= s.n_primal
        k = np.where(is_con, (r_ - s.n_primal) // nx, -1)
        in_a = is_con & (c_ < s.n_primal) & (c_ // m == k) & ((c_ % m) < nx)
        grp = np.where(in_a, (ngroups * k) // (N - 1), grp)
    return grp


def test_adjoint_gradient_matches_central_differences():
    torch = pytest.importorskip("torch")
    from amigo_b200.autograd import kkt_solve

    N, nx, nu, na, nb = 40, 4, 2, 4, 4
    s = optimal_control_kkt(N=N, nx=nx, nu=nu, nrhs=1, seed=11)
    grp = _a_groups(s, N, nx, nu, na)
    assert (grp >= 0).sum() == 2 * (N - 1) * nx * nx
    rng = np.random.default_rng(5)
    shifts = rng.standard_normal((nb, s.n))
    theta0 = 0.05 * rng.standard_normal(na + nb)

    def params(theta):
        scale = np.ones(s.nnz)
        sel = grp >= 0
        scale[sel] += theta[grp[sel]]
        return s.vals * scale, s.rhs[:, 0] + shifts.T @ theta[na:]

    def loss_ref(theta):
        v, b = params(theta)
        r = ref.RefLDL(s.rowp, s.cols, order=int(OrderingType.AMD))
        r.factor(v, s.diag)
        x = r.solve(b.reshape(-1, 1))[:, 0]
        return 0.5 * float(np.sum(x[:s.n_primal] ** 2))

    dev = torch.device("cuda:0")
    th = torch.tensor(theta0, dtype=torch.float64, device=dev, requires_grad=True)
    G = torch.zeros((s.nnz, na), dtype=torch.float64, device=dev)
    sel = np.nonzero(grp >= 0)[0]
    G[torch.as_tensor(sel, device=dev), torch.as_tensor(grp[sel], device=dev)] = 1.0
    v0 = torch.as_tensor(s.vals, device=dev)
    vals = v0 * (1.0 + G @ th[:na])
    b = torch.as_tensor(s.rhs[:, 0], device=dev) + torch.as_tensor(shifts.T, device=dev) @ th[na:]
    diag = torch.as_tensor(s.diag, device=dev)
    ldl = SparseLDL(CSRMat(s.n, s.n, s.rowp, s.cols, vals.detach()), order=OrderingType.AMD)
    x = kkt_solve(ldl, vals, diag, b)
    loss = 0.5 * (x[:s.n_primal] ** 2).sum()
    loss.backward()
    g = th.grad.cpu().numpy()
    lv = float(loss.detach())
    assert abs(lv - loss_ref(theta0)) <= 1e-8 * max(1.0, abs(lv))

    h = 1e-6
    fd = np.zeros_like(theta0)
    for i in range(len(theta0)):
        e = np.zeros_like(theta0)
        e[i] = h
        fd[i] = (loss_ref(theta0 + e) - loss_ref(theta0 - e)) / (2 * h)
    err = np.abs(g - fd).max() / np.abs(fd).max()
    assert err < 1e-5, (err, g, fd)


def test_value_and_diagonal_gradients_directional():
    torch = pytest.importorskip("torch")
    from amigo_b200.autograd import kkt_solve

    s = optimal_control_kkt(N=30, nx=4, nu=2, nrhs=2, seed=2)
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(1)
    # a symmetric direction in the values, a direction in the diagonal
    rows = np.repeat(np.arange(s.n), np.diff(s.rowp))
    w = rng.standard_normal(s.nnz)
    key = np.minimum(rows, s.cols) * s.n + np.maximum(rows, s.cols)
    _, inv = np.unique(key, return_inverse=True)
    dv = w[inv] * np.abs(s.vals) * 1e-2
    dd = rng.standard_normal(s.n) * 1e-2 * np.abs(s.diag)
    vals = torch.tensor(s.vals, device=dev, requires_grad=True)
    diag = torch.tensor(s.diag, device=dev, requires_grad=True)
    b = torch.tensor(np.asfortranarray(s.rhs), device=dev)
    ldl = SparseLDL(CSRMat(s.n, s.n, s.rowp, s.cols, vals.detach()), order=OrderingType.AMD)
    x = kkt_solve(ldl, vals, diag, b)
    loss = 0.5 * (x ** 2).sum()
    loss.backward()
    pred = float((vals.grad.cpu().numpy() * dv).sum() + (diag.grad.cpu().numpy() * dd).sum())

    def loss_ref(t):
        r = ref.RefLDL(s.rowp, s.cols, order=int(OrderingType.AMD))
        r.factor(s.vals + t * dv, s.diag + t * dd)
        xx = r.solve(s.rhs)
        return 0.5 * float(np.sum(xx ** 2))

    h = 1e-5
    fd = (loss_ref(h) - loss_ref(-h)) / (2 * h)
    assert abs(pred - fd) <= 1e-5 * abs(fd), (pred, fd)
