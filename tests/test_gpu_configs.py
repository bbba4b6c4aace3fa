"""GPU checks at the sizes of the batched and differentiation workloads, and
of a front larger than the chained panel kernel takes.

Batched: 512 independent optimal-control systems with N ~ U{50..400},
nx = 6, nu = 3 (the batched workload's own generator and seed) in one handle;
every system's inertia must be the compiled reference's, every backward
error at the FP64 level.

Differentiation: 64 instances of the optimal-control structure with N = 500
(nx = 4, nu = 2), each with 16 parameters: 8 scale groups of its A_k blocks
(the entries and their mirrors), 8 shift its right-hand side.
Loss = sum over instances of 1/2 ||x_primal||^2. The gradient comes from
one backward pass of ``kkt_solve`` on the batch handle (adjoint solve on the
stored factor + the value-gradient kernel). It must match FP64 central
differences of the compiled reference (h = 1e-6) for a few instances, and
for every instance the reference's post-optimality route restated with the
compiled reference: one factorization, psi = K^-1 (-df/dx), and
df/dtheta = psi^T dR/dtheta with R = K x - b (amigo/algorithm/ipm_driver.py:
297-353, method "adjoint"). The factorization is FP64: at these front sizes
(all below 144 rows) the mixed-precision mode has no tensor-core tiles.
"""

import numpy as np
import pytest

from amigo_b200.sparse_ldl import CSRMat, OrderingType, SparseLDL, SparseLDLBatch, Vector
from amigo_b200.workloads import batched_optimal_control, optimal_control_kkt, plane_stress_kkt
from oracle import ref
from tests.conftest import backward_error
from tests.test_gpu_batch_autograd import _a_groups

pytestmark = pytest.mark.gpu

BERR_TOL = 1e-12


def test_batched_workload_512_systems():
    systems = batched_optimal_control()  # 512 systems, N ~ U{50..400}, nx 6, nu 3, seed 0
    assert len(systems) == 512
    mats = [CSRMat(s.n, s.n, s.rowp, s.cols, s.vals) for s in systems]
    batch = SparseLDLBatch(mats, order=OrderingType.AMD)
    assert batch.factor([s.diag for s in systems]) == 0
    inertia = batch.system_inertia()
    b = np.concatenate([s.rhs[:, 0] for s in systems])
    x = b.copy()
    batch.solve(x)
    for s, got, xs, bs in zip(systems, inertia, batch.split(x), batch.split(b)):
        r = ref.RefLDL(s.rowp, s.cols, order=int(OrderingType.AMD))
        r.factor(s.vals, s.diag)
        assert got == tuple(r.inertia()) == s.expected_inertia
        assert backward_error(s, xs, bs) <= BERR_TOL


def _instances(num=64, N=500, nx=4, nu=2, na=8, nb=8):
    out = []
    for i in range(num):
        s = optimal_control_kkt(N=N, nx=nx, nu=nu, nrhs=1, seed=1000 + i)
        grp = _a_groups(s, N, nx, nu, na)
        shifts = np.random.default_rng(2000 + i).standard_normal((nb, s.n))
        out.append((s, grp, shifts))
    return out


def _ref_loss(s, grp, shifts, theta, na):
    scale = np.ones(s.nnz)
    sel = grp >= 0
    scale[sel] += theta[grp[sel]]
    r = ref.RefLDL(s.rowp, s.cols, order=int(OrderingType.AMD))
    r.factor(s.vals * scale, s.diag)
    x = r.solve((s.rhs[:, 0] + shifts.T @ theta[na:]).reshape(-1, 1))[:, 0]
    return 0.5 * float(np.sum(x[:s.n_primal] ** 2))


def _ref_adjoint_gradient(s, grp, shifts, theta, na):
    """The reference's post-optimality route: factor once, psi = K^-1
    (-df/dx), df/dtheta = psi^T dR/dtheta for R(x, theta) = K(theta) x -
    b(theta) (df/dtheta has no direct term here)."""
    scale = np.ones(s.nnz)
    sel = grp >= 0
    scale[sel] += theta[grp[sel]]
    vals = s.vals * scale
    r = ref.RefLDL(s.rowp, s.cols, order=int(OrderingType.AMD))
    r.factor(vals, s.diag)
    b = s.rhs[:, 0] + shifts.T @ theta[na:]
    x = r.solve(b.reshape(-1, 1))[:, 0]
    dfdx = np.zeros(s.n)
    dfdx[:s.n_primal] = x[:s.n_primal]
    psi = r.solve((-dfdx).reshape(-1, 1))[:, 0]
    rows = np.repeat(np.arange(s.n), np.diff(s.rowp))
    g = np.zeros(na + len(shifts))
    # dR/dtheta_j for an A-group scale: the group's entries times x
    for j in range(na):
        e = np.nonzero(grp == j)[0]
        g[j] = float(np.sum(psi[rows[e]] * s.vals[e] * x[s.cols[e]]))
    # dR/dtheta for a right-hand-side shift: -shift
    g[na:] = -(shifts @ psi)
    return g


def test_differentiation_workload_64_instances():
    torch = pytest.importorskip("torch")
    from amigo_b200.autograd import kkt_solve

    na, nb = 8, 8
    inst = _instances(na=na, nb=nb)
    systems = [s for s, _, _ in inst]
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(7)
    theta0 = 0.05 * rng.standard_normal((len(inst), na + nb))

    # parameter -> value maps of the concatenated systems
    offs = np.concatenate([[0], np.cumsum([s.n for s in systems])])
    voffs = np.concatenate([[0], np.cumsum([s.nnz for s in systems])])
    n_all, nnz_all = int(offs[-1]), int(voffs[-1])
    G = torch.zeros((nnz_all, len(inst) * na), dtype=torch.float64, device=dev)
    S = torch.zeros((n_all, len(inst) * nb), dtype=torch.float64, device=dev)
    primal = torch.zeros(n_all, dtype=torch.float64, device=dev)
    for i, (s, grp, shifts) in enumerate(inst):
        e = np.nonzero(grp >= 0)[0]
        G[torch.as_tensor(voffs[i] + e, device=dev),
          torch.as_tensor(i * na + grp[e], device=dev)] = 1.0
        S[int(offs[i]):int(offs[i + 1]), i * nb:(i + 1) * nb] = torch.as_tensor(shifts.T,
                                                                                  device=dev)
        primal[int(offs[i]):int(offs[i]) + s.n_primal] = 1.0
    v0 = torch.as_tensor(np.concatenate([s.vals for s in systems]), device=dev)
    b0 = torch.as_tensor(np.concatenate([s.rhs[:, 0] for s in systems]), device=dev)
    diag = torch.as_tensor(np.concatenate([s.diag for s in systems]), device=dev)

    th = torch.tensor(theta0, dtype=torch.float64, device=dev, requires_grad=True)
    vals = v0 * (1.0 + G @ th[:, :na].reshape(-1))
    b = b0 + S @ th[:, na:].reshape(-1)
    batch = SparseLDLBatch([CSRMat(s.n, s.n, s.rowp, s.cols, s.vals) for s in systems],
                           order=OrderingType.AMD)
    x = kkt_solve(batch, vals, diag, b)
    loss = 0.5 * ((x * primal) ** 2).sum()
    loss.backward()
    g = th.grad.cpu().numpy()
    inertia = batch.system_inertia()

    for i, (s, grp, shifts) in enumerate(inst):
        assert inertia[i] == s.expected_inertia
        gr = _ref_adjoint_gradient(s, grp, shifts, theta0[i], na)
        assert np.abs(g[i] - gr).max() <= 1e-8 * np.abs(gr).max(), (i, g[i], gr)

    h = 1e-6
    for i in (0, 31, 63):
        s, grp, shifts = inst[i]
        fd = np.zeros(na + nb)
        for j in range(na + nb):
            e = np.zeros(na + nb)
            e[j] = h
            fd[j] = (_ref_loss(s, grp, shifts, theta0[i] + e, na)
                     - _ref_loss(s, grp, shifts, theta0[i] - e, na)) / (2 * h)
        assert np.abs(g[i] - fd).max() <= 1e-5 * np.abs(fd).max(), (i, g[i], fd)


def _perturbed_values(s, seed=123, eps_vals=0.01, eps_sigma=0.3):
    """Values of the same pattern at a neighbouring iterate: entries scaled
    by 1 + eps N(0,1) (the same factor for (i, j) and (j, i)), the positive
    diagonal (Sigma) by exp(eps_sigma N(0,1))."""
    rng = np.random.default_rng(seed)
    r = np.repeat(np.arange(s.n), np.diff(s.rowp))
    key = r.astype(np.int64) * s.n + s.cols
    tkey = s.cols.astype(np.int64) * s.n + r
    order = np.argsort(key)
    pos = order[np.searchsorted(key[order], tkey)]
    f = rng.standard_normal(s.nnz)
    f = 0.5 * (f + f[pos])
    v = s.vals * (1.0 + eps_vals * f)
    d = s.diag.copy()
    m = d > 0
    d[m] *= np.exp(eps_sigma * rng.standard_normal(int(m.sum())))
    return v, d


def test_front_above_the_chained_panel_limit():
    """The 256 x 256 plane-stress system factored with the pivot order of a
    neighbouring iterate: candidates the record no longer suits are delayed
    up to the root, whose front grows past the ~7,100 rows the chained panel
    kernel holds. The root's a-posteriori panels then leave candidates that
    the per-pivot panel kernel finishes with Bunch-Kaufman. Inertia as the
    compiled reference gives it for this system (pinned by the 256 x 256
    parity test in test_gpu_parity.py), backward error at the FP64 level."""
    torch = pytest.importorskip("torch")
    s = plane_stress_kkt(256)
    dev = torch.device("cuda:0")
    vals = torch.as_tensor(s.vals, device=dev)
    diag = torch.as_tensor(s.diag, device=dev)
    ldl = SparseLDL(CSRMat(s.n, s.n, s.rowp, s.cols, vals), order=OrderingType.AMD)
    pv, pd = _perturbed_values(s)
    vals.copy_(torch.as_tensor(pv, device=dev))
    diag.copy_(torch.as_tensor(pd, device=dev))
    assert ldl.factor(Vector(diag)) == 0
    ldl.reuse_pivot_order()
    vals.copy_(torch.as_tensor(s.vals, device=dev))
    diag.copy_(torch.as_tensor(s.diag, device=dev))
    assert ldl.factor(Vector(diag)) == 0
    st = ldl.stats()
    assert st["max_front"] > 7100
    assert tuple(ldl.get_inertia()) == s.expected_inertia
    b = torch.as_tensor(np.ascontiguousarray(s.rhs.T), device=dev).t()
    x = b.t().contiguous().t().clone()
    ldl.solve(x)
    assert backward_error(s, x.cpu().numpy(), s.rhs) <= BERR_TOL
