"""FP64 iterative refinement (b200ldl_solve_refine) on the GPU: with the
exact FP64 factor it keeps the backward error at the FP64 level; with the
factor of a perturbed matrix it recovers the backward error against the
exact matrix to the requested tolerance within a few corrections."""

import numpy as np
import pytest

from amigo_b200.sparse_ldl import CSRMat, OrderingType, SparseLDL, Vector
from amigo_b200.workloads import optimal_control_kkt, plane_stress_kkt
from oracle import ref
from tests.conftest import backward_error

pytestmark = pytest.mark.gpu


def _device(torch, s, vals, diag):
    dev = torch.device("cuda:0")
    return (torch.as_tensor(vals, device=dev), torch.as_tensor(diag, device=dev),
            torch.as_tensor(np.ascontiguousarray(s.rhs.T), device=dev).t())


@pytest.mark.parametrize("make", [lambda: optimal_control_kkt(), lambda: plane_stress_kkt(64)],
                         ids=["optimal_control", "plane_stress_64"])
def test_refine_exact_factor(make):
    torch = pytest.importorskip("torch")
    s = make()
    v, d, b = _device(torch, s, s.vals, s.diag)
    ldl = SparseLDL(CSRMat(s.n, s.n, s.rowp, s.cols, v), order=OrderingType.AMD)
    assert ldl.factor(Vector(d)) == 0
    x, berr, iters = ldl.solve_refine(b, max_iter=3, tol=1e-14, diagonal=Vector(d))
    xh = x.cpu().numpy()
    assert backward_error(s, xh, s.rhs) <= 1e-14
    assert np.all(berr <= 1e-14)
    r = ref.RefLDL(s.rowp, s.cols, order=ref.ORDER_AMD)
    r.factor(s.vals, s.diag)
    assert tuple(ldl.get_inertia()) == tuple(r.inertia())
    xr = r.solve(s.rhs)
    assert np.abs(xh - xr).max() / np.abs(xr).max() < 1e-6


def test_refine_recovers_from_a_perturbed_factor():
    torch = pytest.importorskip("torch")
    s = plane_stress_kkt(48)
    rng = np.random.default_rng(5)
    # the factor of values perturbed by 1e-5 (relative), the residual of the
    # exact matrix: an approximate factor, as a mixed-precision one is
    r = np.repeat(np.arange(s.n), np.diff(s.rowp))
    key = r.astype(np.int64) * s.n + s.cols
    tkey = s.cols.astype(np.int64) * s.n + r
    order = np.argsort(key)
    pos = order[np.searchsorted(key[order], tkey)]
    f = rng.standard_normal(s.nnz)
    f = 0.5 * (f + f[pos])
    vp = s.vals * (1.0 + 1e-5 * f)
    vpd, d, b = _device(torch, s, vp, s.diag)
    ldl = SparseLDL(CSRMat(s.n, s.n, s.rowp, s.cols, vpd), order=OrderingType.AMD)
    assert ldl.factor(Vector(d)) == 0
    # one plain solve with the approximate factor misses the target
    x0 = b.clone()
    ldl.solve(x0)
    assert backward_error(s, x0.cpu().numpy(), s.rhs) > 1e-10
    ldl.mat.vals = torch.as_tensor(s.vals, device=vpd.device)
    x, berr, iters = ldl.solve_refine(b, max_iter=10, tol=1e-12, diagonal=Vector(d))
    assert 1 <= iters <= 10
    assert np.all(berr <= 1e-12)
    assert backward_error(s, x.cpu().numpy(), s.rhs) <= 1e-12
