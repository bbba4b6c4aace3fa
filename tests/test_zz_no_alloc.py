"""The allocation-free dense solve, checked against the oracle and the regular
entry points.

Some callers cannot allocate device memory once they are running: a
real-time loop that re-solves a small KKT system every few milliseconds,
where an allocation has unbounded latency and may synchronize the device,
or a plugin inside a process whose framework already holds the device
memory. b200ldl_dense_solve_noalloc serves them: inputs and outputs come
from the caller, and the working matrix is a fixed array inside the library.

The tests call it through the C ABI:
  - on the reference's own unit-test matrices (tests/golden/ldl_cases.npz:
    exact inertia, 7 right-hand sides of A x = A 1 to 1e-11);
  - on KKT systems ordered constraints first with -1e-8 on their diagonal
    and a zero Hessian on half the primal variables, so that Bunch-Kaufman
    must interchange rows and take 2x2 pivots (checked with a restatement of
    its pivot rule), against the compiled reference oracle and the regular
    create / factor / solve entry points;
  - twice in a row on different systems (the second call reuses the array
    the first one left behind);
  - with padded leading dimensions and garbage in the unread upper triangle,
    and with no right-hand side.
Nothing here depends on earlier tests, so the file passes alone in a fresh
process and after the rest of the suite.
"""

import ctypes

import numpy as np
import pytest

from amigo_b200 import _native
from amigo_b200.sparse_ldl import CSRMat, OrderingType, SparseLDL
from amigo_b200.workloads import dense_to_csr
from oracle import ref

pytestmark = pytest.mark.gpu

BERR_TOL = 1e-12   # backward error bound used by the GPU parity tests
REL_TOL = 1e-6     # forward agreement bound used by the GPU parity tests
GOLDEN_TOL = 1e-11  # the reference's unit tests (tests/unit/test_ldl.py:230-314)


def _constraint_first_kkt(nprim, ncon, nrhs, seed):
    """[[-1e-8 I, A], [A^T, H]] with the constraints first and H diagonal,
    zero on every other primal variable."""
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((ncon, nprim))
    h = np.abs(rng.standard_normal(nprim)) + 0.1
    h[::2] = 0.0
    n = nprim + ncon
    k = np.zeros((n, n))
    k[:ncon, :ncon] = -1e-8 * np.eye(ncon)
    k[:ncon, ncon:] = a
    k[ncon:, :ncon] = a.T
    k[ncon:, ncon:] = np.diag(h)
    return k, rng.standard_normal((n, nrhs))


def _bk_pivots(a):
    """Numbers of 2x2 pivots and of row interchanges that Bunch-Kaufman
    pivoting (the published dsytf2 rule on the lower triangle, alpha =
    (1 + sqrt(17)) / 8) takes on the symmetric matrix a."""
    a = np.array(a, dtype=np.float64)
    n = a.shape[0]
    alpha = (1.0 + np.sqrt(17.0)) / 8.0
    k = two = swaps = 0
    while k < n:
        col = np.abs(a[k + 1:, k])
        colmax = col.max() if col.size else 0.0
        imax = k + 1 + int(np.argmax(col)) if col.size else k
        akk = abs(a[k, k])
        kp, ks = k, 1
        if max(akk, colmax) == 0.0:
            pass
        elif akk < alpha * colmax:
            row = np.abs(np.concatenate([a[imax, k:imax], a[imax + 1:, imax]]))
            rowmax = row.max()
            if akk >= alpha * colmax * (colmax / rowmax):
                pass
            elif abs(a[imax, imax]) >= alpha * rowmax:
                kp = imax
            else:
                kp, ks = imax, 2
        kk = k + ks - 1
        if kp != kk:
            swaps += 1
            a[[kk, kp], :] = a[[kp, kk], :]
            a[:, [kk, kp]] = a[:, [kp, kk]]
        if ks == 1:
            if a[k, k] != 0.0:
                l = a[k + 1:, k] / a[k, k]
                a[k + 1:, k + 1:] -= np.outer(l, a[k + 1:, k])
        else:
            d = a[k:k + 2, k:k + 2]
            w = a[k + 2:, k:k + 2]
            a[k + 2:, k + 2:] -= w @ np.linalg.solve(d, w.T)
            two += 1
        k += ks
    return two, swaps


def _backward_error(k, x, b):
    r = b - k @ x
    den = np.abs(k).sum(axis=1).max() * np.abs(x).max(axis=0) + np.abs(b).max(axis=0)
    return float(np.max(np.abs(r).max(axis=0) / den))


def _noalloc(torch, k, b, lda=None, garbage=False):
    """One call on caller-owned device buffers; returns (status, x, inertia)."""
    lib = _native.load()
    dev = torch.device("cuda:0")
    n = k.shape[0]
    lda = n if lda is None else lda
    nrhs = b.shape[1]
    abuf = np.full((n, lda), np.nan if garbage else 0.0)  # row c = column c, column-major
    abuf[:, :n] = k.T
    if garbage:
        abuf[np.triu_indices(n, 1)[1], np.triu_indices(n, 1)[0]] = np.nan  # strict upper
    bbuf = np.full((max(nrhs, 1), lda), np.nan if garbage else 0.0)
    bbuf[:nrhs, :n] = b.T
    a_dev = torch.as_tensor(abuf, device=dev)
    b_dev = torch.as_tensor(bbuf, device=dev)
    inertia_dev = torch.full((2,), -1, dtype=torch.int32, device=dev)
    st = lib.b200ldl_dense_solve_noalloc(
        n, ctypes.c_void_p(a_dev.data_ptr()), lda, ctypes.c_void_p(b_dev.data_ptr()), lda,
        nrhs, ctypes.c_void_p(inertia_dev.data_ptr()), None)
    torch.cuda.synchronize()
    x = b_dev.cpu().numpy()[:nrhs, :n].T.copy()
    return st, x, tuple(int(v) for v in inertia_dev.cpu())


def test_noalloc_golden_unit_cases(golden):
    torch = pytest.importorskip("torch")
    for name in golden["names"]:
        if not str(name).startswith("dense"):
            continue
        rowp, cols, vals = (golden[f"{name}/{key}"] for key in ("rowp", "cols", "vals"))
        n = len(rowp) - 1
        k = np.zeros((n, n))
        k[np.repeat(np.arange(n), np.diff(rowp)), cols] = vals
        b = np.tile(golden[f"{name}/rhs"][:, None], (1, 7))
        st, x, inertia = _noalloc(torch, k, b)
        assert st == 0, name
        assert inertia == tuple(int(v) for v in golden[f"{name}/inertia"]), name
        assert np.abs(x - golden[f"{name}/x"][:, None]).max() < GOLDEN_TOL, name


def test_noalloc_dense_solve_matches_oracle_and_regular_path():
    torch = pytest.importorskip("torch")
    for nprim, ncon, seed in ((150, 90, 0), (300, 200, 1)):
        k, b = _constraint_first_kkt(nprim, ncon, 3, seed)
        n = k.shape[0]
        two, swaps = _bk_pivots(k)
        assert two >= 1 and swaps >= 1, (two, swaps)

        # the compiled reference (oracle) and the regular entry points
        rowp, cols, vals = dense_to_csr(k)
        r = ref.RefLDL(rowp, cols, order=ref.ORDER_AMD)
        r.factor(vals)
        x_oracle = r.solve(b)
        assert tuple(r.inertia()) == (nprim, ncon)
        ldl = SparseLDL(CSRMat(n, n, rowp, cols, vals), order=OrderingType.AMD)
        assert ldl.factor() == 0
        x_reg = np.asfortranarray(b.copy())
        ldl.solve(x_reg)

        # the allocation-free entry point, twice in a row over the loop
        st, x, inertia = _noalloc(torch, k, b)
        assert st == 0
        assert inertia == tuple(r.inertia()) == tuple(ldl.get_inertia())
        assert _backward_error(k, x, b) <= BERR_TOL
        for other in (x_oracle, x_reg):
            rel = np.abs(x - other).max() / np.abs(other).max()
            assert rel < REL_TOL, rel


def test_noalloc_padded_buffers_and_no_rhs():
    torch = pytest.importorskip("torch")
    k, b = _constraint_first_kkt(60, 40, 2, 7)
    st, x, inertia = _noalloc(torch, k, b)
    assert st == 0
    # leading dimensions n + 7 with NaN in the padding and in the strict upper
    # triangle, which the entry point does not read
    st2, x2, inertia2 = _noalloc(torch, k, b, lda=k.shape[0] + 7, garbage=True)
    assert st2 == 0 and inertia2 == inertia
    assert np.array_equal(x2, x)
    # no right-hand side: only the inertia is produced
    st3, _, inertia3 = _noalloc(torch, k, np.zeros((k.shape[0], 0)))
    assert st3 == 0 and inertia3 == inertia


def test_noalloc_rejects_sizes_beyond_its_array():
    lib = _native.load()
    # rejected before any device work, so no buffers are needed
    assert lib.b200ldl_dense_solve_noalloc(513, None, 513, None, 513, 1, None, None) == -6
