"""The allocation-free dense solve, checked against the regular entry points.

Some callers cannot allocate device memory once they are running: a
real-time loop that re-solves a small KKT system every few milliseconds,
where an allocation has unbounded latency and may synchronize the device,
or a plugin inside a process whose framework already holds the device
memory. b200ldl_dense_solve_noalloc serves them: inputs and outputs come
from the caller, and the working matrix is a fixed array inside the library.

This test calls it through the C ABI on two different systems in a row (the
second call reuses the array the first one left behind) and compares each
solution and inertia with the regular create / factor / solve entry points
on the same matrix. It needs nothing from earlier tests, so it passes alone
in a fresh process and after the rest of the suite.
"""

import ctypes

import numpy as np
import pytest

from amigo_b200 import _native
from amigo_b200.sparse_ldl import CSRMat, OrderingType, SparseLDL
from amigo_b200.workloads import dense_to_csr

pytestmark = pytest.mark.gpu

BERR_TOL = 1e-12   # backward error bound used by the GPU parity tests
REL_TOL = 1e-6     # forward agreement bound used by the GPU parity tests


def _dense_kkt(nprim, ncon, nrhs, seed):
    rng = np.random.default_rng(seed)
    m = rng.standard_normal((nprim, nprim))
    h = m @ m.T / nprim + np.eye(nprim)
    a = rng.standard_normal((ncon, nprim))
    k = np.zeros((nprim + ncon, nprim + ncon))
    k[:nprim, :nprim] = h
    k[nprim:, :nprim] = a
    k[:nprim, nprim:] = a.T
    k[nprim:, nprim:] = -1e-8 * np.eye(ncon)
    return k, rng.standard_normal((nprim + ncon, nrhs))


def _backward_error(k, x, b):
    r = b - k @ x
    den = np.abs(k).sum(axis=1).max() * np.abs(x).max(axis=0) + np.abs(b).max(axis=0)
    return float(np.max(np.abs(r).max(axis=0) / den))


def test_noalloc_dense_solve_matches_regular_path():
    torch = pytest.importorskip("torch")
    lib = _native.load()
    dev = torch.device("cuda:0")
    for nprim, ncon, seed in ((150, 90, 0), (300, 200, 1)):
        k, b = _dense_kkt(nprim, ncon, 3, seed)
        n = k.shape[0]

        # regular entry points: create (symbolic), factor, solve, inertia
        rowp, cols, vals = dense_to_csr(k)
        ldl = SparseLDL(CSRMat(n, n, rowp, cols, vals), order=OrderingType.AMD)
        assert ldl.factor() == 0
        x_ref = np.asfortranarray(b.copy())
        ldl.solve(x_ref)
        inertia_ref = tuple(ldl.get_inertia())
        assert inertia_ref == (nprim, ncon)

        # allocation-free entry point on device buffers owned by the caller
        a_dev = torch.as_tensor(np.ascontiguousarray(k.T), device=dev)  # column-major
        b_dev = torch.as_tensor(np.ascontiguousarray(b.T), device=dev)  # n x 3 column-major
        inertia_dev = torch.zeros(2, dtype=torch.int32, device=dev)
        st = lib.b200ldl_dense_solve_noalloc(
            n, ctypes.c_void_p(a_dev.data_ptr()), n, ctypes.c_void_p(b_dev.data_ptr()), n,
            b.shape[1], ctypes.c_void_p(inertia_dev.data_ptr()), None)
        assert st == 0
        torch.cuda.synchronize()
        x = b_dev.cpu().numpy().T
        assert tuple(int(v) for v in inertia_dev.cpu()) == inertia_ref
        assert _backward_error(k, x, b) <= BERR_TOL
        rel = np.abs(x - x_ref).max() / np.abs(x_ref).max()
        assert rel < REL_TOL, rel


def test_noalloc_rejects_sizes_beyond_its_array():
    lib = _native.load()
    # rejected before any device work, so no buffers are needed
    assert lib.b200ldl_dense_solve_noalloc(513, None, 513, None, 513, 1, None, None) == -6
