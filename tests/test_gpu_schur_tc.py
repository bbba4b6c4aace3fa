"""The tensor-core Schur-complement update (tcgen05, 3xTF32 products with
FP32 accumulation in tensor memory) against the same update in FP64."""

import ctypes

import numpy as np
import pytest

from amigo_b200 import _native

pytestmark = pytest.mark.gpu

# 3xTF32 products carry about 21 significant bits and the sum is accumulated
# in FP32: the error of each entry is bounded by a small multiple of
# 2^-21 sum_c |a_ic b_jc| (plus FP32 rounding of the partial sums)
REL_TOL = 2e-5


def _update(torch, a, b, c, lower):
    lib = _native.load()
    dev = torch.device("cuda:0")
    m, k = a.shape
    n = b.shape[0]
    ta = torch.as_tensor(np.asfortranarray(a).T.copy(), device=dev)  # column-major m x k
    tb = torch.as_tensor(np.asfortranarray(b).T.copy(), device=dev)
    tc = torch.as_tensor(np.asfortranarray(c).T.copy(), device=dev)
    st = lib.b200ldl_schur_update_tc(m, n, k, ctypes.c_void_p(ta.data_ptr()), m,
                                     ctypes.c_void_p(tb.data_ptr()), n,
                                     ctypes.c_void_p(tc.data_ptr()), m, int(lower), None)
    assert st == 0
    return tc.cpu().numpy().T


@pytest.mark.parametrize("m,n,k,lower", [(128, 128, 32, 0), (300, 250, 70, 0), (257, 257, 129, 1),
                                         (40, 520, 8, 0)])
def test_schur_update_matches_fp64(m, n, k, lower):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(m * 7 + n + k)
    a = rng.standard_normal((m, k)) * np.exp(rng.uniform(-3, 3, (m, 1)))
    b = rng.standard_normal((n, k)) * np.exp(rng.uniform(-3, 3, (n, 1)))
    c = rng.standard_normal((m, n))
    got = _update(torch, a, b, c, lower)
    want = c - a @ b.T
    scale = np.abs(a) @ np.abs(b).T
    err = np.abs(got - want) / np.maximum(scale, 1e-300)
    if lower:
        iu = np.triu_indices(m, 1, n)
        assert np.array_equal(got[iu], c[iu])  # the strict upper triangle is untouched
        il = np.tril_indices(m, 0, n)
        assert err[il].max() < REL_TOL, err[il].max()
    else:
        assert err.max() < REL_TOL, err.max()
