"""GPU KKT assembly: the gather kernel's CSR values are bit-identical to the
reference's own add_row assembly (compiled into the oracle) on the same
element blocks, and they feed the factorization on the device."""

import numpy as np
import pytest

from amigo_b200.assembly import CSRAssembly
from amigo_b200.sparse_ldl import CSRMat, OrderingType, SparseLDL, Vector
from oracle import ref
from tests.test_assembly import element_system

pytestmark = pytest.mark.gpu


def test_device_assembly_matches_reference_and_factors():
    import torch

    dev = torch.device("cuda:0")
    rowp, cols, conn, blocks = element_system(seed=5, n=400,
                                              groups=((600, 6), (300, 9), (50, 2)), drop=20)
    asm = CSRAssembly(rowp, cols, conn)
    assert asm.dropped > 0
    want = ref.csr_assemble(rowp, cols, conn, blocks)
    flat = torch.as_tensor(np.concatenate([b.ravel() for b in blocks]), device=dev)
    v1 = asm.values(flat)
    v2 = asm.values([torch.as_tensor(b, device=dev) for b in blocks])
    torch.cuda.synchronize()
    assert np.array_equal(v1.cpu().numpy(), want)
    assert np.array_equal(v2.cpu().numpy(), want)
    # the device values go straight into the factorization
    n = len(rowp) - 1
    diag = np.random.default_rng(7).uniform(0.5, 1.5, n)
    ldl = SparseLDL(CSRMat(n, n, rowp, cols, v1), order=OrderingType.AMD)
    assert ldl.factor(Vector(torch.as_tensor(diag, device=dev))) == 0
    r = ref.RefLDL(rowp, cols, order=int(OrderingType.AMD))
    r.factor(want, diag)
    assert tuple(ldl.get_inertia()) == tuple(r.inertia())
