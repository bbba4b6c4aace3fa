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


@pytest.mark.parametrize("n,groups", [(400, ((600, 6), (300, 9), (50, 2))),
                                      (3000, ((3000, 8), (400, 12)))],
                         ids=["small_fronts", "big_fronts"])
def test_factor_from_element_blocks(n, groups):
    """b200ldl_factor_elements assembles the fronts from the element blocks
    through the assembly plan, never forming the CSR values; the fronts get
    the same bits as from the CSR values, so the factorization (and its
    solution) is bit-identical to CSRAssembly.values followed by factor, on
    the reference's pivot sequence and after pivot-order reuse (the
    a-posteriori panels)."""
    import torch

    from amigo_b200._native import NativeError

    dev = torch.device("cuda:0")
    rowp, cols, conn, blocks = element_system(seed=9, n=n, groups=groups, drop=20)
    asm = CSRAssembly(rowp, cols, conn)
    flat = torch.as_tensor(np.concatenate([b.ravel() for b in blocks]), device=dev)
    vals = asm.values(flat)
    rng = np.random.default_rng(3)
    diag = torch.as_tensor(rng.uniform(0.5, 1.5, n), device=dev)
    rhs = torch.as_tensor(rng.standard_normal(n), device=dev)
    via_csr = SparseLDL(CSRMat(n, n, rowp, cols, vals), order=OrderingType.AMD)
    direct = SparseLDL(CSRMat(n, n, rowp, cols, vals), order=OrderingType.AMD)

    def solutions():
        assert via_csr.factor(Vector(diag)) == 0
        assert direct.factor_elements(asm, flat, Vector(diag)) == 0
        x1, x2 = rhs.clone(), rhs.clone()
        via_csr.solve(x1)
        direct.solve(x2)
        assert tuple(via_csr.get_inertia()) == tuple(direct.get_inertia())
        return x1.cpu().numpy(), x2.cpu().numpy()

    x1, x2 = solutions()
    assert np.array_equal(x1, x2)
    if n > 1000:
        assert direct.stats()["max_front"] > 640  # the big-front assembly ran
    via_csr.reuse_pivot_order()
    direct.reuse_pivot_order()
    x1, x2 = solutions()
    assert np.array_equal(x1, x2)
    r = ref.RefLDL(rowp, cols, order=int(OrderingType.AMD))
    r.factor(asm.values(flat).cpu().numpy(), diag.cpu().numpy())
    assert tuple(direct.get_inertia()) == tuple(r.inertia())
    # the mixed mode refines against CSR values, which this path never forms
    direct.set_precision("mixed")
    with pytest.raises(NativeError):
        direct.factor_elements(asm, flat, Vector(diag))
