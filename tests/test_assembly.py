"""KKT assembly: the host plan against the reference's own add_row assembly
(compiled into the oracle), on CPU. Summing every CSR entry's planned
contributions in plan order must give the reference's values bit for bit;
the GPU test runs the same plan in the kernel."""

import numpy as np
import pytest

from amigo_b200 import _native
from amigo_b200.assembly import CSRAssembly
from amigo_b200.workloads import csr_from_coo
from oracle import ref


def element_system(seed=0, n=60, groups=((40, 4), (25, 6), (3, 1)), drop=0):
    """Random component groups over n variables, their symmetric element
    blocks, and the CSR pattern of their union (minus `drop` off-diagonal
    pairs, so that some contributions fall outside the pattern)."""
    rng = np.random.default_rng(seed)
    conn, blocks, rows, cols = [], [], [], []
    for ne, m in groups:
        c = np.stack([rng.choice(n, size=m, replace=False) for _ in range(ne)]).astype(np.int32)
        b = rng.standard_normal((ne, m, m))
        b = b + np.transpose(b, (0, 2, 1))
        conn.append(c)
        blocks.append(b)
        for e in range(ne):
            rows.extend(np.repeat(c[e], m))
            cols.extend(np.tile(c[e], m))
    r = np.array(rows)
    k = np.array(cols)
    if drop:
        off = np.flatnonzero(r != k)
        pick = rng.choice(off, size=drop, replace=False)
        bad = set(zip(r[pick], k[pick])) | set(zip(k[pick], r[pick]))
        keep = np.array([(a, b) not in bad for a, b in zip(r, k)])
        r, k = r[keep], k[keep]
    rowp, colsp, _ = csr_from_coo(n, r, k, np.ones(len(r)))
    return rowp, colsp, conn, blocks


def plan_sum(asm, blocks):
    ptr, src = asm.plan()
    flat = np.concatenate([b.ravel() for b in blocks])
    out = np.zeros(asm.nnz)
    for p in range(asm.nnz):
        v = 0.0
        for s in src[ptr[p]:ptr[p + 1]]:
            v += flat[s]
        out[p] = v
    return out


@pytest.mark.parametrize("drop", [0, 12])
def test_plan_sums_bit_exact_with_reference_add_row(drop):
    rowp, cols, conn, blocks = element_system(seed=drop, drop=drop)
    asm = CSRAssembly(rowp, cols, conn)
    want = ref.csr_assemble(rowp, cols, conn, blocks)
    assert np.array_equal(plan_sum(asm, blocks), want)
    total = sum(c.shape[0] * c.shape[1] ** 2 for c in conn)
    assert asm.nvals == total and asm.kept + asm.dropped == total
    assert (asm.dropped > 0) == (drop > 0)


def test_plan_keeps_the_reference_order():
    """Every entry's contributions come in (group, element, column, row)
    order: their flat block positions increase."""
    rowp, cols, conn, _ = element_system(seed=3)
    ptr, src = CSRAssembly(rowp, cols, conn).plan()
    for p in range(len(ptr) - 1):
        assert np.all(np.diff(src[ptr[p]:ptr[p + 1]]) > 0)


def test_create_rejects_bad_input():
    rowp, cols, conn, _ = element_system(seed=1)
    bad = [c.copy() for c in conn]
    bad[0][0, 0] = len(rowp) - 1  # variable index out of range
    with pytest.raises(_native.NativeError, match="out of range"):
        CSRAssembly(rowp, cols, bad)
    unsorted = cols.copy()
    unsorted[[0, 1]] = unsorted[[1, 0]]
    with pytest.raises(_native.NativeError, match="not sorted"):
        CSRAssembly(rowp, unsorted, conn)
