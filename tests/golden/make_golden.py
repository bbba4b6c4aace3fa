"""Generate tests/golden/ldl_cases.npz from the reference's own unit tests.

Runs in the build container only (it reads the reference sources):

    python tests/golden/make_golden.py <reference checkout>

1. Executes ``get_matrix`` and ``get_poisson_2d`` from the reference's
   tests/unit/test_ldl.py (with the compiled ``amigo`` module replaced by a
   recorder of the CSR arrays) to obtain the exact test matrices: the seven
   small dense cases (lines 20-82) and the 2D Poisson matrices n = 10, 20, 50
   after ``np.random.seed(0)`` (lines 85-118, 230-314).
2. Records the expected inertia the reference test asserts
   (``np.linalg.eigh`` counts / (m^2, 0)) and the right-hand side A @ 1.
3. Runs the compiled reference oracle (oracle/_ref/liboracle_ref.so) with
   the test's settings (ustab = 0.4, NATURAL and AMD) and stores its inertia
   and 7-RHS solution, so later runs can pin the oracle without the
   reference sources.
"""

from __future__ import annotations

import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


class _RecCSR:
    def __init__(self, nrows, ncols, rowp, cols, vals):
        self.nrows, self.ncols = nrows, ncols
        self.rowp = np.asarray(rowp, np.int32)
        self.cols = np.asarray(cols, np.int32)
        self.vals = np.asarray(vals, np.float64)


def _load_reference_helpers(ref_root: str):
    src = open(os.path.join(ref_root, "tests", "unit", "test_ldl.py")).read()
    am = types.ModuleType("amigo")
    am.CSRMat = _RecCSR
    sys.modules["amigo"] = am
    ns: dict = {}
    exec(compile(src, "test_ldl.py", "exec"), ns)
    return ns["get_matrix"], ns["get_poisson_2d"]


def main(ref_root: str) -> None:
    from oracle import ref

    get_matrix, get_poisson_2d = _load_reference_helpers(ref_root)
    out = {}
    names = []
    cases = []
    for i in range(7):
        csr, x, rhs, inertia = get_matrix(i)
        cases.append((f"dense{i}", csr, x, rhs, inertia))
    for n in (10, 20, 50):
        np.random.seed(0)
        csr, x, rhs, inertia = get_poisson_2d(n)
        cases.append((f"poisson{n}", csr, x, rhs, inertia))
    nrhs = 7
    for name, csr, x, rhs, inertia in cases:
        names.append(name)
        out[f"{name}/rowp"] = csr.rowp
        out[f"{name}/cols"] = csr.cols
        out[f"{name}/vals"] = csr.vals
        out[f"{name}/x"] = np.asarray(x, np.float64)
        out[f"{name}/rhs"] = np.asarray(rhs, np.float64)
        out[f"{name}/inertia"] = np.asarray(inertia, np.int32)
        for order, oname in ((ref.ORDER_NATURAL, "natural"), (ref.ORDER_AMD, "amd")):
            r = ref.RefLDL(csr.rowp, csr.cols, order=order, ustab=0.4)
            r.factor(csr.vals)
            X = np.tile(np.asarray(rhs, np.float64)[:, None], (1, nrhs))
            out[f"{name}/{oname}/inertia"] = np.asarray(r.inertia(), np.int32)
            out[f"{name}/{oname}/solution"] = r.solve(X)
            r.close()
    out["names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "ldl_cases.npz"), **out)
    print(f"wrote {len(names)} cases")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <reference checkout>")
    main(sys.argv[1])
