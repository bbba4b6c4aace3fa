"""Generate tests/golden/inertia_correction.json from the reference's own
inertia corrector.

Runs in the build container only (it reads the reference sources):

    python tests/golden/make_inertia_golden.py [/path/to/reference]

Loads amigo/algorithm/solvers/inertia_correction.py (plain Python, no
imports) straight from the reference tree and drives its InertiaCorrector
through the scripted systems of tests/ipm_fakes.py (every branch of
Algorithm IC: the primal-shift schedule, its overflow, and the Jacobian,
Hessian and combined degeneracy tests). For every system it records each
factorization's shifts (delta_w, delta_c), the inertia the scripted solver
returned and the perturbed diagonal, then the result and the final shifts.
"""

from __future__ import annotations

import importlib.util
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tests.ipm_fakes import run_scenario, scenarios  # noqa: E402


def load_reference(ref_root):
    path = os.path.join(ref_root, "amigo", "algorithm", "solvers", "inertia_correction.py")
    spec = importlib.util.spec_from_file_location("ref_inertia_correction", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.InertiaCorrector


def main(argv):
    if len(argv) != 2:
        sys.exit("usage: python tests/golden/make_inertia_golden.py <reference checkout>")
    ref_root = argv[1]
    cls = load_reference(ref_root)
    out = {}
    for name, systems in scenarios().items():
        res = run_scenario(cls, lambda c: (c._delta_x_curr, c._delta_c_curr), systems)
        for r in res:
            r["attempts"] = [[dw, dc, npos, nneg, list(map(float, d))]
                             for dw, dc, npos, nneg, d in r["attempts"]]
        out[name] = res
    path = os.path.join(HERE, "inertia_correction.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=None, separators=(",", ":"))
    print(f"wrote {path}: " + ", ".join(f"{k} {len(v)} systems, "
                                        f"{sum(len(r['attempts']) for r in v)} attempts"
                                        for k, v in out.items()))


if __name__ == "__main__":
    main(sys.argv)
