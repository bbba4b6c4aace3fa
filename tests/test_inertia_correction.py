"""Inertia correction (Algorithm IC) against the reference's InertiaCorrector.

tests/golden/inertia_correction.json holds what the reference's class did on
scripted systems (tests/golden/make_inertia_golden.py): every factorization's
shifts, the inertia it saw and the perturbed diagonal. The mirror in
amigo_b200.inertia_correction must take exactly the same steps. CPU only:
the solver here is scripted; the GPU test drives the real factorization."""

import json
import os

import numpy as np
import pytest

from amigo_b200.inertia_correction import InertiaCorrector
from tests.ipm_fakes import run_scenario, scenarios

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def ref_runs():
    with open(os.path.join(ROOT, "tests", "golden", "inertia_correction.json")) as f:
        return json.load(f)


def _shifts(c):
    return (c._dw, c._dc)


@pytest.mark.parametrize("name", list(scenarios()))
def test_same_attempts_as_reference(ref_runs, name):
    mine = run_scenario(InertiaCorrector, _shifts, scenarios()[name])
    ref = ref_runs[name]
    assert len(mine) == len(ref)
    for k, (m, r) in enumerate(zip(mine, ref)):
        assert m["ok"] == r["ok"], (name, k)
        assert m["last_delta_w"] == r["last_delta_w"], (name, k)
        assert m["last_delta_c"] == r["last_delta_c"], (name, k)
        assert m["pivtols"] == r["pivtols"], (name, k)
        assert len(m["attempts"]) == len(r["attempts"]), (name, k)
        for a, b in zip(m["attempts"], r["attempts"]):
            assert tuple(a[:4]) == tuple(b[:4]), (name, k)
            assert np.array_equal(a[4], np.array(b[4])), (name, k)  # bit-exact diagonal


@pytest.mark.parametrize("name", list(scenarios()))
def test_device_attempts_skip_only_repeats(ref_runs, name):
    """Attempts through factor_perturbed: the same decisions; an attempt
    whose shifts repeat the previous one's (after the pivot tolerance was
    raised, which this solver ignores) is not refactored."""
    mine = run_scenario(InertiaCorrector, _shifts, scenarios()[name], device=True)
    for k, (m, r) in enumerate(zip(mine, ref_runs[name])):
        assert (m["ok"], m["last_delta_w"], m["last_delta_c"]) == \
            (r["ok"], r["last_delta_w"], r["last_delta_c"]), (name, k)
        want = []
        for b in r["attempts"]:
            if not want or tuple(want[-1][:2]) != tuple(b[:2]):
                want.append(b)
        assert len(m["attempts"]) == len(want), (name, k)
        for a, b in zip(m["attempts"], want):
            assert tuple(a[:4]) == tuple(b[:4]), (name, k)
            assert np.array_equal(a[4], np.array(b[4])), (name, k)


def test_fixture_covers_every_branch(ref_runs):
    """The scripted systems reach the overflow restart with a constraint
    shift, the degeneracy verdicts and a failed correction."""
    ov = ref_runs["primal_shift_overflow"]
    assert not ov[0]["ok"] and not ov[2]["ok"]
    assert any(a[1] > 0 for a in ov[2]["attempts"])  # constraint shift after the overflow
    jac = ref_runs["jacobian_degenerate"]
    assert len(jac[3]["attempts"]) == 1 and jac[3]["attempts"][0][1] > 0  # pre-applied
    hess = ref_runs["hessian_degenerate"]
    assert len(hess[3]["attempts"]) == 1 and hess[3]["attempts"][0][0] > 0


def test_perturbation_entry_points_reject_bad_arguments():
    """Host-side checks of the C ABI, made before any device work."""
    from amigo_b200 import _native
    from amigo_b200.sparse_ldl import CSRMat, SparseLDL
    from amigo_b200.workloads import poisson_2d

    rowp, cols, vals = poisson_2d(5)
    n = len(rowp) - 1
    ldl = SparseLDL(CSRMat(n, n, rowp, cols, vals))
    for primal, dual, why in (([0, n], [1], "out of range"), ([0, 0], [1], "twice"),
                              ([0], [-1], "out of range"), ([0], [2, 2], "twice")):
        with pytest.raises(_native.NativeError, match=why):
            ldl.set_perturbation_rows(primal, dual)
    lib = _native.load()
    st = lib.b200ldl_factor_perturbed(ldl._h, None, None, 0.0, 0.0, None, None)
    assert st < 0 and b"vals is null" in lib.b200ldl_last_error(ldl._h)
    st = lib.b200ldl_copy_perturbed_diagonal(ldl._h, None)
    assert st < 0
