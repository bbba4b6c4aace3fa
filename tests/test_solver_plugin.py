"""Host logic of the B200LdlSolver plugin's pivot-order reuse (no GPU): when
the structure is re-planned from the last pivot record. The re-plan drops
the current factor, so it must come right before a factorization and never
between a factorization and its solves."""

import numpy as np

from amigo_b200.solver import B200LdlSolver


class _FakeLDL:
    """Stands in for SparseLDL: records the calls and reports a chosen
    number of delayed pivots for each factorization."""

    def __init__(self, n, delays):
        self.n = n
        self.delays = list(delays)
        self.calls = []
        self._last = 0

    def reuse_pivot_order(self):
        self.calls.append("replan")

    def factor(self, diagonal):
        self.calls.append("factor")
        self._last = self.delays.pop(0)
        return 0

    def factor_perturbed(self, dx, dc, vals, diag):
        self.calls.append("factor")
        self._last = self.delays.pop(0)
        return (1, 1)

    def stats(self):
        return {"delayed": self._last}

    def solve(self, x):
        self.calls.append("solve")


def _solver(ldl, reuse, refresh=0.01):
    s = object.__new__(B200LdlSolver)
    s.hessian = object()
    s.ldl = ldl
    s.reuse_pivot_order = reuse
    s.refresh_delays = refresh
    s._replan = False
    s._planned = False
    return s


def _loop(s, steps):
    for _ in range(steps):
        s.factor(s.hessian, None)
        s.solve(np.zeros(3), np.zeros(3))


def test_no_reuse_never_replans():
    ldl = _FakeLDL(1000, [500, 500, 500])
    _loop(_solver(ldl, False), 3)
    assert "replan" not in ldl.calls


def test_replans_before_the_second_factorization_then_on_stale_records():
    # delays: the first factorization (reference order) delays many; the
    # re-planned ones delay few (no re-plan) until one delays 2% of n
    ldl = _FakeLDL(1000, [500, 3, 4, 20, 5, 6])
    _loop(_solver(ldl, True, refresh=0.01), 6)
    assert ldl.calls == ["factor", "solve",
                         "replan", "factor", "solve",
                         "factor", "solve",
                         "factor", "solve",
                         "replan", "factor", "solve",
                         "factor", "solve"]


def test_replan_only_right_before_a_factorization():
    ldl = _FakeLDL(100, [50, 50, 50, 50])
    s = _solver(ldl, True, refresh=0.0)
    for _ in range(4):
        s.factor(s.hessian, None)
        for _ in range(2):
            s.solve(np.zeros(3), np.zeros(3))
    # every re-plan is immediately followed by a factorization
    for i, c in enumerate(ldl.calls):
        if c == "replan":
            assert ldl.calls[i + 1] == "factor"
    assert ldl.calls.count("replan") == 3
