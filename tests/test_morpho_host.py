"""Host logic of the quasi-steady morphodynamic loop (CPU, no device): the period's
bookkeeping against a scripted stand-in for the Simulation (accept, retry without the
jump, fallback to plain stepping), the forcing interpolation and the case set-up."""
import math

import numpy as np
import pytest


class FakeParams:
    dT = 1.0


class FakeSim:
    """Records the calls; steady_residual returns inf for the snapshot that opens a warm
    phase (the first call after set_time) and the scripted values, in order, after the
    warm steps."""

    def __init__(self, residuals):
        self.params = FakeParams()
        self.t = 7200.0
        self.saved = None
        self.calls = []
        self.res = list(residuals)
        self.opening = False

    def checkpoint(self):
        self.saved = self.t
        self.calls.append("checkpoint")

    def restore(self):
        self.t = self.saved
        self.calls.append("restore")

    def set_time(self, t):
        self.t = t
        self.opening = True
        self.calls.append(("set_time", t))

    def steady_residual(self, snapshot=True):
        if self.opening:
            self.opening = False
            return math.inf, math.inf
        r = self.res.pop(0)
        return r, r

    def step(self, n=1):
        self.t += n * self.params.dT
        self.calls.append(("step", n))

    def mass_balance(self):
        return {"nonfinite": 0}

    def add_levels(self, du, dv, dz, i0, j0):
        self.calls.append("add_levels")


class FakeCase:
    class params:
        bed_period = 600.0


class FakeJump:
    crop = (1, 10, 1, 10)

    def increments(self, sim, Q, stage):
        return (0, 0, 0)


def _qs(sim, jump=None, **kw):
    from hydist import morpho as MO
    MO.forcing_at = lambda case, t: (500.0, 0.0)  # the fake case has no tables
    return MO.QuasiSteady(sim, FakeCase, jump=jump, **kw)


def test_accepted_period_ends_on_the_bed_update_step():
    from hydist import morpho as MO
    keep = MO.forcing_at
    try:
        sim = FakeSim([5e-4, 5e-5])  # steady after the second warm step
        q = _qs(sim, warm=20, gate=1e-4)
        ok, steps = q.period()
        assert ok and steps == 3 and q.accepted == 1 and q.fallbacks == 0
        # warm steps from t_end - 20, then the clock to t_end - 1 and the last step
        assert ("set_time", 7800.0 - 20) in sim.calls and ("set_time", 7799.0) in sim.calls
        assert sim.t == 7800.0
        assert "restore" not in sim.calls
    finally:
        MO.forcing_at = keep


def test_rejected_jump_is_retried_without_it_then_falls_back():
    from hydist import morpho as MO
    keep = MO.forcing_at
    try:
        # the jump's 19 warm steps never pass; the retry from the checkpoint passes at once
        sim = FakeSim([1e-2] * 19 + [5e-5])
        q = _qs(sim, jump=FakeJump(), warm=20, gate=1e-4)
        ok, steps = q.period()
        assert "add_levels" in sim.calls and sim.calls.count("restore") == 1
        assert ok and q.accepted == 1 and q.jump_accepted == 0 and q.fallbacks == 0
        assert steps == 19 + 2 and sim.t == 7800.0
        # a period whose retry fails too is stepped plainly from the checkpoint
        sim2 = FakeSim([1e-2] * 38)
        q2 = _qs(sim2, jump=FakeJump(), warm=20, gate=1e-4)
        ok, steps = q2.period()
        assert not ok and q2.fallbacks == 1 and sim2.calls.count("restore") == 2
        assert sim2.calls[-1] == ("step", 600) and sim2.t == 7800.0
        assert steps == 19 + 19 + 600
        # a jump that passes counts as one
        sim3 = FakeSim([5e-5])
        q3 = _qs(sim3, jump=FakeJump(), warm=20, gate=1e-4)
        ok, steps = q3.period()
        assert ok and q3.jump_accepted == 1 and steps == 2
    finally:
        MO.forcing_at = keep


def test_forcing_at_interpolates_hourly_knots():
    from hydist import cases, morpho as MO
    c = cases.config5_case(days=0.2)
    q = c.tables[cases.EDGE_LEFT][0]
    Q, st = MO.forcing_at(c, 3600.0 * 2 + 900.0)
    assert Q == pytest.approx(q[2] + 0.25 * (q[3] - q[2]))
    assert np.isfinite(st)


def test_config5_case_and_crop():
    from hydist import cases, morpho as MO
    c = cases.config5_case(days=0.5)
    p = c.params
    assert p.bed_feedback == 1 and p.bed_period == 600.0 and p.Toe == cases.MORPHO_TOE
    assert p.bed_fixed == 16 and p.bed_min_depth == cases.MORPHO_MIN_DEPTH
    assert all(float(np.abs(t).max()) == 0.0 for t in c.cc)  # clear-water inflow
    q = c.tables[cases.EDGE_LEFT][0]
    assert q[0] == 0.0 and 500.0 <= q[5] <= 875.0
    i0, rows, j0, cols = MO.reach_crop(c)
    assert (i0, rows) == (1, c.N) and 0 < cols < c.M
    h = c.fields["h"][1:c.N + 1, j0:j0 + cols] - p.NANGDAY
    assert (h > 0).any()
    c4 = cases.config4_morpho_case()
    assert c4.params.morfac == 10.0 and c4.params.bed_fixed == 64
    assert float(np.abs(c4.tables[cases.EDGE_RIGHT]).max()) == 0.0
