"""Morphodynamic feedback (GPU): the bed change applied to the bed, against the oracle and
over the large reach's stated 24 hours.

The reference accumulates dH and never applies it (Sediment_Transport.cu:504, quirk Q5);
with bed_feedback = 0 the library reproduces that (every parity test runs that way).
With bed_feedback = 1 each Exner update (every bed_period s from bed_change_start on)
takes the change morfac x bed_period / (1 - Dorong) x rate, filters it by the 3 x 3
binomial kernel (which removes the grid-scale oscillation of the explicit rate), limits it
to a tenth of the local depth and to 0.05 m, adds it to dH as a Kahan sum and sets
h = h0 + dH, and the set-up's depth-derived fields are re-derived.  The oracle restates
the same option, so the GPU is held to the parity tolerance against it.
"""
import time

import numpy as np
import pytest

from helpers import REL_TOL, rel_linf

pytestmark = pytest.mark.gpu

# config 4's 24 h morphodynamic run, FP32-bulk mixed form against FP64: the bed's stated
# bound (m) and the water budget's closure (relative to the volume)
MIXED_24H_BED_TOL = 0.1
MIXED_24H_CLOSURE = 1e-6  # FP32 rounding of the continuity fluxes (measured 1.3e-7)
# the FP64 run's closure over 24 h (relative to the volume): FP64 rounding of the sums
# (measured 2.5e-14), the bed's share and the cells the sweeps leave unsolved included
FP64_24H_CLOSURE = 1e-10


def _feedback(case, morfac, period):
    p = case.params.copy()
    p.bed_feedback = 1
    p.morfac = float(morfac)
    p.bed_period = float(period)
    case.params = p
    return case


@pytest.mark.parametrize("fixed", [0, 5])
def test_feedback_matches_oracle(oracle_lib, fixed):
    """Islands reach with sediment from t = 0 and a fed-back bed update every 10 s at
    morfac 10: 240 steps (23 updates) on the GPU and on the oracle; with fixed = 5 the bed
    of the cells within 5 cells of the edges, and where the water is shallower than 0.3 m,
    stays put."""
    import oracle
    from hydist import cases
    from hydist.lib import Simulation
    c = _feedback(cases.islands_case(), 10.0, 10.0)
    c.params.bed_fixed = fixed
    c.params.bed_min_depth = 0.3 if fixed else 0.0
    n = 240
    sim = Simulation.from_case(c)
    h_start = sim.get("h")
    sim.step(n)
    ora = oracle.OracleSim(c)
    ora.init()
    ora.step(n)
    for f in ("z", "u", "v", "FS", "dH", "h", "htaiz", "H_moi", "Htdu", "Htdv", "Kx1", "Ky1", "hi"):
        e = rel_linf(sim.get(f), ora.get(f))
        assert e <= REL_TOL, "%s rel L-inf %.3e" % (f, e)
    for f in ("khouot", "moci", "mocj"):
        assert np.array_equal(sim.get(f), ora.get(f)), f
    # the bed moved, by dH
    h = sim.get("h")
    dH = sim.get("dH")
    assert np.isfinite(dH).all()
    assert np.abs(h - h_start).max() > 0
    assert np.allclose(h - h_start, dH, rtol=0, atol=1e-12)
    if fixed:
        N, M = c.N, c.M
        band = np.ones_like(dH, dtype=bool)
        band[2 + fixed:N - fixed + 1, 2 + fixed:M - fixed + 1] = False
        assert np.array_equal(h[band], h_start[band])
    sim.close()


def test_feedback_off_keeps_the_bed():
    """Without feedback the bed never changes and dH only accumulates (quirk Q5)."""
    from hydist import cases
    from hydist.lib import Simulation
    c = cases.islands_case()
    sim = Simulation.from_case(c)
    h0 = sim.get("h")
    sim.step(120)
    assert np.array_equal(sim.get("h"), h0)
    assert np.nanmax(np.abs(sim.get("dH"))) > 0
    sim.close()


def _run_24h(precision):
    from hydist import cases
    from hydist.lib import Simulation
    c = cases.config4_morpho_case()
    p = c.params.copy()
    p.precision_mode = precision
    c.params = p
    sim = Simulation.from_case(c)
    sim.step(1)
    v0 = sim.mass_balance()["volume"]
    b0 = sim.mass_budget()
    t0 = time.perf_counter()
    worst = 0.0
    for hour in range(24):
        sim.step(3600 if hour < 23 else 3599)
        mb = sim.mass_balance()
        assert mb["nonfinite"] == 0, "non-finite values by hour %d" % (hour + 1)
        b = sim.mass_budget()
        dv = mb["volume"] - v0
        pred = (b["net_in"] - b0["net_in"]) + (b["opened"] - b0["opened"]) - (b["closed"] - b0["closed"]) + (
            b["bed"] - b0["bed"]) - (b["leak"] - b0["leak"])
        worst = max(worst, abs(dv - pred) / mb["volume"])
    wall = time.perf_counter() - t0
    assert sim.t == 86400.0
    fields = {f: sim.get(f) for f in ("z", "u", "v", "FS", "dH", "khouot")}
    bed_vol = sim.mass_budget()["bed"]
    sim.close()
    return fields, wall, worst, bed_vol


def test_config4_24h_morfac10():
    """The 4096 x 2048 reach over its stated 24 h (86 400 steps of 1 s) with hydraulics,
    sediment and the bed change fed back at morphological factor 10, the bed updated every
    10 min (cases.config4_morpho_case: steady discharge, fixed stage, with_feedback's
    long-run sediment), in FP64 and in the FP32-bulk mixed form: each finite throughout,
    its water budget closed with the bed's share (the cumulative drift stated), the
    simulated hours per wall second reported, and the mixed form's per-field L-inf and L2
    differences from FP64 at 24 h reported (bounded by MIXED_24H_BED_TOL on the bed)."""
    from hydist.params import PRECISION_FP64, PRECISION_MIXED
    ref, wall, worst, bed_vol = _run_24h(PRECISION_FP64)
    mx = float(np.abs(ref["dH"]).max())
    print("config4 24 h morfac 10, FP64: %.1f s wall, %.2f sim-h/wall-s, max |dH| %.4f m, bed volume to the water "
          "column %.1f m3, closure worst rel %.2e" % (wall, 24.0 / wall, mx, bed_vol, worst))
    # each 10-min update moves a cell's bed by at most 0.05 m (the feedback's limit)
    assert 0 < mx <= 0.05 * 144 + 1e-9
    assert worst <= FP64_24H_CLOSURE
    mix, wall_m, worst_m, _ = _run_24h(PRECISION_MIXED)
    print("  mixed: %.1f s wall (%.2fx FP64), closure worst rel %.2e" % (wall_m, wall / wall_m, worst_m))
    wet = (ref["khouot"] == 0) & (mix["khouot"] == 0)
    for f in ("z", "u", "v", "FS", "dH"):
        d = (mix[f] - ref[f])[wet]
        print("  %-3s L-inf %.3e  L2 (RMS) %.3e" % (f, float(np.abs(d).max()), float(np.sqrt((d * d).mean()))))
    print("  mask cells differing %d" % int((ref["khouot"] != mix["khouot"]).sum()))
    assert worst_m <= MIXED_24H_CLOSURE
    assert float(np.abs(mix["dH"] - ref["dH"]).max()) <= MIXED_24H_BED_TOL
