"""Mass balance closed (GPU): the domain's water volume against the library's budget, and
the domain sums of hyd_mass_balance against numpy sums over the oracle's fields.

Both sweeps' continuity rows are in flux form (UVZSolver_multithread.cu:345-349, 402-406),
so between two times the volume (hyd_mass_balance out[0]: the depths of the wet interior
cells) changes by the volume that crossed the open edges plus the cells the wetting pass
opened minus those the drying pass closed (support_funcs.cu:75-186).  hyd_mass_budget
accumulates those terms on the device every half-step; the closure tolerance below is
set by FP64 rounding of the sums, not by the scheme.  The boundary-only closure (no
wet/dry terms) is reported as well: it is what a budget that ignores wetting and drying
would see.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CLOSURE_TOL = 1e-10  # relative to the volume


def _closure(sim, steps, chunk):
    """Volume and budget after one step (the first step sets H_moi), then every `chunk`
    steps; returns the worst relative closure errors (with and without wet/dry terms)."""
    sim.step(1)
    v0 = sim.mass_balance()["volume"]
    b0 = sim.mass_budget()
    worst, worst_bnd, done = 0.0, 0.0, 1
    rows = []
    while done < steps:
        n = min(chunk, steps - done)
        sim.step(n)
        done += n
        mb = sim.mass_balance()
        assert mb["nonfinite"] == 0
        b = sim.mass_budget()
        dv = mb["volume"] - v0
        net = b["net_in"] - b0["net_in"]
        wd = (b["opened"] - b0["opened"]) - (b["closed"] - b0["closed"]) + (b["bed"] - b0["bed"]) - (
            b["leak"] - b0["leak"])
        err = abs(dv - net - wd) / mb["volume"]
        err_bnd = abs(dv - net) / mb["volume"]
        worst = max(worst, err)
        worst_bnd = max(worst_bnd, err_bnd)
        rows.append((done, mb["volume"], dv, net, wd, err))
    return worst, worst_bnd, rows


def test_budget_closes_config1_full_run():
    """Config 1 (400 x 60 channel, Q = 150 m3/s in, stage out), its 1800 steps."""
    from hydist import cases
    from hydist.lib import Simulation
    c = cases.config1_case()
    sim = Simulation.from_case(c)
    worst, worst_bnd, rows = _closure(sim, c.nsteps, 300)
    print("config1 closure: worst rel %.3e (boundary only %.3e); last %s" % (worst, worst_bnd, rows[-1]))
    assert worst <= CLOSURE_TOL
    # the channel fills: the inflow carried water in
    b = sim.mass_budget()
    assert b["gross_in"] > 0 and b["edge_net"][2] > 0
    sim.close()


def test_budget_closes_config2_with_wetting_and_drying():
    """Config 2 (1048 x 980 meander) through its discharge ramp, the start of the tide and
    the first hour with sediment: 3600 steps, with cells wetting and drying on the banks."""
    from hydist import cases
    from hydist.lib import Simulation
    c = cases.config2_case()
    sim = Simulation.from_case(c)
    worst, worst_bnd, rows = _closure(sim, 3600, 600)
    b = sim.mass_budget()
    print("config2 closure: worst rel %.3e (boundary only %.3e); opened %.1f m3 closed %.1f m3; last %s" % (
        worst, worst_bnd, b["opened"], b["closed"], rows[-1]))
    assert worst <= CLOSURE_TOL
    assert b["opened"] > 0  # the banks wetted
    sim.close()


def test_budget_closes_islands_with_levels_set_on_unsolved_cells():
    """The islands reach (a shelf that wets and dries, a stage edge): the segment scan leaves
    wet cells of the last two rows or columns out of a sweep, and the stage boundary still
    sets their level; the budget's leak term carries both the flux into those cells and the
    level change put on them, and closes to FP64 rounding (without the level change the
    residual reached 1e-6 of the volume within minutes)."""
    from hydist import cases
    from hydist.lib import Simulation
    sim = Simulation.from_case(cases.islands_case())
    worst, worst_bnd, rows = _closure(sim, 1200, 100)
    b = sim.mass_budget()
    print("islands closure: worst rel %.3e (boundary only %.3e); leak term %.3e m3; last %s" % (
        worst, worst_bnd, b["leak"], rows[-1]))
    assert worst <= CLOSURE_TOL
    assert b["leak"] != 0.0  # the unsolved cells were exercised
    sim.close()


def test_mass_balance_sums_match_numpy_over_oracle_fields(oracle_lib):
    """hyd_mass_balance's domain sums against numpy sums over the oracle's fields after the
    same steps (sediment and an Exner update active)."""
    import golden
    import oracle
    from hydist.lib import Simulation
    case, _ = golden.load("islands")
    sim = Simulation.from_case(case)
    sim.step(case.nsteps)
    ora = oracle.OracleSim(case)
    ora.init()
    ora.step(case.nsteps)
    N, M = case.N, case.M
    kh = ora.get("khouot")[2:N + 1, 2:M + 1]
    H = ora.get("H_moi")[2:N + 1, 2:M + 1]
    FS = ora.get("FS")[2:N + 1, 2:M + 1]
    dH = ora.get("dH")[2:N + 1, 2:M + 1]
    wet = kh == 0
    area = case.params.dX * case.params.dY
    vol = H[wet].sum() * area
    sus = (FS[wet] * H[wet]).sum() * area
    bed = dH[np.isfinite(dH)].sum() * area
    mb = sim.mass_balance()
    assert mb["wet_cells"] == int(wet.sum())
    assert mb["nonfinite"] == 0
    for got, want in ((mb["volume"], vol), (mb["suspended"], sus), (mb["bed_change"], bed)):
        assert abs(got - want) <= 1e-9 * max(abs(want), 1e-300), (got, want)
    sim.close()
