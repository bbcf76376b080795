"""Edge cases on the GPU: the grid-size limits, a grid with no water, the smallest grid the
library takes, and a line with more wet segments than the reference's segment_limit (20).
Fields against the oracle within 1e-9 relative L-infinity; the masks exactly."""
import numpy as np
import pytest

from helpers import REL_TOL, rel_linf

pytestmark = pytest.mark.gpu

FIELDS = ("z", "u", "v", "t_z", "t_u", "t_v", "FS", "dH", "H_moi")


def _vs_oracle(case, steps):
    import oracle
    from hydist.lib import Simulation
    sim = Simulation.from_case(case)
    try:
        ora = oracle.OracleSim(case)
        ora.init()
        for k in steps:
            sim.step(k)
            ora.step(k)
            for f in FIELDS:
                e = rel_linf(sim.get(f), ora.get(f))
                assert e <= REL_TOL, "%s t=%g: %s rel L-inf %.3e" % (case.name, ora.t, f, e)
            for f in ("khouot", "moci", "mocj"):
                assert np.array_equal(sim.get(f), ora.get(f)), "%s: %s differs" % (case.name, f)
        return sim.mass_balance()
    finally:
        sim.close()


def test_grid_size_limits_rejected():
    """Fewer than 6 or more than 25000 cells along a direction: a clear error before any
    device allocation."""
    from hydist import cases
    from hydist.lib import HydError, Simulation
    p = cases.islands_case().params
    for N, M in ((5, 36), (48, 5), (25001, 8), (8, 25001)):
        with pytest.raises(HydError, match="grid too"):
            Simulation(p, N, M)


def test_dry_grid_vs_oracle(oracle_lib):
    """No wet cell anywhere (every bed above the water): the step leaves the state as the
    reference's kernels do, and nothing is wet."""
    from hydist import cases
    c = cases.islands_case(N=24, M=20, seed=3)
    c.fields["h"] = np.full_like(c.fields["h"], -1.0) + c.params.NANGDAY
    c.name = "dry24x20"
    mb = _vs_oracle(c, (1, 11))
    assert mb["wet_cells"] == 0 and mb["nonfinite"] == 0


def test_smallest_grid_vs_oracle(oracle_lib):
    """The smallest grid taken (8 x 8 here; the limit is 6): a straight channel with
    hydraulics, sediment from t = 0 and the bed update at t = 5 s."""
    from hydist import cases
    c = cases.meander_case(N=8, M=8, dX=5.0, amp=0.0, width=30.0, depth=2.0, floodplain=1.0,
                           noise_sigma=0.0, Q0=2.0, Q1=2.0, tide_amp=0.05, end_cells=0, hours=1.0,
                           sediment_start=0.0, bed_change_start=5.0, name="small8x8")
    mb = _vs_oracle(c, (1, 4, 7))
    assert mb["wet_cells"] > 0 and mb["nonfinite"] == 0


def test_segment_limit_reported():
    """Wet stripes across a 100-row reach give every column 25 wet runs: more than the 20
    segments a line may hold.  The library reports it (the reference would write past its
    segment tables) instead of stepping on."""
    from hydist import cases
    from hydist.lib import HydError, Simulation
    c = cases.meander_case(N=100, M=16, dX=5.0, amp=0.0, width=60.0, depth=2.0, floodplain=1.0,
                           noise_sigma=0.0, Q0=5.0, Q1=5.0, tide_amp=0.0, end_cells=0, hours=1.0,
                           name="stripes")
    h = c.fields["h"] - c.params.NANGDAY
    rows = np.arange(h.shape[0])
    stripe = ((rows // 2) % 2 == 1)[:, None] & (np.arange(h.shape[1]) > 0)[None, :]
    h[stripe] = -1.0
    c.fields["h"] = h + c.params.NANGDAY
    with pytest.raises(HydError, match="segment_limit"):
        sim = Simulation.from_case(c)
        try:
            sim.step(1)
        finally:
            sim.close()
