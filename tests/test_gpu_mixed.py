"""The FP32-bulk mixed form (precision_mode = HYD_PRECISION_MIXED) against the FP64 form.

The mixed form runs the coefficient assembly, both line sweeps, the explicit momentum and
the sediment transport in FP32; the sweeps solve for the level increment z' - z, and the
continuity update z' = z + increment, the mass sums and the Exner accumulation stay FP64.
Its error is stated per field (L-infinity and RMS over the interior) against the FP64
oracle on the small reach and against the library's FP64 form (itself within 2e-12 of the
oracle, test_gpu_parity) on configs 2 and 4.  The bounds below are the stated tolerance of
the mixed form, not of the FP64 parity path.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("z", "u", "v", "FS", "dH", "H_moi")
# stated tolerances of the mixed form against FP64, L-infinity and RMS over the interior in
# the field's units (m, m/s, FS's volume fraction, m), on the configured reaches (configs 2
# and 4: measured z 2.1e-3 m L-inf, 1.5e-5 m RMS at t = 4200 s on config 4)
LINF_BOUND = {"z": 5e-3, "u": 0.02, "v": 0.02, "FS": 1e-6, "dH": 1e-6, "H_moi": 5e-3}
RMS_BOUND = {"z": 1e-4, "u": 1e-4, "v": 1e-4, "FS": 1e-8, "dH": 1e-8, "H_moi": 1e-4}
# the islands reach is the stress case: a 3-5 cm shelf that wets and dries every tidal
# cycle, where the friction term divides by the face depth; measured z 2.0e-2 m L-inf,
# 3.1e-3 m RMS after 240 steps against the FP64 oracle
ISLANDS_LINF = {"z": 3e-2, "u": 0.15, "v": 0.15, "FS": 1e-5, "dH": 2e-4, "H_moi": 3e-2}
ISLANDS_RMS = {"z": 5e-3, "u": 1.5e-2, "v": 1.5e-2, "FS": 1e-6, "dH": 1e-5, "H_moi": 5e-3}
# the mixed form's continuity rows take FP32 fluxes while the budget sums the FP64 fields:
# the water budget closes to FP32 rounding per step (measured 2.4e-9 relative over 4200
# steps of config 4, 4.1e-9 on config 2)
MIXED_CLOSURE = 1e-7


def _mixed(case):
    from hydist.params import PRECISION_MIXED
    p = case.params.copy()
    p.precision_mode = PRECISION_MIXED
    return p


def field_errors(get_a, get_b, N, M):
    out = {}
    for f in FIELDS:
        a = get_a(f)[2:N + 1, 2:M + 1]
        b = get_b(f)[2:N + 1, 2:M + 1]
        m = np.isfinite(a) & np.isfinite(b)
        d = np.abs(a[m] - b[m])
        out[f] = (float(d.max()) if d.size else 0.0, float(np.sqrt((d ** 2).mean())) if d.size else 0.0)
    return out


def _report(label, errs, mask_diff):
    print("%s: mask cells differing %d" % (label, mask_diff))
    for f, (linf, rms) in errs.items():
        print("  %-6s L-inf %.3e  RMS %.3e" % (f, linf, rms))


def _check(errs, linf_bound=LINF_BOUND, rms_bound=RMS_BOUND):
    for f, (linf, rms) in errs.items():
        assert np.isfinite(linf)
        assert linf <= linf_bound[f], "%s: L-inf %.3e over %.1e" % (f, linf, linf_bound[f])
        assert rms <= rms_bound[f], "%s: RMS %.3e over %.1e" % (f, rms, rms_bound[f])


def test_mixed_islands_vs_oracle(oracle_lib):
    """The islands reach (wetting and drying, sediment from t = 0, Exner updates) for 240
    steps in the mixed form against the FP64 oracle."""
    import oracle
    from hydist import cases
    from hydist.lib import Simulation
    c = cases.islands_case()
    n = 240
    sim = Simulation(_mixed(c), c.N, c.M)
    sim.load_case(c)
    sim.step(n)
    ora = oracle.OracleSim(c)
    ora.init()
    ora.step(n)
    errs = field_errors(sim.get, ora.get, c.N, c.M)
    md = int((sim.get("khouot") != ora.get("khouot")).sum())
    _report("islands mixed vs oracle", errs, md)
    _check(errs, ISLANDS_LINF, ISLANDS_RMS)
    sim.close()


@pytest.mark.parametrize("name,steps", [("config2", 4200), ("config4", 4200)])
def test_mixed_vs_fp64(name, steps):
    """Configs 2 and 4 from t = 0 through the ramp, the sediment start (1800 s) and the
    first Exner update (3600 s) to t = 4200 s, in both forms; the water budget of the
    mixed form is closed like the FP64 one's."""
    from hydist import cases
    from hydist.lib import Simulation
    c = getattr(cases, name + "_case")()
    a = Simulation.from_case(c)
    b = Simulation(_mixed(c), c.N, c.M)
    b.load_case(c)
    for sim in (a, b):
        sim.step(1)
    v0 = b.mass_balance()["volume"]
    b0 = b.mass_budget()
    a.step(steps - 1)
    b.step(steps - 1)
    errs = field_errors(b.get, a.get, c.N, c.M)
    md = int((a.get("khouot") != b.get("khouot")).sum())
    mb = b.mass_balance()
    bb = b.mass_budget()
    pred = (bb["net_in"] - b0["net_in"]) + (bb["opened"] - b0["opened"]) - (bb["closed"] - b0["closed"]) + (
        bb["bed"] - b0["bed"]) - (bb["leak"] - b0["leak"])
    closure = abs(mb["volume"] - v0 - pred) / mb["volume"]
    vol_rel = abs(mb["volume"] - a.mass_balance()["volume"]) / a.mass_balance()["volume"]
    _report("%s mixed vs FP64 at t = %d s (closure %.2e, volume rel diff %.2e)" % (name, steps, closure, vol_rel),
            errs, md)
    _check(errs)
    assert mb["nonfinite"] == 0
    assert closure <= MIXED_CLOSURE
    a.close()
    b.close()
