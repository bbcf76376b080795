"""Long lines against the oracle on the GPU: the large single reach (config 4, 4096 x 2048
at 2.5 m, the longest columns about 5,100 tridiagonal rows) and the global-scratch
sweeps, which a line takes when its rows do not fit a sweep CTA's shared memory.
Tolerance: 1e-9 relative L-infinity on every floating-point field; the wet mask and the
segment tables must match exactly."""
import numpy as np
import pytest

from helpers import REL_TOL, rel_linf

pytestmark = pytest.mark.gpu

FLOAT_OUT = ("z", "u", "v", "t_z", "t_u", "t_v", "H_moi", "FS", "tFS", "dH", "Htdu", "Htdv", "VTH", "Kx", "Ky")
INT_OUT = ("khouot", "moci", "mocj", "daui", "cuoii", "dauj", "cuoij")


def _check(sim, ora, label):
    for f in FLOAT_OUT:
        e = rel_linf(sim.get(f), ora.get(f))
        assert e <= REL_TOL, "%s: %s rel L-inf %.3e" % (label, f, e)
    for f in INT_OUT:
        a, b = sim.get(f), ora.get(f)
        assert np.array_equal(a, b), "%s: %s differs at %s" % (label, f, np.argwhere(a != b)[:3].tolist())


def _longest_column_cells(sim):
    kh = sim.get("khouot")
    return int((kh[2:-1, 2:-1] == 0).sum(0).max())


@pytest.fixture(scope="module")
def config4():
    from hydist import cases
    return cases.config4_case()


def test_gpu_config4_first_steps_vs_oracle(oracle_lib, config4, monkeypatch):
    import oracle
    from hydist.lib import Simulation
    monkeypatch.delenv("HYD_SWEEP_ROWS", raising=False)
    monkeypatch.delenv("HYD_SOLVER", raising=False)
    sim = Simulation.from_case(config4)
    try:
        # the UZ sweep's longest columns take the two-level CTA solve with thousands of rows
        assert _longest_column_cells(sim) > 2000
        ora = oracle.OracleSim(config4)
        ora.init()
        _check(sim, ora, "config4 init")
        for k in (1, 4):
            sim.step(k)
            ora.step(k)
            _check(sim, ora, "config4 t=%g" % ora.t)
    finally:
        sim.close()


def test_gpu_config4_resume_vs_oracle(oracle_lib, config4, monkeypatch):
    """The GPU runs config 4 to t = 1850 s (sediment active), the oracle resumes from the
    GPU's state and both run 6 more steps."""
    import oracle
    from hydist.lib import Simulation
    monkeypatch.delenv("HYD_SWEEP_ROWS", raising=False)
    monkeypatch.delenv("HYD_SOLVER", raising=False)
    sim = Simulation.from_case(config4)
    try:
        sim.step(1850)
        ora = oracle.OracleSim(config4)
        ora.load_state(sim.get, sim.t, sim.get("hmax"))
        sim.step(6)
        ora.step(6)
        _check(sim, ora, "config4 t=%g" % ora.t)
        assert sim.mass_balance()["nonfinite"] == 0
    finally:
        sim.close()


def test_gpu_config4_bed_update_vs_oracle(oracle_lib, config4, monkeypatch):
    """The bench's window on config 4: the GPU runs to t = 3590 s, the oracle resumes from
    the GPU's state and both run across the Exner update at t = 3600 s."""
    import oracle
    from hydist.lib import Simulation
    monkeypatch.delenv("HYD_SWEEP_ROWS", raising=False)
    monkeypatch.delenv("HYD_SOLVER", raising=False)
    sim = Simulation.from_case(config4)
    try:
        sim.step(3590)
        ora = oracle.OracleSim(config4)
        ora.load_state(sim.get, sim.t, sim.get("hmax"))
        sim.step(12)
        ora.step(12)
        _check(sim, ora, "config4 t=%g" % ora.t)
        dH = sim.get("dH")
        assert np.abs(dH[np.isfinite(dH)]).max() > 0  # the bed update ran
    finally:
        sim.close()


def test_gpu_global_scratch_sweeps_vs_oracle(oracle_lib, monkeypatch):
    """Config 2 with at most 512 rows of a line in shared memory: its long columns (up to
    about 1,300 rows) and long sediment lines run in the sweep CTAs' global scratch
    regions.  Against the oracle from t = 1850 s (sediment active)."""
    import oracle
    from hydist import cases
    from hydist.lib import Simulation
    c = cases.config2_case()
    monkeypatch.setenv("HYD_SWEEP_ROWS", "512")
    monkeypatch.delenv("HYD_SOLVER", raising=False)
    sim = Simulation.from_case(c)
    monkeypatch.delenv("HYD_SWEEP_ROWS")
    try:
        assert _longest_column_cells(sim) > 300  # lines of more than 512 rows
        sim.step(1850)
        ora = oracle.OracleSim(c)
        ora.load_state(sim.get, sim.t, sim.get("hmax"))
        for k in (3, 7):
            sim.step(k)
            ora.step(k)
            _check(sim, ora, "global scratch t=%g" % ora.t)
    finally:
        sim.close()
