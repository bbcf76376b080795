"""Parity of the CUDA library with the reference on the GPU.

Golden fixtures hold the reference's own kernels' fields (tests/golden); the oracle
(the C restatement, bit-exact against those kernels) checks the full-size configs.
Tolerance: 1e-9 relative L-infinity on every floating-point field; the wet mask and
the segment tables must match exactly."""
import numpy as np
import pytest

import golden
from helpers import REL_TOL, rel_linf

pytestmark = pytest.mark.gpu

FLOAT_OUT = ("z", "u", "v", "t_z", "t_u", "t_v", "H_moi", "FS", "tFS", "dH", "Htdu", "Htdv", "VTH", "Kx", "Ky",
             "Qbx", "Qby", "ubt", "ubp", "vbt", "vbd", "hi")
INT_OUT = ("khouot", "daui", "cuoii", "moci", "dauj", "cuoij", "mocj")


def _sim(case, solver, monkeypatch):
    from hydist.lib import Simulation
    if solver == "thomas":
        monkeypatch.setenv("HYD_SOLVER", "thomas")
    else:
        monkeypatch.delenv("HYD_SOLVER", raising=False)
    return Simulation.from_case(case)


def _check(sim, get_ref, label, fields=None):
    worst = {}
    for f in FLOAT_OUT:
        if fields is not None and f not in fields:
            continue
        e = rel_linf(sim.get(f), get_ref(f))
        worst[f] = e
        assert e <= REL_TOL, "%s: %s rel L-inf %.3e" % (label, f, e)
    for f in INT_OUT:
        if fields is not None and f not in fields:
            continue
        a, b = sim.get(f), get_ref(f)
        assert np.array_equal(a, b), "%s: %s differs at %s" % (label, f, np.argwhere(a != b)[:3].tolist())
    return worst


@pytest.mark.parametrize("solver", ["partitioned", "thomas"])
@pytest.mark.parametrize("name", golden.names())
def test_gpu_matches_reference_golden(name, solver, monkeypatch):
    case, out = golden.load(name)
    sim = _sim(case, solver, monkeypatch)
    sim.step(case.nsteps)
    _check(sim, lambda f: out[f], "%s/%s" % (name, solver), fields=set(out))


def test_gpu_config1_full_run_vs_oracle(oracle_lib, monkeypatch):
    """Config 1 (400 x 60 channel, dt = 2 s) for the full 1800 steps."""
    import oracle
    from hydist import cases
    c = cases.config1_case()
    sim = _sim(c, "partitioned", monkeypatch)
    ora = oracle.OracleSim(c)
    ora.init()
    for _ in range(6):
        sim.step(300)
        ora.step(300)
        _check(sim, ora.get, "config1 t=%g" % ora.t)
    mb = sim.mass_balance()
    assert mb["nonfinite"] == 0


def test_gpu_config2_resume_vs_oracle(oracle_lib, monkeypatch):
    """Config 2 at full size (1048 x 980): the GPU runs to t = 3590 s (sediment active),
    the oracle resumes from the GPU's state and both run 40 steps across the Exner update
    at t = 3600 s."""
    import oracle
    from hydist import cases
    c = cases.config2_case()
    sim = _sim(c, "partitioned", monkeypatch)
    sim.step(3590)
    ora = oracle.OracleSim(c)
    ora.load_state(sim.get, sim.t, sim.get("hmax"))
    for k in (5, 15, 20):
        sim.step(k)
        ora.step(k)
        _check(sim, ora.get, "config2 t=%g" % ora.t)
    assert np.isfinite(sim.get("z")).all()


def test_gpu_config2_first_steps_vs_oracle(oracle_lib, monkeypatch):
    import oracle
    from hydist import cases
    c = cases.config2_case()
    sim = _sim(c, "partitioned", monkeypatch)
    ora = oracle.OracleSim(c)
    ora.init()
    _check(sim, ora.get, "config2 init")
    for k in (1, 9, 40):
        sim.step(k)
        ora.step(k)
        _check(sim, ora.get, "config2 t=%g" % ora.t)
