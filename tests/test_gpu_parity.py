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


def test_gpu_config2_fields_set_mid_run_vs_oracle(oracle_lib, monkeypatch):
    """Fields written between steps (the host round trip of Engine.py's output loop): an
    unchanged write keeps the span-limited step; a velocity written on never-wet cells
    away from every wet run forces whole-grid passes.  Both against the oracle given the
    same writes."""
    import oracle
    from hydist import cases
    c = cases.config2_case()
    sim = _sim(c, "partitioned", monkeypatch)
    sim.step(1850)          # sediment active from t = 1800 s
    ora = oracle.OracleSim(c)
    ora.load_state(sim.get, sim.t, sim.get("hmax"))
    for f in ("z", "u", "v", "FS"):
        sim.set(f, sim.get(f))
    sim.step(10)
    ora.step(10)
    _check(sim, ora.get, "unchanged writes t=%g" % ora.t)
    # a never-wet cell at least 8 cells from any cell that can be wet, in its row and column
    kh = sim.get("khouot")
    N, M = c.N, c.M
    open_ = kh != 2
    i0, j0 = None, None
    for i in range(2, N - 1):
        cols = np.flatnonzero(open_[i])
        for j in range(2, M - 1):
            if kh[i, j] != 2:
                continue
            if cols.size and np.abs(cols - j).min() < 8:
                continue
            if open_[max(i - 8, 0):i + 9, j].any():
                continue
            i0, j0 = i, j
            break
        if i0 is not None:
            break
    assert i0 is not None
    u = sim.get("u")
    u[i0, j0] = 0.05
    sim.set("u", u)
    ora.view("u")[i0, j0] = 0.05
    sim.step(10)
    ora.step(10)
    _check(sim, ora.get, "u written at (%d, %d) t=%g" % (i0, j0, ora.t))
    sim.step(5)
    ora.step(5)
    _check(sim, ora.get, "after the whole-grid pass t=%g" % ora.t)


def test_gpu_config2_full_horizon_vs_oracle(oracle_lib, monkeypatch):
    """Config 2 over its whole stated horizon (the 1 h ramp and 6 h: 25 200 steps, sediment
    from t = 1800 s, seven Exner updates) against the oracle on all host cores, compared
    every two simulated hours and at the end (about two minutes, mostly the oracle)."""
    import os
    import oracle
    from hydist import cases
    c = cases.config2_case()
    sim = _sim(c, "partitioned", monkeypatch)
    ora = oracle.OracleSim(c, threads=os.cpu_count() or 1)
    ora.init()
    for n in (7200, 7200, 7200, 3600):
        sim.step(n)
        ora.step(n)
        _check(sim, ora.get, "config2 t=%g" % ora.t, fields=("z", "u", "v", "t_z", "t_u", "t_v", "H_moi", "FS",
                                                               "dH", "khouot", "moci", "mocj"))
    sim.close()
