"""Pick-up, the Engine-shaped run loop and the writers through the CUDA library (GPU),
checked against the oracle."""
import os

import numpy as np
import pytest

import golden
from helpers import REL_TOL, rel_linf

pytestmark = pytest.mark.gpu

FIELDS = ("z", "u", "v", "FS", "dH")


class _OracleTarget:
    """Lets hydist.io.load_initial_condition write into an OracleSim."""

    def __init__(self, ora):
        self.ora = ora

    def set(self, name, a):
        self.ora.view(name)[...] = a


def test_gpu_pickup_matches_oracle(tmp_path, oracle_lib):
    import oracle
    from hydist import engine, io
    from hydist.lib import Simulation
    case, _ = golden.load("islands")
    first = Simulation.from_case(case)
    first.step(40)
    io.save_pickup(first, str(tmp_path))
    first.close()
    sim, *_ = engine.gpu_init(case, pick_up=True, pickup_dirs=str(tmp_path))
    ora = oracle.OracleSim(case)
    io.load_initial_condition(_OracleTarget(ora), str(tmp_path), case)
    ora.init_pickup()
    assert np.array_equal(sim.get("khouot"), ora.get("khouot"))
    sim.step(30)
    ora.step(30)
    for f in FIELDS:
        e = rel_linf(sim.get(f), ora.get(f))
        assert e <= REL_TOL, "%s rel L-inf %.3e" % (f, e)
    sim.close()


def test_gpu_engine_run_loop_matches_oracle(tmp_path, oracle_lib):
    import oracle
    from hydist import engine
    case, _ = golden.load("islands")
    p = case.params
    sim, *_ = engine.gpu_init(case)
    u_l, v_l, z_l, fs_l = engine.hydraulic_Calculation(
        400, sim, ketdinh=bool(p.ketdinh), kenhhepd=int(p.kenhhepd), kenhhepng=int(p.kenhhepng), interval=100,
        sediment_start=p.sediment_start, bed_change_start=p.bed_change_start, save_grid=True,
        out_dir=str(tmp_path))
    assert len(z_l) == 4 and len(fs_l) == 1
    ora = oracle.OracleSim(case)
    ora.init()
    ora.step(400)
    for got, f in ((u_l[-1], "u"), (v_l[-1], "v"), (z_l[-1], "z")):
        e = rel_linf(got, ora.get(f))
        assert e <= REL_TOL, "%s rel L-inf %.3e" % (f, e)
    grd = tmp_path / "FS_GPU" / "fs_360.0.grd"
    lines = grd.read_text().splitlines()
    assert lines[0] == "DSAA" and len(lines) == 5 + case.N - 2
    sim.close()


def test_gpu_export_level_file(tmp_path):
    from hydist import io
    from hydist.lib import Simulation
    case, _ = golden.load("islands")
    sim = Simulation.from_case(case)
    t = sim.step(50)
    io.export_velocity_and_level(sim, t, str(tmp_path))
    z = sim.get("z")
    rows = (tmp_path / "water_level" / ("mucnuoc%ss.grid" % t)).read_text().splitlines()
    assert len(rows) == case.N
    assert rows[0].split() == ["%.2f" % z[1, j] for j in range(1, case.M + 1)]
    recs = (tmp_path / "velocity" / ("VTH%ss.data" % t)).read_text().splitlines()
    assert len(recs) == case.N * case.M and recs[0].startswith("%.1f 1 1 " % t)
    sim.close()
