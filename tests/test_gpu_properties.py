"""Size-independent properties of the CUDA path at full size: determinism, checkpoint
round trip, finiteness and volume bookkeeping."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _config2():
    from hydist import cases
    return cases.config2_case()


def test_deterministic_bitwise():
    from hydist.lib import Simulation
    c = _config2()
    a = Simulation.from_case(c)
    b = Simulation.from_case(c)
    a.step(200)
    b.step(200)
    for f in ("z", "u", "v", "FS", "khouot", "H_moi"):
        assert np.array_equal(a.get(f), b.get(f)), f


def test_checkpoint_roundtrip_bitwise():
    from hydist.lib import Simulation
    c = _config2()
    a = Simulation.from_case(c)
    a.step(1850)          # sediment active from t = 1800 s
    state = a.get_state()
    a.step(25)
    ref = {f: a.get(f) for f in ("z", "u", "v", "FS", "dH", "khouot")}
    b = Simulation(c.params, c.N, c.M)
    b.set_boundary(c.boundary_type, c.tables, c.cc, c.total_time)
    b.set_state(state)
    assert b.t == 1850.0
    b.step(25)
    for f, v in ref.items():
        assert np.array_equal(b.get(f), v, equal_nan=True), f


def test_volume_responds_to_inflow():
    """Water volume grows while the discharge ramps up against a fixed downstream stage."""
    from hydist.lib import Simulation
    c = _config2()
    a = Simulation.from_case(c)
    v0 = a.mass_balance()["volume"]
    a.step(600)
    mb = a.mass_balance()
    assert mb["nonfinite"] == 0
    assert mb["volume"] > v0


def test_step_argument_errors():
    from hydist.lib import HydError, Simulation
    c = _config2()
    a = Simulation.from_case(c)
    with pytest.raises(HydError):
        a.step(10 ** 9)   # beyond the boundary tables
    with pytest.raises((HydError, ValueError)):
        a.set("z", np.zeros((3, 3)))


def test_async_level_reads_match_sync_reads():
    """hyd_get_field_async snapshots the field in order with the steps: each buffer holds
    the levels of the step it followed, although later steps run during the copies."""
    from hydist.lib import Simulation
    c = _config2()
    a = Simulation.from_case(c)
    b = Simulation.from_case(c)
    shape = (c.N + 3, c.M + 3)
    bufs = [np.empty(shape) for _ in range(5)]
    want = []
    for k in range(5):
        a.step(3, sync=False)
        a.get_async("z", bufs[k])
        b.step(3)
        want.append(b.get("z"))
        if k >= 2:  # two later calls have returned: the read of call k - 2 is complete
            assert np.array_equal(bufs[k - 2], want[k - 2]), k - 2
    a.wait_fields()
    for k in range(5):
        assert np.array_equal(bufs[k], want[k]), k
    with pytest.raises(Exception):
        a.get_async("khouot", np.empty(shape))
    a.close()
    b.close()


def test_update_boundary_changes_forcing():
    """Tables sent between steps drive the following steps like tables set at the start."""
    from hydist.lib import Simulation
    c = _config2()
    tabs2 = [t * 1.1 for t in c.tables]
    a = Simulation.from_case(c)
    a.update_boundary(tabs2, c.cc)
    a.step(20)
    c2 = _config2()
    c2.tables = tabs2
    b = Simulation.from_case(c2)
    b.step(20)
    for f in ("z", "u", "v"):
        assert np.array_equal(a.get(f), b.get(f)), f
    a.close()
    b.close()


@pytest.mark.parametrize("name", ["z", "u"])
def test_mirror_matches_sync_reads(name):
    """hyd_mirror_update_async keeps a host copy equal to the field after every step while
    copying only the box of cells a span-limited step can change: across whole-grid steps
    (the first ones, and after a field write) and span-limited ones, with sediment and the
    Exner update (bed change from t = 10 s on this reach)."""
    from hydist import cases
    from hydist.lib import Simulation
    c = cases.islands_case(N=96, M=72, seed=11, bed_change_start=10.0)
    a = Simulation.from_case(c)
    b = Simulation.from_case(c)
    a.mirror_open(name)
    full = (c.N + 3) * (c.M + 3) * 8
    moved = []
    views = []
    for k in range(24):
        a.step(1, sync=False)
        view, n = a.mirror_update()
        moved.append(n)
        b.step(1)
        want = b.get(name)
        views.append((view, want))
        if k >= 1:  # the next update has returned: the copy of update k - 1 is complete
            v, w = views[k - 1]
            assert np.array_equal(v, w), (name, k - 1)
        if k == 12:  # a field write (whole-grid event) in both
            u = b.get("u")
            a.set("u", u)
            b.set("u", u)
    a.wait_fields()
    v, w = views[-1]
    assert np.array_equal(v, w)
    # whole copies after the set-up and the write, boxes in between
    assert moved[0] == full and min(moved[3:12]) < full
    a.mirror_close()
    a.close()
    b.close()
