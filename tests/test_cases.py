"""Synthetic case generators: layout and well-posedness."""
import numpy as np

from hydist import cases


def _bad_faces(H):
    cell = np.full(H.shape, -1.0)
    cell[1:, 1:] = (H[:-1, :-1] + H[:-1, 1:] + H[1:, :-1] + H[1:, 1:]) * 0.25
    wet = cell > 0
    fu = np.full(H.shape, 1.0)
    fu[:, 1:] = (H[:, :-1] + H[:, 1:]) * 0.5
    fv = np.full(H.shape, 1.0)
    fv[1:, :] = (H[:-1, :] + H[1:, :]) * 0.5
    bu = (fu <= 0) & wet & np.roll(wet, -1, axis=0)
    bv = (fv <= 0) & wet & np.roll(wet, -1, axis=1)
    bu[-1, :] = False
    bv[:, -1] = False
    return int(bu.sum() + bv.sum())


def test_config1_layout():
    c = cases.config1_case()
    assert (c.N, c.M) == (400, 60) and c.params.dT == 2.0 and c.nsteps == 1800
    h = c.fields["h"]
    assert h.shape == (403, 63)
    # banks at +2 m (h = -2) on data columns 0..4 and 55..59 -> array columns 1..5 and 56..60
    assert (h[1:401, 1:6] == -2).all() and (h[1:401, 56:61] == -2).all()
    assert np.allclose(h[1:401, 6:56].mean(axis=1), 3 + 1e-4 * 5 * np.arange(400))
    assert c.boundary_type[cases.EDGE_LEFT, 0] == 2 and c.boundary_type[cases.EDGE_RIGHT, 0] == 1


def test_config2_layout_and_wellposed():
    c = cases.config2_case()
    assert (c.N, c.M) == (1048, 980) and c.params.dT == 1.0
    assert abs(c.notes["wss"] - 0.008) < 2e-5
    assert _bad_faces(c.fields["h"]) == 0
    assert c.params.sediment_start == 1800 and c.params.bed_change_start == 3600


def test_islands_wellposed():
    for seed in (7, 11, 23):
        c = cases.islands_case(seed=seed)
        assert _bad_faces(c.fields["h"]) == 0


def test_config4_layout_and_wellposed():
    """The 4096 x 2048 reach at 2.5 m: config 2's meander scaled x2, dt = 1 s, the tide
    held at 0 through the discharge ramp and then starting from 0."""
    c = cases.config4_case()
    assert (c.N, c.M) == (4096, 2048) and c.params.dX == 2.5 and c.params.dT == 1.0
    assert c.fields["h"].shape == (4099, 2051)
    assert _bad_faces(c.fields["h"] - c.params.NANGDAY) == 0
    zt = c.tables[cases.EDGE_RIGHT][0]
    assert zt[0] == 0 and zt[1] == 0 and zt[2] > 0.4
    q = c.tables[cases.EDGE_LEFT][0]
    assert q[0] == 0 and q[1] == 2 * 2000.0 * cases.CONFIG2_Q_SCALE
    assert c.notes["morfac"] == 10.0
    wet = (c.fields["h"][2:-1, 2:-1] - c.params.NANGDAY) > 0
    assert 0.04 < wet.mean() < 0.08
