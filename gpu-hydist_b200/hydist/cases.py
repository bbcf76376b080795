"""Synthetic cases in the reference's input layout.

The reference loads a real reach (Global_Variables.py:27-133): topography ``h``
(depth below datum, positive down, defined on cell corners), roughness ``hsnham``,
viscosity ``VISCOINDX``, sediment friction ``Fw``, each transposed, flipped and
edge-padded to ``(N+3, M+3)``; boundary types per edge (``boundary_type.txt``:
0 wall, 1 stage Z, 2 discharge Q) and hourly boundary tables per edge segment.
The generators here build the same arrays from closed-form geometry with a fixed
seed; no dataset is needed.  A data array ``d`` of shape (N, M) is placed like the
reference places its input maps: ``np.pad(d, ((1, 2), (1, 2)), 'edge')``.
"""
from dataclasses import dataclass, field
import math

import numpy as np

from .params import default_params, derive, settling_velocity

SEGMENT_LIMIT = 20
EDGE_UP, EDGE_DOWN, EDGE_LEFT, EDGE_RIGHT = 0, 1, 2, 3
GRID_FIELDS = ("h", "hsnham", "VISCOIDX", "Fw", "Tsxw", "Tsyw", "u", "v", "z", "FS")


@dataclass
class Case:
    name: str
    N: int
    M: int
    params: object
    fields: dict
    boundary_type: np.ndarray
    tables: list
    cc: list
    total_time: int
    t_start: float = 0.0
    nsteps: int = 1
    notes: dict = field(default_factory=dict)

    @property
    def shape(self):
        return (self.N + 3, self.M + 3)

    def nseg(self):
        return [int(t.shape[0]) for t in self.tables]

    def interior_cells(self):
        return self.N * self.M


def pad_edge(d):
    """Edge padding of an (N, M) input map to (N+3, M+3) (Global_Variables.py:71-89)."""
    return np.pad(np.asarray(d, dtype=np.float64), ((1, 2), (1, 2)), "edge")


def _prismatic_ends(h):
    """Make the first two and the last two cross-sections identical.

    The reference weights a discharge edge by pow(face depth, 5/3) of the corner
    depths on the edge row (support_funcs.cu:451-511); with identical first two rows
    a cell is wet exactly where its edge face depth is positive, so the weights are
    finite.  The same is done at the outflow end."""
    h[0, :] = h[1, :]
    h[-1, :] = h[-2, :]
    return h


def _heal_faces(h, fill=0.05, max_iter=50):
    """Raise corner depths so that every cell face between two wet cells has a positive
    mean corner depth.

    The reference's Manning factor pow(face depth, -2*mu_mn) (support_funcs.cu:53-57) is
    NaN or infinite on such a face, and a wet cell next to it then produces NaN
    velocities; measured bathymetry is smooth enough not to contain such faces.
    Cells are wet when their four-corner mean is positive (support_funcs.cu:42)."""
    for _ in range(max_iter):
        H = pad_edge(h)
        n1, m1 = H.shape
        cell = np.full(H.shape, -1.0)
        cell[1:, 1:] = (H[:-1, :-1] + H[:-1, 1:] + H[1:, :-1] + H[1:, 1:]) * 0.25
        wet = cell > 0
        bad = np.zeros(H.shape, dtype=bool)
        # face between (i, j) and (i+1, j): corners H[i, j-1], H[i, j]
        fu = np.full(H.shape, 1.0)
        fu[:, 1:] = (H[:, :-1] + H[:, 1:]) * 0.5
        bu = (fu <= 0) & wet & np.roll(wet, -1, axis=0)
        # face between (i, j) and (i, j+1): corners H[i-1, j], H[i, j]
        fv = np.full(H.shape, 1.0)
        fv[1:, :] = (H[:-1, :] + H[1:, :]) * 0.5
        bv = (fv <= 0) & wet & np.roll(wet, -1, axis=1)
        bu[-1, :] = False
        bv[:, -1] = False
        if not (bu.any() or bv.any()):
            return h
        for i, j in np.argwhere(bu):
            for jj in (j - 1, j):
                bad[i, jj] = True
        for i, j in np.argwhere(bv):
            for ii in (i - 1, i):
                bad[ii, j] = True
        bad &= H <= 0
        for i, j in np.argwhere(bad):
            a = min(max(i - 1, 0), h.shape[0] - 1)
            b = min(max(j - 1, 0), h.shape[1] - 1)
            h[a, b] = fill
    return h


def _tables(btype_row, values_per_seg, total_time):
    nseg = max(1, int(np.count_nonzero(btype_row)))
    t = np.zeros((nseg, total_time), dtype=np.float64)
    for k in range(nseg):
        t[k, :] = values_per_seg[k] if k < len(values_per_seg) else values_per_seg[-1]
    return t


def _gaussian_field(rng, shape, sigma_cells, std):
    """Gaussian-correlated noise (periodic FFT filter), scaled to standard deviation `std`."""
    w = rng.standard_normal(shape)
    ky = np.fft.fftfreq(shape[0])[:, None]
    kx = np.fft.rfftfreq(shape[1])[None, :]
    filt = np.exp(-2.0 * (math.pi * sigma_cells) ** 2 * (kx ** 2 + ky ** 2))
    f = np.fft.irfft2(np.fft.rfft2(w) * filt, s=shape)
    f -= f.mean()
    s = f.std()
    return f * (std / s) if s > 0 else f


def channel_case(N=400, M=60, dX=5.0, dT=2.0, bank=5, depth=3.0, slope=1e-4, bank_height=2.0,
                 manning=0.025, Q=150.0, hours=1, z_out=0.0, name="channel"):
    """Straight channel (the repo's horizontal-channel test): x along i, banks across j.

    Bed z_b = -depth - slope*x (x from upstream), so h = depth + slope*x; the first and
    last `bank` cross cells are dry banks at +bank_height.  Upstream (left edge, i=2)
    discharge Q, downstream (right edge, i=N) stage z_out, walls up/down.  No sediment.
    """
    p = default_params(dX=dX, dY=dX, dT=dT, sediment_start=1e12, bed_change_start=1e12)
    derive(p)
    x = np.arange(N, dtype=np.float64)[:, None] * dX
    h = np.repeat(depth + slope * x, M, axis=1)
    h[:, :bank] = -bank_height
    h[:, M - bank:] = -bank_height
    shape = (N + 3, M + 3)
    fields = {
        "h": pad_edge(h) + p.NANGDAY,
        "hsnham": pad_edge(np.full((N, M), manning)),
        "VISCOIDX": pad_edge(np.full((N, M), 1e-6)),
        "Fw": np.zeros(shape),
        "Tsxw": np.zeros(shape),
        "Tsyw": np.zeros(shape),
        "u": np.zeros(shape),
        "v": np.zeros(shape),
        "z": np.zeros(shape),
        "FS": np.zeros(shape),
    }
    bt = np.zeros((4, SEGMENT_LIMIT), dtype=np.int32)
    bt[EDGE_LEFT, 0] = 2
    bt[EDGE_RIGHT, 0] = 1
    total_time = int(hours) + 3
    tables = [
        np.zeros((1, total_time)),
        np.zeros((1, total_time)),
        _tables(bt[EDGE_LEFT], [Q], total_time),
        _tables(bt[EDGE_RIGHT], [z_out], total_time),
    ]
    cc = [np.zeros((1, total_time)) for _ in range(4)]
    nsteps = int(round(hours * 3600 / dT))
    return Case(name, N, M, p, fields, bt, tables, cc, total_time, 0.0, nsteps,
                notes={"Q": Q, "bank_cells": bank})


def meander_case(N=1048, M=980, dX=5.0, dT=1.0, hours=6.0, seed=20261203, amp=120.0,
                 wavelength=1500.0, width=150.0, depth=8.0, floodplain=1.5, noise_sigma=0.2,
                 noise_len=50.0, manning=0.025, manning_spread=0.10, Q0=2000.0, Q1=3500.0,
                 tide_amp=1.0, tide_period_h=12.42, d50=1e-4, Sx=2.7125, cc_in=0.2,
                 sediment_start=1800.0, bed_change_start=3600.0, y_center=None, spinup_h=0.0,
                 end_cells=8, tide_delay_h=0.0, name="meander"):
    """Seeded meandering reach with a parabolic channel, floodplain and bed noise.

    Centreline y = y_c + amp*sin(2*pi*x/wavelength); parabolic section of `width` and
    `depth`, floodplain at +floodplain; Gaussian-correlated bed noise (sigma, length);
    lognormal Manning n.  Upstream (left edge) discharge rising as a half-cosine from
    Q0 to Q1 over `hours`; downstream (right edge) tidal stage; walls up/down.
    Single-grain cohesive sediment (d50, Sx chosen so that wss() = 0.0080 m/s),
    inflow concentration cc_in, sediment from `sediment_start`, bed change from
    `bed_change_start`.  The reference's hourly tables are linearly interpolated
    (support_funcs.cu:547-565), so the boundary forcing is given at hourly knots.

    The first and last `end_cells` cross-sections are rectangular (full depth across
    the channel width) and blend into the parabola over the next `end_cells`.

    With spinup_h > 0 the discharge first ramps linearly from 0 to Q0 over spinup_h
    hours (the scheme cannot carry the bore of an impulsive start at Q0 into water at
    rest) and the stated hydrograph follows.  With tide_delay_h > 0 the stage stays at 0
    for that many hours and the tide starts from there.  sediment_start and bed_change_start are
    absolute times: the reference's Exner step divides by the speed VTH that only the
    sediment phase computes (Sediment_Transport.cu:365-374), so the bed must not start
    changing before the sediment does.
    """
    rng = np.random.default_rng(seed)
    p = default_params(dX=dX, dY=dX, dT=dT, dm=d50, Sx=Sx, Ks=2.5 * d50,
                       sediment_start=sediment_start,
                       bed_change_start=bed_change_start, ketdinh=1)
    derive(p)
    x = np.arange(N, dtype=np.float64)[:, None] * dX
    y = np.arange(M, dtype=np.float64)[None, :] * dX
    yc = (M * dX / 2.0 if y_center is None else y_center) + amp * np.sin(2 * math.pi * x / wavelength)
    d = np.abs(y - yc)
    half = width / 2.0
    zb = np.where(d <= half, -depth * (1.0 - (d / half) ** 2), floodplain)
    if end_cells > 0:
        # rectangular inlet/outlet sections blended into the parabola: the reference
        # derives the stage-edge velocity from continuity divided by the edge face
        # depth (UVZSolver_multithread.cu:720), which shallow bank cells make unstable
        rect = np.where(d <= half, -depth, floodplain)
        a = np.arange(N, dtype=np.float64)[:, None]
        dist = np.minimum(a, N - 1 - a)
        w = np.clip((2.0 * end_cells - dist) / end_cells, 0.0, 1.0)
        zb = w * rect + (1.0 - w) * zb
    zb = zb + _gaussian_field(rng, (N, M), noise_len / dX, noise_sigma)
    h = -zb
    _prismatic_ends(h)
    _heal_faces(h)
    n = manning * np.exp(manning_spread * rng.standard_normal((N, M)))
    hpos = np.maximum(h, 0.1)
    fw = np.where(h > 0, p.g * n ** 2 / hpos ** (1.0 / 3.0), 0.0)
    shape = (N + 3, M + 3)
    fields = {
        "h": pad_edge(h) + p.NANGDAY,
        "hsnham": pad_edge(n),
        "VISCOIDX": pad_edge(np.full((N, M), 1e-6)),
        "Fw": pad_edge(fw),
        "Tsxw": np.zeros(shape),
        "Tsyw": np.zeros(shape),
        "u": np.zeros(shape),
        "v": np.zeros(shape),
        "z": np.zeros(shape),
        "FS": np.zeros(shape),
    }
    bt = np.zeros((4, SEGMENT_LIMIT), dtype=np.int32)
    bt[EDGE_LEFT, 0] = 2
    bt[EDGE_RIGHT, 0] = 1
    total_time = int(math.ceil(hours + spinup_h)) + 3
    th = np.arange(total_time, dtype=np.float64)
    tr = np.clip(th - spinup_h, 0.0, hours)
    q = Q0 + (Q1 - Q0) * 0.5 * (1.0 - np.cos(math.pi * tr / hours))
    if spinup_h > 0:
        q = np.where(th < spinup_h, Q0 * th / spinup_h, q)
    zt = np.where(th >= tide_delay_h, tide_amp * np.sin(2 * math.pi * (th - tide_delay_h) / tide_period_h), 0.0)
    tables = [np.zeros((1, total_time)), np.zeros((1, total_time)), q[None, :].copy(), zt[None, :].copy()]
    cc = [np.zeros((1, total_time)), np.zeros((1, total_time)),
          np.full((1, total_time), cc_in), np.zeros((1, total_time))]
    nsteps = int(round((hours + spinup_h) * 3600 / dT))
    return Case(name, N, M, p, fields, bt, tables, cc, total_time, 0.0, nsteps,
                notes={"wss": settling_velocity(p), "seed": seed, "spinup_steps": int(round(spinup_h * 3600 / dT)),
                       "end_cells": end_cells})


def islands_case(N=48, M=36, dX=5.0, dT=1.0, seed=7, hours=1.0, sediment_start=0.0,
                 bed_change_start=10.0, name="islands"):
    """Small irregular reach for parity tests: random islands give several wet segments
    per line, single-cell segments, shallow cells that dry and re-wet, a discharge edge
    and a stage edge; sediment and bed change active within a few steps."""
    rng = np.random.default_rng(seed)
    c = meander_case(N=N, M=M, dX=dX, dT=dT, hours=hours, seed=seed, amp=M * dX * 0.15,
                     wavelength=N * dX * 0.7, width=M * dX * 0.55, depth=3.0, floodplain=1.0,
                     noise_sigma=0.05, noise_len=3 * dX, Q0=40.0, Q1=60.0, tide_amp=0.3,
                     tide_period_h=2.0, sediment_start=sediment_start,
                     bed_change_start=bed_change_start, name=name)
    h = c.fields["h"][1:N + 1, 1:M + 1].copy()
    # a shallow shelf that wets and dries with the tide
    shelf = (h > 0) & (h < 0.8)
    h[shelf] = 0.03 + 0.02 * rng.random(int(shelf.sum()))
    # 2x2-corner islands in deep water: each blocks one cell and splits the lines through it
    k = max(1, (N * M) // 120)
    ii = rng.integers(4, N - 5, size=k)
    jj = rng.integers(4, M - 5, size=k)
    for a, b in zip(ii, jj):
        if (h[a - 1:a + 3, b - 1:b + 3] > 1.0).all():
            h[a:a + 2, b:b + 2] = -0.5
    _prismatic_ends(h)
    _heal_faces(h)
    c.fields["h"] = pad_edge(h) + c.params.NANGDAY
    c.fields["Fw"] = pad_edge(np.where(h > 0, 0.004, 0.0))
    return c


def steps_for(case, hours):
    return int(round(hours * 3600 / case.params.dT))


# --------------------------------------------------------------------------------
# Named workloads

def config1_case():
    """Plain FP64 hydraulics, straight channel 400 x 60, dx = 5 m, dt = 2 s, 1800 steps."""
    return channel_case(N=400, M=60, dX=5.0, dT=2.0, bank=5, depth=3.0, slope=1e-4, bank_height=2.0,
                        manning=0.025, Q=150.0, hours=1, z_out=0.0, name="config1_channel")


CONFIG2_Q_SCALE = 0.25


def config2_case(spinup_h=1.0, q_scale=CONFIG2_Q_SCALE):
    """Meandering reach 1048 x 980, dx = 5 m, dt = 1 s, hydraulics + sediment + bed change.

    Stated geometry, grid, time step, roughness, tide, sediment and start times.  Three
    changes make the run stable under the reference's own scheme (the oracle and the
    reference's kernels both reach NaN otherwise): a one-hour discharge ramp from rest,
    rectangular inlet/outlet sections, and the 2000 -> 3500 m3/s hydrograph scaled by
    `q_scale` (at full scale the explicit central-difference cross-advection develops a
    2-cell oscillation once velocities pass about 2.5 m/s)."""
    return meander_case(N=1048, M=980, dX=5.0, dT=1.0, hours=6.0, spinup_h=spinup_h,
                        Q0=2000.0 * q_scale, Q1=3500.0 * q_scale, name="config2_meander")


def config4_case(spinup_h=1.0, q_scale=CONFIG2_Q_SCALE, hours=24.0, dT=1.0, end_cells=32, tide_delay_h=None,
                 tide_amp=1.0):
    """Large single reach 4096 x 2048, dx = 2.5 m, hydraulics + sediment + bed change.

    The config-2 meander scaled x2 in length and width: centreline amplitude 240 m,
    wavelength 3000 m, channel width 300 m (depth 8 m and floodplain +1.5 m unchanged),
    bed-noise correlation length 100 m, rectangular end sections of 32 cells (80 m).
    The hydrograph is config 2's (with its stability scale) times 2, the channel width
    ratio, so that velocities match config 2's.  Sediment from t = 1800 s, bed change
    from t = 3600 s, as in config 2.

    No time step is stated for this workload; dt = 1 s as in config 2.  One change keeps
    the reference's own scheme finite here: the tide starts after the discharge ramp
    (tide_delay_h = spinup_h).  Started with the ramp, the rising tide of this 4x larger
    reach pours more water in at the stage edge than the ramped discharge carries out,
    and under that inflow the scheme's stage-edge velocity at the channel's bank cell
    grows without bound: the oracle reaches NaN by t = 1100 s (at dt = 0.5 s by
    t = 1600 s).  With the delay the run stays finite (checked for 4 h at dt = 1 s and
    dt = 0.5 s).  The morphological factor 10 of this workload is kept in
    notes["morfac"]; the parity runs leave the bed unchanged (the reference's behaviour),
    and the morphodynamic runs set bed_feedback with morfac = notes["morfac"]."""
    c = meander_case(N=4096, M=2048, dX=2.5, dT=dT, hours=hours, spinup_h=spinup_h, amp=240.0,
                     wavelength=3000.0, width=300.0, noise_len=100.0,
                     Q0=2000.0 * q_scale * 2.0, Q1=3500.0 * q_scale * 2.0, end_cells=end_cells,
                     tide_delay_h=spinup_h if tide_delay_h is None else tide_delay_h, tide_amp=tide_amp,
                     name="config4_large_meander")
    c.notes["morfac"] = 10.0
    return c


MORPHO_TOE = 1.0  # Pa: erosion threshold of the morphodynamic workloads' sediment
MORPHO_MIN_DEPTH = 0.5  # m: no bed change in shallower water


def with_feedback(case, morfac=1.0, bed_period=600.0, fixed=None):
    """The case made morphodynamic: the bed change fed back (bed_feedback) every
    `bed_period` s at `morfac`, with the sediment set up for runs of days.

    The parity cases' sediment (constant.cuh's erosion threshold Toe = 0.15 Pa and a
    sediment-laden inflow of 0.2 kg/m3) is a parity set-up, not a long-run one: fed back,
    its Exner rate moves the bed by centimetres per 10-min update (up to the 5 cm cap per
    update within a few updates near the inflow, where the inflowing load settles), and
    within two hours of config 4 the bed cuts lines into more than 20 wet segments.  So the
    morphodynamic runs take a clear-water inflow (concentration 0), an erosion threshold of
    MORPHO_TOE, a fixed bed within `fixed` cells of the edges (default: twice the
    meander's rectangular end sections, i.e. the inlet and outlet sections and their
    blends) and where the water is shallower than MORPHO_MIN_DEPTH (the banks' fringe).
    On config 2 this gives mean bed changes of about 0.1 mm per update."""
    p = case.params.copy()
    p.bed_feedback = 1
    p.morfac = float(morfac)
    p.bed_period = float(bed_period)
    p.Toe = MORPHO_TOE
    p.bed_fixed = int(fixed if fixed is not None else 2 * case.notes.get("end_cells", 8))
    p.bed_min_depth = MORPHO_MIN_DEPTH
    case.params = p
    for e in range(4):
        case.cc[e] = np.zeros_like(case.cc[e])
    return case


CONFIG4_MORPHO_Q = 800.0  # m3/s: the steady discharge of config 4's 24-hour morphodynamic run


def config4_morpho_case(morfac=10.0, bed_period=600.0, dT=1.0, Q=CONFIG4_MORPHO_Q):
    """Config 4's 24-hour morphodynamic run: the 4096 x 2048 reach with the bed fed back
    every `bed_period` s at morphological factor `morfac` (with_feedback's long-run
    sediment), a steady discharge Q after the one-hour ramp and a fixed stage of 0 m.

    The workload states no forcing.  Under the parity case's tide (1 m) or its rising
    hydrograph (to 1750 m3/s) the reference's scheme on this 2.5 m grid goes unstable after
    2 to 10 hours, with or without the bed fed back (velocities past about 1.1 m/s at low
    water, then a blow-up in the channel), at dt = 1 s and at 0.5 s alike.  A steady 800
    m3/s with a fixed stage keeps the velocities below 0.9 m/s, and the run stays finite
    over the 24 hours at morfac 10 (checked at dt = 1 s and 0.5 s; bed changes up to
    1.2 m, about ten morphological days)."""
    c = config4_case(dT=dT, tide_amp=0.0)
    q = c.tables[EDGE_LEFT][0]
    th = np.arange(q.size, dtype=np.float64)
    q[:] = np.where(th < 1.0, Q * th, Q)
    c.name = "config4_morpho"
    return with_feedback(c, morfac=morfac, bed_period=bed_period)


CONFIG5_Q_MEAN, CONFIG5_Q_AMP = 687.5, 187.5  # config 2's scaled 500-875 m3/s range
CONFIG5_Q_PERIOD_H, CONFIG5_STAGE_PERIOD_H, CONFIG5_STAGE_AMP = 240.0, 354.4, 0.3


def config5_case(seed=20261205, days=30.0, spinup_h=1.0, bed_period=600.0, morfac=1.0, q_phase=None,
                 stage_phase=None, feedback=True, name="config5_morpho"):
    """Morphodynamic reach for the surrogate-assisted runs: the config-2 meander (1048 x 980,
    5 m cells, dt = 1 s, the generator with this seed: bed noise and roughness), `days` of
    hydraulics + sediment with the bed change fed back every `bed_period` s (bed_feedback,
    morfac), sediment from 0.5 h and bed change from 1 h as in config 2.

    Forcing (none is stated for this workload): over a 30-day run the hydraulics follow
    the slow variations, so the upstream discharge is config 2's scaled 500-875 m3/s range
    as a sine of 10-day period and the downstream stage a 0.3 m sine of the 14.77-day
    spring-neap period (the 12.42 h tide is averaged out), both with phases drawn from the
    seed unless given; the first `spinup_h` hours ramp the discharge linearly from rest.
    Hourly tables, linearly interpolated like the reference's.  The sediment is
    with_feedback's (clear-water inflow, erosion threshold MORPHO_TOE, a fixed bed in the
    inlet and outlet sections); feedback=False keeps that sediment with the bed unchanged."""
    rng = np.random.default_rng(seed + 1)
    qph = rng.uniform(0, 2 * math.pi) if q_phase is None else q_phase
    sph = rng.uniform(0, 2 * math.pi) if stage_phase is None else stage_phase
    hours = days * 24.0
    c = meander_case(N=1048, M=980, dX=5.0, dT=1.0, hours=hours, spinup_h=spinup_h, seed=seed,
                     Q0=CONFIG5_Q_MEAN, Q1=CONFIG5_Q_MEAN, tide_amp=0.0, name=name)
    th = np.arange(c.total_time, dtype=np.float64)
    tr = np.maximum(th - spinup_h, 0.0)
    q = CONFIG5_Q_MEAN + CONFIG5_Q_AMP * np.sin(2 * math.pi * tr / CONFIG5_Q_PERIOD_H + qph)
    q = np.where(th < spinup_h, q[int(math.ceil(spinup_h))] * th / spinup_h, q) if spinup_h > 0 else q
    zs = CONFIG5_STAGE_AMP * np.sin(2 * math.pi * tr / CONFIG5_STAGE_PERIOD_H + sph)
    zs = np.where(th < spinup_h, 0.0, zs) if spinup_h > 0 else zs
    c.tables[EDGE_LEFT] = q[None, :].copy()
    c.tables[EDGE_RIGHT] = zs[None, :].copy()
    with_feedback(c, morfac=morfac, bed_period=bed_period)
    if not feedback:
        p = c.params.copy()
        p.bed_feedback = 0
        c.params = p
    c.notes.update({"q_phase": qph, "stage_phase": sph, "days": days})
    return c


def config3_cases(n=96, seed=20261204, nx_range=(128, 1024), ny_range=(64, 512), hours=2.0, spinup_h=0.5):
    """The ensemble of independent reaches: n seeded meandering channels.

    Per reach: nx log-uniform in nx_range, ny log-uniform in ny_range, dx = dy = 5 m,
    dt = 1 s; sinuosity amplitude uniform 0-150 m (cut so that the channel stays inside
    the domain) and wavelength uniform 800-2500 m; Manning n uniform 0.018-0.035;
    discharge Q uniform 100-3000 m3/s.  Hydraulics + sediment for `hours` after a
    `spinup_h` discharge ramp (sediment from the end of the ramp, bed change an hour
    later).  The channel is the meander generator's parabolic section, its width
    min(150 m, 35 % of the domain width) and depth 4 m + 4 m x width / 150 m; Q is scaled
    by the width ratio and by the same stability factor as config 2 (the reference's
    scheme blows up on the full discharges, see config2_case)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        nx = int(round(math.exp(rng.uniform(math.log(nx_range[0]), math.log(nx_range[1])))))
        ny = int(round(math.exp(rng.uniform(math.log(ny_range[0]), math.log(ny_range[1])))))
        dX = 5.0
        width = min(150.0, 0.35 * ny * dX)
        depth = 4.0 + 4.0 * width / 150.0
        amp = min(rng.uniform(0.0, 150.0), max(0.0, (ny * dX - width) / 2.0 - 4 * dX))
        wavelength = rng.uniform(800.0, 2500.0)
        manning = rng.uniform(0.018, 0.035)
        q = rng.uniform(100.0, 3000.0) * CONFIG2_Q_SCALE * width / 150.0
        c = meander_case(N=nx, M=ny, dX=dX, dT=1.0, hours=hours, seed=seed + 1 + k, amp=amp,
                         wavelength=wavelength, width=width, depth=depth, manning=manning,
                         manning_spread=0.0, Q0=q, Q1=q, tide_amp=0.5, spinup_h=spinup_h,
                         sediment_start=spinup_h * 3600.0, bed_change_start=spinup_h * 3600.0 + 3600.0,
                         end_cells=min(8, nx // 16), name="config3_reach%02d" % k)
        c.notes.update({"Q": q, "amp": amp, "wavelength": wavelength, "manning": manning})
        out.append(c)
    return out
