"""Case inputs, pick-up files and outputs in the reference's text formats.

  read_dirs(path)                       a DirsOfInputs file: "key path" per line
  load_case_dir(dirs, ...)              the maps and hourly tables it names -> Case
                                        (Global_Variables.py:27-133)
  tanchau_case(input_dir)               the shipped Tan Chau reach (Inputs/TanChau)
  load_initial_condition(sim, dirs, case)
                                        pick-up text files u, v, z, khouot, FS
                                        (rep.py:41-52)
  save_fs_grd(FS, filename, ros, ...)   DSAA grid of FS * ros (Visualizor.py:32-47)
  export_velocity_and_level(...)        hourly speed/direction and water-level text
                                        (Engine.py:433-465)
"""
import math
import os

import numpy as np

from .cases import Case
from .params import default_params

SEGL = 20


def read_dirs(path):
    """Parse a DirsOfInputs file into {key: path} (Global_Variables.py:27-28)."""
    out = {}
    with open(path) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 2:
                out[parts[0]] = parts[1]
    return out


def read_boundary_type(path):
    """boundary_type[4][20] (Global_Variables.py:30-37): one line per edge (up, down, left,
    right), the types of its segments (0 wall, 1 stage, 2 discharge), or NA."""
    bt = np.zeros((4, SEGL), dtype=np.int32)
    with open(path) as f:
        lines = [ln.strip() for ln in f]
    for i, inp in enumerate(lines[:4]):
        if inp and inp != "NA":
            vals = [int(float(x)) for x in inp.split()]
            bt[i, :len(vals)] = vals
    return bt


def _table(path):
    """An hourly boundary table as [segment][hour] (Global_Variables.py:39-47)."""
    return np.atleast_2d(np.transpose(np.loadtxt(path)))


def load_case_dir(dirs, base_dir=".", params=None, t_start=0.0, nsteps=1, name="case", notes=None):
    """Build a Case from the files named in `dirs` (keys of DirsOfInputs_1.txt:
    topography, visco_map, roughness_map, friction_map, boundary_type, up, down, left,
    right, CC_u, CC_d, CC_l, CC_r), resolved against base_dir.

    As in Global_Variables.py:49-133: total_time = the length of the first open edge's
    table per segment; h = flipped, padded depth + NANGDAY; hsnham, VISCOIDX, Fw read the
    same way; u, v, z, FS start at zero.  A map whose extent differs from the
    topography's is cut to the topography's extent (the reference would pass the
    mismatched arrays through unchecked)."""
    p = params if params is not None else default_params()
    path = lambda k: os.path.join(base_dir, dirs[k])
    bt = read_boundary_type(path("boundary_type"))
    topo = np.transpose(np.loadtxt(path("topography")))
    N, M = topo.shape
    notes = dict(notes or {})

    def grid_map(key):
        raw = np.transpose(np.loadtxt(path(key)))
        if raw.shape != (N, M):
            notes[key] = "map %dx%d cut to the topography's %dx%d" % (raw.shape[0], raw.shape[1], N, M)
            if raw.shape[0] < N or raw.shape[1] < M:
                raise ValueError("%s is smaller than the topography" % key)
            raw = raw[:N, :M]
        return np.pad(np.flip(raw, 1), ((1, 2), (1, 2)), "edge")

    h = np.pad(np.flip(topo, 1), ((1, 2), (1, 2)), "edge") + p.NANGDAY
    fields = {"h": h, "hsnham": grid_map("roughness_map"), "VISCOIDX": grid_map("visco_map"),
              "Fw": grid_map("friction_map")}
    shape = (N + 3, M + 3)
    for k in ("Tsxw", "Tsyw", "u", "v", "z", "FS"):
        fields[k] = np.zeros(shape)
    raw_tabs = [_table(path(k)) for k in ("up", "down", "left", "right")]
    raw_cc = [_table(path(k)) for k in ("CC_u", "CC_d", "CC_l", "CC_r")]
    open_edges = [e for e in range(4) if np.count_nonzero(bt[e])]
    if not open_edges:
        raise ValueError("no open boundary in boundary_type")
    e0 = open_edges[0]
    total_time = int(raw_tabs[e0].size // np.count_nonzero(bt[e0]))
    tables, cc = [], []
    for e in range(4):
        nseg = int(np.count_nonzero(bt[e]))
        t, c = raw_tabs[e], raw_cc[e]
        if nseg == 0:
            tables.append(np.zeros((0, total_time)))
            cc.append(np.zeros((0, total_time)))
            continue
        if t.shape[0] < nseg or c.shape[0] < nseg or t.shape[1] < total_time or c.shape[1] < total_time:
            raise ValueError("boundary table of edge %d shorter than %d segments x %d hours" % (e, nseg, total_time))
        tables.append(np.ascontiguousarray(t[:nseg, :total_time], dtype=np.float64))
        cc.append(np.ascontiguousarray(c[:nseg, :total_time], dtype=np.float64))
    return Case(name=name, N=N, M=M, params=p, fields=fields, boundary_type=bt, tables=tables, cc=cc,
                total_time=total_time, t_start=float(t_start), nsteps=int(nsteps), notes=notes)


# The reference's DirsOfInputs_1.txt names Inputs/TanChau2/..., which is not shipped; the
# files of Inputs/TanChau carry these names.
TANCHAU_FILES = {
    "topography": "dosauTanChau.txt",
    "visco_map": "bandohsnhotroiA.txt",
    "roughness_map": "bandohsnham.txt",
    "friction_map": "bandoFw.txt",
    "boundary_type": "boundary_type.txt",
    "up": "bientren_Q_TC.txt",
    "down": "bienduoi.txt",
    "left": "bientrai.txt",
    "right": "bienphai_Z_TC.txt",
    "CC_u": "FS_bientren.txt",
    "CC_d": "FS_bienduoi.txt",
    "CC_l": "FS_bientrai.txt",
    "CC_r": "FS_bienphai.txt",
}


def tanchau_case(input_dir, params=None, nsteps=1):
    """The Tan Chau reach from a copy of the reference's Inputs/TanChau directory, with the
    case constants of constant_TanChau.cuh (equal to constant.cuh's except segment_limit,
    10 there; the library always allows 20)."""
    return load_case_dir(TANCHAU_FILES, base_dir=input_dir, params=params, nsteps=nsteps, name="tanchau")


def load_initial_condition(sim, dirs, case):
    """Pick-up (rep.py:41-52): u.txt, v.txt, z.txt (one header line each), khouot.txt and
    FS.txt in directory `dirs`, (N+2)x(M+2) each, padded by one row and column after
    (edge values; the mask with 2).  The reference reads the mask from the working
    directory by a keyword slip (`loadtxt(dirs = 'khouot.txt')`); here it is read from
    `dirs` like the others.  Call Simulation.init_pickup afterwards, which keeps the mask
    (the reference loads these between Onetime_init and the segment scans)."""
    join = lambda f: os.path.join(dirs, f)
    want = (case.N + 3, case.M + 3)

    def edge(a):
        a = np.pad(a, ((0, 1), (0, 1)), "edge")
        if a.shape != want:
            raise ValueError("pick-up field has shape %s, expected %s" % (a.shape, want))
        return a

    u = edge(np.loadtxt(join("u.txt"), skiprows=1))
    v = edge(np.loadtxt(join("v.txt"), skiprows=1))
    z = edge(np.loadtxt(join("z.txt"), skiprows=1))
    kh = np.pad(np.loadtxt(join("khouot.txt"), dtype=np.int32), ((0, 1), (0, 1)), "constant", constant_values=2)
    if kh.shape != want:
        raise ValueError("pick-up mask has shape %s, expected %s" % (kh.shape, want))
    fs = edge(np.loadtxt(join("FS.txt")))
    for name, a in (("u", u), ("v", v), ("z", z), ("khouot", kh), ("FS", fs)):
        sim.set(name, a)


def save_pickup(sim, dirs):
    """Write the fields load_initial_condition reads (the inverse of rep.py:41-52)."""
    os.makedirs(dirs, exist_ok=True)
    for name in ("u", "v", "z"):
        a = sim.get(name)[:-1, :-1]
        np.savetxt(os.path.join(dirs, name + ".txt"), a, header=name, comments="")
    np.savetxt(os.path.join(dirs, "khouot.txt"), sim.get("khouot")[:-1, :-1], fmt="%d")
    np.savetxt(os.path.join(dirs, "FS.txt"), sim.get("FS")[:-1, :-1])


def save_fs_grd(FS, filename, ros, val_range=(0, 10), mode="DSAA"):
    """DSAA (Surfer ASCII) grid of FS * ros over rows 2..N-1 and columns 2..M-1, with the
    header of Visualizor.py:32-47 (its loop stops one short of the N x M extent it
    declares; the same values are written here)."""
    N, M = FS.shape[0] - 3, FS.shape[1] - 3
    d = os.path.dirname(filename)
    if d:
        os.makedirs(d, exist_ok=True)
    with open(filename, "w") as f:
        f.write(mode + "\n")
        f.write("%d %d\n" % (N - 1, M - 1))
        f.write("%d %d\n" % (2, N))
        f.write("%d %d\n" % (2, M))
        f.write("%s %s\n" % (val_range[0], val_range[1]))
        for i in range(2, N):
            f.write(" ".join(repr(float(FS[i, j] * ros)) for j in range(2, M)) + " \n")


def velocity_and_angle(u, v, htaiz, NANGDAY):
    """Cell speed and direction (degrees) at cells 1..N x 1..M (Engine.py:440-459), as
    arrays.  In the third quadrant the reference adds 180 to a misspelled name
    (`angl += 180`), which raises in Python; the intended angle + 180 is used here."""
    N, M = u.shape[0] - 3, u.shape[1] - 3
    vt = (v[1:N + 1, 0:M] + v[1:N + 1, 1:M + 1]) * 0.5
    ut = (u[1:N + 1, 1:M + 1] + u[0:N, 1:M + 1]) * 0.5
    vth = np.sqrt(vt * vt + ut * ut)
    vth = np.where(htaiz[1:N + 1, 1:M + 1] <= NANGDAY, 0.0, vth)
    with np.errstate(divide="ignore", invalid="ignore"):
        base = 180 * np.arctan(np.abs(vt / np.where(ut != 0, ut, 1.0))) / math.pi
    ang = np.where(ut != 0, base, np.where(vt > 0, 90.0, np.where(vt < 0, 270.0, 0.0)))
    ang = np.where((ut != 0) & (vt < 0) & (ut > 0), 360 - base, ang)
    ang = np.where((ut != 0) & (vt > 0) & (ut < 0), 180 - base, ang)
    ang = np.where((ut != 0) & (vt < 0) & (ut < 0), base + 180, ang)
    return vth, ang


def export_velocity_and_level(sim, t, out_dir="Outputs"):
    """Hourly export (Engine.py:433-465): <out_dir>/velocity/VTH<t>s.data with "t i j vth
    angle" records, and <out_dir>/water_level/mucnuoc<t>s.grid with z over 1..N x 1..M.
    The reference writes the velocity records without separators; one record per line
    here."""
    p = sim.params
    u, v, z, htaiz = sim.get("u"), sim.get("v"), sim.get("z"), sim.get("htaiz")
    N, M = u.shape[0] - 3, u.shape[1] - 3
    vth, ang = velocity_and_angle(u, v, htaiz, p.NANGDAY)
    vdir = os.path.join(out_dir, "velocity")
    zdir = os.path.join(out_dir, "water_level")
    os.makedirs(vdir, exist_ok=True)
    os.makedirs(zdir, exist_ok=True)
    with open(os.path.join(vdir, "VTH%ss.data" % t), "w") as f:
        for i in range(N):
            for j in range(M):
                f.write("%.1f %d %d %.2f %.2f\n" % (t, i + 1, j + 1, vth[i, j], ang[i, j]))
    with open(os.path.join(zdir, "mucnuoc%ss.grid" % t), "w") as f:
        for i in range(1, N + 1):
            f.write("".join("%.2f " % z[i, j] for j in range(1, M + 1)) + "\n")
