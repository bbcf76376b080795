"""Case loader, pick-up files and output writers (CPU).

The loader follows Global_Variables.py:27-133, the pick-up rep.py:41-52, the writers
Visualizor.py:32-47 and Engine.py:433-465.  The Tan Chau test reads the reference's
shipped inputs and is skipped where the reference tree is absent; the pick-up pin runs
the reference's own kernels (oracle/_ref) against the oracle."""
import math
import os

import numpy as np
import pytest

from hydist import io

REF_TANCHAU = os.path.join(os.environ.get("HYDIST_REFERENCE", "/root/reference"), "Inputs", "TanChau")


def _write_case_dir(d, N=7, M=5, nseg_up=2, hours=6, seed=3):
    rng = np.random.default_rng(seed)
    topo = rng.uniform(-1, 5, size=(M, N))  # files hold the transposed, flipped map
    np.savetxt(os.path.join(d, "topo.txt"), topo)
    np.savetxt(os.path.join(d, "n.txt"), rng.uniform(0.02, 0.03, size=(M, N)))
    np.savetxt(os.path.join(d, "visc.txt"), rng.uniform(0.5, 1.5, size=(M + 1, N + 2)))  # larger: cut
    np.savetxt(os.path.join(d, "fw.txt"), rng.uniform(0, 1e-3, size=(M, N)))
    with open(os.path.join(d, "bt.txt"), "w") as f:
        f.write(" ".join(["2"] * nseg_up) + "\nNA\n0\n1\n")
    up = rng.uniform(100, 200, size=(hours, nseg_up))  # one column per segment
    np.savetxt(os.path.join(d, "up.txt"), up)
    np.savetxt(os.path.join(d, "right.txt"), rng.uniform(-1, 1, size=hours + 3))  # longer: cut
    for k in ("down", "left", "ccd", "ccl"):
        np.savetxt(os.path.join(d, k + ".txt"), np.zeros(hours))
    np.savetxt(os.path.join(d, "ccu.txt"), rng.uniform(0, 0.2, size=(hours, nseg_up)))
    np.savetxt(os.path.join(d, "ccr.txt"), rng.uniform(0, 0.2, size=hours + 3))
    dirs = {"topography": "topo.txt", "visco_map": "visc.txt", "roughness_map": "n.txt", "friction_map": "fw.txt",
            "boundary_type": "bt.txt", "up": "up.txt", "down": "down.txt", "left": "left.txt", "right": "right.txt",
            "CC_u": "ccu.txt", "CC_d": "ccd.txt", "CC_l": "ccl.txt", "CC_r": "ccr.txt"}
    with open(os.path.join(d, "dirs.txt"), "w") as f:
        for k, v in dirs.items():
            f.write("%s %s\n" % (k, v))
    return topo, up


def test_load_case_dir_layout(tmp_path):
    topo, up = _write_case_dir(str(tmp_path))
    dirs = io.read_dirs(str(tmp_path / "dirs.txt"))
    c = io.load_case_dir(dirs, base_dir=str(tmp_path))
    N, M = topo.shape[1], topo.shape[0]
    assert (c.N, c.M) == (N, M)
    # Global_Variables.py:67-72: transpose, flip along j, pad (1, 2) with edge values, + NANGDAY
    expect = np.pad(np.flip(topo.T, 1), ((1, 2), (1, 2)), "edge") + c.params.NANGDAY
    assert np.array_equal(c.fields["h"], expect)
    assert c.fields["VISCOIDX"].shape == (N + 3, M + 3) and "visco_map" in c.notes
    assert c.boundary_type[0, :3].tolist() == [2, 2, 0]
    assert not c.boundary_type[1].any() and c.boundary_type[3, 0] == 1
    assert c.total_time == up.shape[0]
    assert c.tables[0].shape == (2, up.shape[0]) and np.array_equal(c.tables[0], up.T)
    assert c.tables[3].shape == (1, c.total_time) and c.tables[1].shape[0] == 0


@pytest.mark.skipif(not os.path.isdir(REF_TANCHAU), reason="reference inputs not present")
def test_tanchau_inputs():
    c = io.tanchau_case(REF_TANCHAU)
    assert (c.N, c.M) == (464, 324)
    assert c.boundary_type[:, 0].tolist() == [2, 0, 0, 1]
    assert c.total_time == 4246 and c.tables[0][0, 0] == -6910.0
    topo = np.loadtxt(os.path.join(REF_TANCHAU, "dosauTanChau.txt"))
    assert np.array_equal(c.fields["h"][1:-2, 1:-2], np.flip(topo.T, 1) + c.params.NANGDAY)


def test_pickup_files_padding(tmp_path):
    class Rec:
        def __init__(self):
            self.got = {}

        def set(self, name, a):
            self.got[name] = np.array(a)

    class C:
        N, M = 6, 4

    rng = np.random.default_rng(0)
    shape = (C.N + 2, C.M + 2)
    vals = {k: rng.normal(size=shape) for k in ("u", "v", "z", "FS")}
    for k in ("u", "v", "z"):
        np.savetxt(tmp_path / (k + ".txt"), vals[k], header=k, comments="")
    np.savetxt(tmp_path / "FS.txt", vals["FS"])
    mask = rng.integers(0, 3, size=shape)
    np.savetxt(tmp_path / "khouot.txt", mask, fmt="%d")
    r = Rec()
    io.load_initial_condition(r, str(tmp_path), C)
    for k in ("u", "v", "z", "FS"):
        assert r.got[k].shape == (C.N + 3, C.M + 3)
        assert np.array_equal(r.got[k][:-1, :-1], vals[k])
        assert np.array_equal(r.got[k][-1, :-1], vals[k][-1]) and np.array_equal(r.got[k][:-1, -1], vals[k][:, -1])
    assert np.array_equal(r.got["khouot"][:-1, :-1], mask)
    assert (r.got["khouot"][-1] == 2).all() and (r.got["khouot"][:, -1] == 2).all()


def test_save_fs_grd(tmp_path):
    rng = np.random.default_rng(1)
    N, M, ros = 7, 5, 2650.0
    FS = rng.uniform(0, 1e-3, size=(N + 3, M + 3))
    path = tmp_path / "fs.grd"
    io.save_fs_grd(FS, str(path), ros)
    lines = path.read_text().splitlines()
    assert lines[0] == "DSAA" and lines[1] == "%d %d" % (N - 1, M - 1)
    assert lines[2] == "2 %d" % N and lines[3] == "2 %d" % M and lines[4] == "0 10"
    body = np.array([[float(x) for x in ln.split()] for ln in lines[5:]])
    assert body.shape == (N - 2, M - 2)
    assert np.array_equal(body, FS[2:N, 2:M] * ros)


def _angle_loop(u, v, htaiz, NANGDAY):
    # Engine.py:440-459 as a loop, third quadrant with its evident + 180
    N, M = u.shape[0] - 3, u.shape[1] - 3
    vth = np.zeros((N, M))
    ang = np.zeros((N, M))
    for i in range(1, N + 1):
        for j in range(1, M + 1):
            vt = (v[i, j - 1] + v[i, j]) * 0.5
            ut = (u[i, j] + u[i - 1, j]) * 0.5
            s = math.sqrt(vt * vt + ut * ut)
            if htaiz[i, j] <= NANGDAY:
                s = 0
            a = 0
            if ut != 0:
                a = 180 * math.atan(abs(vt / ut)) * 1 / math.pi
                if vt < 0 and ut > 0:
                    a = 360 - a
                elif vt < 0 and ut < 0:
                    a += 180
                elif vt > 0 and ut < 0:
                    a = 180 - a
            else:
                if vt > 0:
                    a = 90.0
                elif vt < 0:
                    a = 270.0
            vth[i - 1, j - 1] = s
            ang[i - 1, j - 1] = a
    return vth, ang


def test_velocity_and_angle_matches_loop():
    rng = np.random.default_rng(2)
    N, M = 9, 6
    u = rng.normal(size=(N + 3, M + 3))
    v = rng.normal(size=(N + 3, M + 3))
    u[3, :] = 0
    v[:, 2] = 0
    htaiz = rng.uniform(-1, 1, size=(N + 3, M + 3))
    vth, ang = io.velocity_and_angle(u, v, htaiz, 0.0)
    lv, la = _angle_loop(u, v, htaiz, 0.0)
    assert np.allclose(vth, lv, rtol=1e-15, atol=0) and np.allclose(ang, la, rtol=1e-13, atol=1e-12)


def test_pickup_oracle_pinned_to_reference(tmp_path, ref_cpu_lib):
    """The pick-up order of rep.py:126-131 (Onetime_init, pick-up files, scans): the
    oracle against the reference's own kernels, bit for bit."""
    import golden
    import oracle
    case, _ = golden.load("islands")
    first = oracle.RefSim(case)
    first.init()
    first.step(40)
    for k in ("u", "v", "z"):
        np.savetxt(tmp_path / (k + ".txt"), first.get(k)[:-1, :-1], header=k, comments="")
    np.savetxt(tmp_path / "FS.txt", first.get("FS")[:-1, :-1])
    np.savetxt(tmp_path / "khouot.txt", first.get("khouot")[:-1, :-1], fmt="%d")

    class Grab:
        def __init__(self):
            self.f = {}

        def set(self, name, a):
            self.f[name] = a

    g = Grab()
    io.load_initial_condition(g, str(tmp_path), case)
    ref = oracle.RefSim(case)
    ora = oracle.OracleSim(case)
    for k in ("u", "v", "z", "FS"):
        a = np.ascontiguousarray(g.f[k], dtype=np.float64)
        ref._check(ref.lib.ref_set_field(ref.h, k.encode(), a.ctypes.data, a.size))
        ora.view(k)[...] = a
    ora.view("khouot")[...] = g.f["khouot"]
    ref.init_pickup(g.f["khouot"])
    ora.init_pickup()
    ref.step(30)
    ora.step(30)
    for f in ("z", "u", "v", "FS", "khouot", "H_moi", "daui", "dauj", "moci", "mocj"):
        assert np.array_equal(ora.get(f), ref.get(f)), f
