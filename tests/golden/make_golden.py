"""Generate the golden fixtures from the reference's own kernel sources.

Run in a container that has the reference tree (the recipe oracle/Makefile compiles
support_funcs.cu, UVZSolver_multithread.cu and Sediment_Transport.cu from it into
oracle/_ref/libhydref_cpu.so and this script executes them launch for launch):

    python tests/golden/make_golden.py
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "gpu-hydist_b200"), os.path.join(ROOT, "oracle"), HERE]

import golden  # noqa: E402
import oracle  # noqa: E402
from hydist import cases  # noqa: E402


def golden_cases():
    c1 = cases.channel_case(N=40, M=16, bank=2, hours=1, name="channel_small")
    c1.nsteps = 150
    c2 = cases.islands_case(N=48, M=36, name="islands")
    c2.nsteps = 120
    c3 = cases.islands_case(N=40, M=52, seed=11, name="islands_wide", sediment_start=20.0,
                            bed_change_start=30.0)
    c3.nsteps = 90
    c4 = cases.meander_case(N=96, M=64, dX=5.0, dT=1.0, hours=1.0, spinup_h=0.0, amp=40.0, wavelength=300.0,
                            width=60.0, depth=4.0, floodplain=1.0, noise_sigma=0.1, noise_len=15.0,
                            Q0=40.0, Q1=60.0, tide_amp=0.3, tide_period_h=1.5, sediment_start=30.0,
                            bed_change_start=60.0, end_cells=4, name="meander_small")
    c4.nsteps = 200
    c5 = cases.channel_case(N=36, M=20, bank=3, hours=1, name="channel_mode")
    c5.params.kenhhepd = 1
    c5.nsteps = 60
    return [c1, c2, c3, c4, c5]


# The shipped Tan Chau reach (the reference's Inputs/TanChau), with sediment from 20 s and
# the bed update at 40 s so that every part of the step runs on the real inputs.  Its
# fixture keeps the prognostic fields and the segment tables only (size).
TANCHAU_OUT = ("z", "u", "v", "FS", "dH", "khouot", "daui", "cuoii", "moci", "dauj", "cuoij", "mocj")


def tanchau_golden(ref_root):
    from hydist import io
    c = io.tanchau_case(os.path.join(ref_root, "Inputs", "TanChau"))
    c.params.sediment_start = 20.0
    c.params.bed_change_start = 40.0
    c.nsteps = 60
    return c


def main(ref_root=os.environ.get("HYDIST_REFERENCE", "/root/reference")):
    oracle.build(("ref_cpu",))
    todo = [(c, golden.OUT_FIELDS) for c in golden_cases()] + [(tanchau_golden(ref_root), TANCHAU_OUT)]
    for c, fields in todo:
        r = oracle.RefSim(c)
        r.init()
        r.step(c.nsteps)
        out = {f: r.get(f) for f in fields}
        path = os.path.join(HERE, c.name + ".npz")
        golden.save(path, c, out)
        print("wrote", path, "t =", r.t, "bytes", os.path.getsize(path))


if __name__ == "__main__":
    main()
