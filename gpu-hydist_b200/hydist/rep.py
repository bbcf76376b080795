"""rep.py-compatible command line over the CUDA library (rep.py:23-40, 145-173).

    python -m hydist.rep [--Device 0] [--hours 10] [--mins 0] [--sediment 10]
                         [--bed_change 20] [--pick_up False] [--pickup_dirs DIR]
                         [--kenhhepng False] [--kenhhepd False] [--plot False]
                         [--dirs DirsOfInputs_1.txt | --case NAME]

The flags keep the reference's names, defaults and meanings: the run lasts
hours * 3600 + mins * 60 s, the sediment phase starts at --sediment hours and the bed
change at --bed_change hours, u, v, z are taken every 3600 s (rep.py:145-160), and the
line "total running time of  <hours> hours is  <seconds>" is printed at the end.  --GPU,
--test and --include_dirs are accepted and ignored (they select PyCUDA set-up that this
library does not need).  --plot is accepted; plotting is not part of this library.

The case: the reference's host reads the input maps and tables named in
DirsOfInputs_1.txt in its working directory (Global_Variables.py:27-28).  --dirs names
such a file (its paths resolved against the file's folder; default: DirsOfInputs_1.txt in
the working directory); --case runs one of the named synthetic cases instead.

String flags: the reference's argparse leaves --pick_up, --kenhhepd and --kenhhepng as
strings when given, so any given value is true ("False" included), and its channel-mode
range shift, which compares the flag with 1, never happens (Engine.py:156,277, quirk
Q11).  The same is done here: a given channel flag selects channel mode without the
shift.
"""
import argparse
import os
import sys
import time

from . import cases, engine, io

NAMED_CASES = {
    "config1": cases.config1_case,
    "config2": cases.config2_case,
    "config4": cases.config4_case,
    "islands": cases.islands_case,
}


def parser():
    ap = argparse.ArgumentParser(prog="python -m hydist.rep", description=__doc__.split("\n\n")[0])
    ap.add_argument("--GPU", type=int, default=1)
    ap.add_argument("--Device", type=int, default=0)
    ap.add_argument("--mins", type=int, default=0)
    ap.add_argument("--hours", type=int, default=10)
    ap.add_argument("--plot", default=False)
    ap.add_argument("--test", default=False)
    ap.add_argument("--sediment", default=10)
    ap.add_argument("--bed_change", default=20)
    ap.add_argument("--pick_up", default=False)
    ap.add_argument("--pickup_dirs", default="/Input/Initial_Condition")
    ap.add_argument("--kenhhepng", default=False)
    ap.add_argument("--kenhhepd", default=False)
    ap.add_argument("--include_dirs", default=None)
    src = ap.add_mutually_exclusive_group()
    src.add_argument("--dirs", default=None, help="a DirsOfInputs file (default: DirsOfInputs_1.txt here)")
    src.add_argument("--case", default=None, choices=sorted(NAMED_CASES), help="a named synthetic case")
    return ap


def load_case(args):
    if args.case:
        return NAMED_CASES[args.case]()
    path = args.dirs or "DirsOfInputs_1.txt"
    if not os.path.exists(path):
        raise SystemExit("rep: %s not found (give --dirs FILE or --case NAME)" % path)
    return io.load_case_dir(io.read_dirs(path), base_dir=os.path.dirname(os.path.abspath(path)),
                            name=os.path.basename(path))


def main(argv=None):
    args = parser().parse_args(argv)
    case = load_case(args)
    Tmax = args.hours * 3600 + args.mins * 60
    sediment_start = float(args.sediment) * 3600
    bed_change_start = float(args.bed_change) * 3600
    # a given string flag is true, and the channel range shift never fires (see above)
    channel_d = 2 if args.kenhhepd not in (False, None) else 0
    channel_ng = 2 if args.kenhhepng not in (False, None) else 0
    pick_up = args.pick_up not in (False, None)
    sim, ctx, arg_ptr, arr_ptr, supmod = engine.gpu_init(case, device_no=args.Device, pick_up=pick_up,
                                                         pickup_dirs=args.pickup_dirs)
    start = time.perf_counter()
    ulist, vlist, zlist, fslist = engine.hydraulic_Calculation(
        Tmax, sim, arg_ptr, arr_ptr, supmod, ctx, kenhhepd=channel_d, kenhhepng=channel_ng, save_grid=False,
        sediment_start=sediment_start, debug=False, plot=args.plot, interval=3600, export=False,
        bed_change_start=bed_change_start)
    stop = time.perf_counter()
    print("total running time of ", args.hours, "hours is ", stop - start)
    sim.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
