"""Engine/rep-compatible host calls over the CUDA library.

Mirrors the reference's step-and-run surface:
  * ``gpu_init(case, device_no=0)``  ~ rep.gpu_init (rep.py:58-142): uploads the case,
    runs the one-time initialisation, returns ``(pointers, ctx, arg_struct_ptr,
    arr_struct_ptr, supmod)`` where ``pointers`` is the device simulation and the other
    four are placeholders kept for call compatibility (there are no PyCUDA objects).
  * ``hydraulic_Calculation(Tmax, pointers, ...)`` ~ Engine.hydraulic_Calculation
    (Engine.py:49-469): advances to Tmax, extracting u, v, z (and FS) every
    ``interval`` seconds and stopping at the first non-finite extract, and returns
    ``(u_list, v_list, z_list, fslist)``.
"""
import math

import numpy as np

from .lib import Simulation


def gpu_init(case, device_no=0, pick_up=False, pickup_dirs=None):
    """Create the device simulation for `case` and run rep.py:126-139's initialisation.

    With pick_up, the initial u, v, z, khouot, FS are read from text files in
    `pickup_dirs` (rep.py:43-55) before the segment scans; see hydist.io."""
    sim = Simulation.from_case(case, device=device_no, init=False)
    if pick_up:
        from .io import load_initial_condition
        load_initial_condition(sim, pickup_dirs, case)
        sim.init_pickup(case.t_start)
    else:
        sim.init(case.t_start)
    return sim, None, None, None, None


def hydraulic_Calculation(Tmax, pointers, arg_struct_ptr=None, arr_struct_ptr=None, supmod=None, ctx=None,
                          ketdinh=True, blk_size=1024, kenhhepd=0, kenhhepng=0, debug=False, interval=1,
                          sediment_start=36000, t_start=None, sec=1, plot=False, export=False, save_grid=False,
                          bed_change_start=72000, out_dir="Outputs"):
    """Run the ADI time loop to Tmax (Engine.py:144-412).

    Returns (u_list, v_list, z_list, fslist): u, v, z copies every `interval` seconds
    of simulated time (Engine.py:398-420) and FS every 360 s when save_grid
    (Engine.py:423-430).  kenhhepd/kenhhepng select the channel-mode boundaries;
    as in the reference only the value 1 shifts the sweep ranges."""
    sim = pointers
    p = sim.params
    p.ketdinh = 1 if ketdinh else 0
    p.sediment_start = float(sediment_start)
    p.bed_change_start = float(bed_change_start)
    p.kenhhepd = _channel_flag(kenhhepd)
    p.kenhhepng = _channel_flag(kenhhepng)
    sim.set_params(p)
    u_list, v_list, z_list, fslist = [], [], [], []
    dT = p.dT
    t = sim.t
    while t < Tmax:
        # advance to the next time at which the reference host looks at the state
        nxt = t + dT
        steps = 1
        while nxt < Tmax and not _host_event(nxt, interval, save_grid, sediment_start, export):
            nxt += dT
            steps += 1
        t = sim.step(steps, sync=True)
        if int(t) % interval == 0 and t - int(t) == 0:
            u, v, z = sim.get("u"), sim.get("v"), sim.get("z")
            if not (np.isfinite(u).all() and np.isfinite(v).all() and np.isfinite(z).all()):
                return u_list, v_list, z_list, fslist
            u_list.append(u)
            v_list.append(v)
            z_list.append(z)
        if save_grid and t >= sediment_start and int(t) % 360 == 0 and t - int(t) == 0:
            from .io import save_fs_grd
            fs = sim.get("FS")
            save_fs_grd(fs, "%s/FS_GPU/fs_%s.grd" % (out_dir, t), p.ros)
            fslist.append(fs)
        if export and int(t) % 3600 == 0 and t - int(t) == 0:
            from .io import export_velocity_and_level
            export_velocity_and_level(sim, t, out_dir)
    return u_list, v_list, z_list, fslist


def _channel_flag(v):
    """Engine.py's use of kenhhepd / kenhhepng: a true value selects the channel-mode
    boundaries (Engine.py:68), and only a value equal to 1 also shifts the sweep ranges
    (Engine.py:156,277).  A string (rep.py's argparse value) is true but never equal to 1
    (quirk Q11), so it maps to 2: channel mode without the shift."""
    if isinstance(v, (bool, int, np.integer)):
        return int(v)
    return 2 if v else 0


def _host_event(t, interval, save_grid, sediment_start, export):
    if t != math.floor(t):
        return False
    it = int(t)
    if it % interval == 0:
        return True
    if save_grid and t >= sediment_start and it % 360 == 0:
        return True
    if export and it % 3600 == 0:
        return True
    return False
