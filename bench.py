"""Benchmark: ADI cell-updates/s of the B200 library on the meandering-reach workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (config 2): 1048 x 980 cells, dx = dy = 5 m, dt = 1 s, FP64 hydraulics with the
suspended-sediment ADI and the Exner update active (--workload config4: the 4096 x 2048
reach at 2.5 m, same physics).  A "step" is one full ADI step (two
half-steps) of the whole grid; one cell-update is one interior cell advanced one step.
The state is first spun up (untimed) to t = 3590 s, where sediment is active and the
Exner update fires every 3600 s.  The span-limited kernels touch only the cells near
water, a working set that fits the 126 MB L2, so every timed step is preceded by an
untimed 256 MB write that flushes L2, and each step is timed alone by CUDA events on the
library's stream (the per-step times are summed).  The back-to-back rate of the same
steps without the flush (how a simulation runs) is reported beside it.

--impl ours       the CUDA library; prints value (device-resident), e2e (through the C
                  ABI from pinned host buffers: the boundary forcing in and the water
                  level out every step, through the library's host mirror of z;
                  e2e_full_field copies every cell of z instead, e2e_state_roundtrip the
                  whole state both ways), roofline of the dominant phase, cpu_baseline
                  (the oracle port on the host cores) and reference_kernels_gpu (the
                  reference's own kernels, built for sm_100a, on the same GPU).
--impl reference  the same scheme on the host cores: the reference has no CPU
                  implementation of this path, so this times the oracle port (a line-for-
                  line C restatement of the reference's kernels, OpenMP) on a bounded sample.
Multi-GPU (torchrun): one independent replica of the reach per GPU ("replicas only":
an ADI line couples the whole domain, so a single reach has no shard).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "gpu-hydist_b200"), os.path.join(ROOT, "oracle")]

SPINUP_STEPS = 3590
METRIC = "ADI cell-updates/s"
# --workload: name -> (case builder in hydist.cases, description, data)
WORKLOADS = {
    "config2": ("config2_case", "config2_meander 1048x980 dx=5m dt=1s FP64 hydraulics+sediment+Exner",
                "synthetic (seeded meandering reach, config-2 shape)"),
    "config4": ("config4_case", "config4_large_meander 4096x2048 dx=2.5m dt=1s FP64 hydraulics+sediment+Exner",
                "synthetic (seeded meandering reach, config-4 shape)"),
}

# algorithmic bytes per launch of each phase, per unit: cells of the extended spans (the
# cells the elementwise kernels visit once the grid is up to date, "span"), cells of the
# spans of cells that can be wet ("core"), or wet cells of the swept lines ("wet"): each
# field the kernel needs read once and each field it produces written once
PHASE_BYTES = {
    "smooth": (20, "span"),        # read t (8) + mask (4), write out (8)
    "post": (152, "span"),         # update: read t_z,t_u,t_v,h (32), write z,u,v,Htdu,Htdv (40);
                                   # with VTH/K: read H_moi,htaiz (16), write VTH,Kx,Ky (24) ...
    "reset_rows": (28, "core"),    # read mask, htaiz, t_z (20), write H_moi (8)
    "reset_cols": (28, "core"),
    "scan": (8, "core"),
    "vth_hesok": (80, "span"),     # read t_u,t_v,H_moi,htaiz,Htdu,Htdv,h (56), write VTH,Kx,Ky (24)
    "update_fs": (16, "span"),
    "sweep_uz": (72, "wet"),       # read a2,c2,d2,f1,f2,f3,f5 (56), write t_z,t_u (16)
    "sweep_vz": (88, "wet"),       # read u,v,z,Htdu,Htdv,H_moi,VISC,Ky1,Tsyw (72), write t_z,t_v (16)
    "explicit_v": (80, "wet"),
    "explicit_u": (24, "wet"),     # read the precomputed u (8), t_u staged (8), write t_u (8)
    "fs_sweep_j": (40, "wet"),     # read aa,bb,cc,dd (32), write tFS (8)
    "fs_sweep_i": (88, "wet"),
    "coef_uz": (128, "wet"),       # read u,v,z,Htdu,Htdv,H_moi,VISC,Kx1,Tsxw (72), write 7 coefficients (56)
    "coef_fsj": (112, "wet"),      # read FS,H_moi,VTH,Fw,t_u,t_v,Htdu,Htdv,Kx,Ky (80), write 4 (32)
    "coef_eu": (80, "wet"),        # read u,v,t_v,z,Kx1,Htdu,H_moi,VISC,Tsxw (72), write 8
    "boundary": (0, "core"),
    "bed": (0, "core"),
}

# phases launched on the library's second stream, beside the main chain
SIDE_PHASES = ("coef_fsj", "fs_sweep_j")

# DRAM traffic per launch (dram__bytes_read.sum + dram__bytes_write.sum) from one ncu
# --set full capture on this reach, with the wet cells of the captured step: scaled to the
# timed workload by its wet cells (the swept cells set the traffic).  Captured in the
# fourth step (t = 4 s) of python bench.py --spinup 0 --steps 3 --warmup 3 --no-cpu-baseline
# (ncu -k regex:k_hydro_sweep -s 6 -c 2: the 7th launch of the sweep kernel, the UZ sweep).
NCU_TRAFFIC = {
    "config2": {"sweep_uz": (2192640, 30650)},
    # config 4: the VZ sweep of the fourth step of python bench.py --workload config4
    # --spinup 0 --steps 3 --warmup 3 --no-cpu-baseline (ncu -k regex:k_hydro_sweep -s 6 -c 2)
    "config4": {"sweep_vz": (32254200 + 61696, 486100)},
}

# DRAM bytes of one whole timed step (dram__bytes_read.sum + dram__bytes_write.sum summed
# over the step's launches, the L2-flush kernels left out) from an ncu launch list of the
# timed steps; the summary, with its command, is the file named in "source".  Filled from
# captures of the current kernels; absent workloads print no step_dram.
STEP_DRAM = {
    "config2": {"bytes_per_step": 46.44e6, "source": "profiles/launch_list_config2_timed.md (ncu, every launch "
                "of 20 timed steps run cold: an upper bound)"},
    "config4": {"bytes_per_step": 501.47e6, "source": "profiles/step_dram_config2_config4.md (ncu, every launch "
                "of a timed step run cold: an upper bound)"},
}


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # the timed region starts once the sampler is running (first sample seen)
            t0 = time.time()
            while not self.lines and time.time() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        self.start_n = max(len(self.lines) - 1, 0)  # the last sample before the region, on
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines[getattr(self, "start_n", 0):]:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def wet_cells_per_line_sweep(sim):
    """Cells covered by the wet segments (the units the line sweeps process)."""
    import numpy as np
    kh = sim.get("khouot")
    return int((kh[2:sim.N + 1, 2:sim.M + 1] == 0).sum())


def span_cells(sim, halo=4):
    """Cells of the row spans of cells that can be wet (mask != 2, "core") and of the
    extended spans (every cell within `halo` rows and columns of those, "span"), the rule
    the library's span-limited kernels follow."""
    import numpy as np
    kh = sim.get("khouot")
    n, m = kh.shape
    act = kh != 2
    lo = np.where(act.any(1), act.argmax(1), n + m)
    hi = np.where(act.any(1), m - 1 - act[:, ::-1].argmax(1), -1)
    core = int(np.maximum(hi - lo + 1, 0).sum())
    elo = np.full(n, n + m)
    ehi = np.full(n, -1)
    for r in range(n):
        a, b = max(0, r - halo), min(n - 1, r + halo)
        lr, hr = lo[a:b + 1].min(), hi[a:b + 1].max()
        if hr >= lr:
            elo[r], ehi[r] = max(lr - halo, 0), min(hr + halo, m - 1)
    span = int(np.maximum(ehi - elo + 1, 0).sum())
    return core, span


def reference_kernels_sample(case, spin, n):
    """The reference's own kernels on this GPU (oracle/_ref/libhydref_gpu.so: its kernel
    sources built for sm_100a, launched as its host launches them): spun up untimed, then
    n steps timed by the harness's CUDA events.  None when that build is absent."""
    import oracle
    path = os.path.join(ROOT, "oracle", "_ref", "libhydref_gpu.so")
    if not os.path.exists(path):
        return None
    rs = oracle.RefSim(case, gpu=True)
    try:
        rs.init()
        rs.step(spin)
        t0 = rs.t
        rs.step(n)
        return {"value": case.N * case.M * n / (rs.last_ms / 1e3), "unit": "cell-updates/s", "steps": n,
                "sample": "the reference's kernels (its sources built for sm_100a, launched as Engine.py launches "
                          "them) on this GPU, %d steps from t=%.0f s after an untimed spin-up" % (n, t0)}
    finally:
        rs.close()


def cpu_port_sample(case, state_get, t0, hmax, budget_s=12.0):
    """Time the oracle port (OpenMP, all host cores) from the GPU's state."""
    import oracle
    ora = oracle.OracleSim(case, threads=os.cpu_count() or 1)
    ora.load_state(state_get, t0, hmax)
    ora.step(2)  # warm caches / thread pool
    steps, t_start = 0, time.perf_counter()
    while True:
        ora.step(10)
        steps += 10
        el = time.perf_counter() - t_start
        if el >= budget_s:
            break
    return steps, el


def run_ours(args, rank, world, local_rank, workload, secondary=False):
    """One workload's measurement.  secondary: the extra workload printed beside the
    default one (its value, back-to-back rate, roofline, level-mirror e2e and a short CPU
    sample; not the heavier e2e variants nor the reference's kernels)."""
    import numpy as np
    import torch
    from hydist import cases
    from hydist.lib import Simulation

    torch.cuda.set_device(local_rank)
    case = getattr(cases, WORKLOADS[workload][0])()
    N, M = case.N, case.M
    cells = N * M
    sim = Simulation.from_case(case, device=local_rank)
    sim.step(args.spinup)
    ext = torch.cuda.ExternalStream(sim.stream_ptr(), device=local_rank)
    # a buffer twice the L2, written (on the library's stream) before every timed step
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def flushed_steps(n, s=None, st=None):
        """Run n steps of simulation s (default: the measured one) on its stream st, each
        after an L2 flush; the summed device time of the steps (ms)."""
        s = sim if s is None else s
        st = ext if st is None else st
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
        with torch.cuda.stream(st):
            for a, b in ev:
                flush.zero_()
                a.record(st)
                s.step(1, sync=False)
                b.record(st)
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in ev)

    def back_to_back(n, s, st):
        """n steps of s queued back to back on its stream st; device ms."""
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        s.step(n, sync=False)
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1)

    def max_ranks(v):
        t = torch.tensor([v], device="cuda")
        if world > 1:
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    # warm-up
    sim.step(args.warmup, sync=True)
    flushed_steps(args.warmup)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    l0 = sim.launch_count()
    with ClockSampler(local_rank) as clk:
        torch.cuda.nvtx.range_push("timed")
        ms = flushed_steps(args.steps)
        torch.cuda.nvtx.range_pop()
    launches = sim.launch_count() - l0
    torch.cuda.synchronize()
    t_max = torch.tensor([ms], device="cuda")
    if world > 1:
        torch.distributed.all_reduce(t_max, op=torch.distributed.ReduceOp.MAX)
        torch.distributed.barrier()
    ms = float(t_max.item())
    value = world * cells * args.steps / (ms / 1e3)
    if args.timed_only:  # profiling runs: the timed steps and nothing after them
        sim.close()
        return {"metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "timed_only": True,
                "config": {"workload": WORKLOADS[workload][1]}}

    # the same steps back to back, L2 kept warm between them
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(ext)
    sim.step(args.steps, sync=False)
    e1.record(ext)
    e1.synchronize()
    warm_ms = e0.elapsed_time(e1)
    t_warm = torch.tensor([warm_ms], device="cuda")
    if world > 1:
        torch.distributed.all_reduce(t_warm, op=torch.distributed.ReduceOp.MAX)
    warm_ms = float(t_warm.item())

    # the FP32-bulk mixed form of the same workload (precision_mode MIXED: coefficient
    # assembly, line sweeps, explicit momentum and sediment in FP32; the level's continuity
    # update, mass sums and Exner sums in FP64), spun up to the same time and timed the
    # same way
    from hydist.params import PRECISION_MIXED
    pm = case.params.copy()
    pm.precision_mode = PRECISION_MIXED
    simm = Simulation(pm, N, M, device=local_rank)
    simm.load_case(case)
    simm.step(args.spinup)
    extm = torch.cuda.ExternalStream(simm.stream_ptr(), device=local_rank)
    simm.step(args.warmup, sync=True)
    flushed_steps(args.warmup, simm, extm)
    mixed_ms = max_ranks(flushed_steps(args.steps, simm, extm))
    mixed_b2b = max_ranks(back_to_back(args.steps, simm, extm))
    simm.close()
    mixed = {"value": world * cells * args.steps / (mixed_ms / 1e3), "ms_per_step": mixed_ms / args.steps,
             "back_to_back": {"value": world * cells * args.steps / (mixed_b2b / 1e3),
                              "ms_per_step": mixed_b2b / args.steps},
             "speedup_vs_fp64": ms / mixed_ms, "dtype": "f32 bulk, f64 z update / mass sums / Exner",
             "model_bytes_per_cell_update": 116,
             "l2": "flushed before every timed step, as value"}

    # simulated hours per wall second of a morphodynamic run on this reach: hydraulics,
    # sediment and the bed change fed back every 10 min (bed_feedback, morfac 1,
    # bed_period 600 s), 2 simulated hours back to back from the spun-up state, FP64 and
    # mixed (the 30-day config-5 shape on the config-2 geometry; config 4's own forcing
    # does not stay stable with the bed fed back, so only config 2 runs it)
    morpho = None
    if not secondary and workload == "config2":
        morpho = {"sim_hours": 2.0, "bed_period_s": 600.0, "morfac": 1.0}
        for label, prec in (("fp64", 0), ("mixed", PRECISION_MIXED)):
            pq = case.params.copy()
            pq.precision_mode = prec
            pq.bed_feedback = 1
            pq.morfac = 1.0
            pq.bed_period = 600.0
            sq = Simulation(pq, N, M, device=local_rank)
            sq.load_case(case)
            sq.step(args.spinup)
            stq = torch.cuda.ExternalStream(sq.stream_ptr(), device=local_rank)
            nq = int(round(2 * 3600 / case.params.dT))
            sq.step(10, sync=True)
            mq = max_ranks(back_to_back(nq, sq, stq))
            assert sq.mass_balance()["nonfinite"] == 0
            morpho[label] = {"sim_h_per_wall_s": 2.0 / (mq / 1e3), "ms_per_step": mq / nq}
            sq.close()
        morpho["mixed_over_fp64"] = morpho["mixed"]["sim_h_per_wall_s"] / morpho["fp64"]["sim_h_per_wall_s"]

    # per-phase device timing: events around every phase (the shares), then around the
    # dominant phase alone (its launch time, disturbed least by the events)
    ksteps = max(20, min(args.steps, 200))
    sim.set_timing(True)
    flushed_steps(ksteps)
    rep = sim.timing_report()
    wet = wet_cells_per_line_sweep(sim)
    core, span = span_cells(sim)
    units = {"span": span, "core": core, "wet": wet}
    total_ms = sum(v[1] for v in rep.values())
    # the dominant kernel: the longest launch (each phase is one kernel launch) of the step's
    # main chain; the first half-step's sediment phases run beside it on a second stream,
    # so their event times include waiting for SMs
    dom = max(((k, v) for k, v in rep.items() if k not in ("bed",) + SIDE_PHASES),
              key=lambda kv: kv[1][1] / kv[1][0])
    dom_name = dom[0]
    sim.set_timing(True, phases=[dom_name])
    flushed_steps(ksteps)
    alone = sim.timing_report()
    sim.set_timing(False)
    dom_n, dom_ms = alone[dom_name]
    per_unit, unit = PHASE_BYTES.get(dom_name, (0, "core"))
    bytes_per_launch = per_unit * units[unit]
    avg_ms = dom_ms / dom_n
    peak, peak_kind = load_peaks()
    achieved = bytes_per_launch / (avg_ms / 1e3) / 1e9
    traffic = None
    captured = NCU_TRAFFIC.get(workload, {})
    if dom_name in captured:
        tb, tw = captured[dom_name]
        traffic = int(round(tb * units["wet"] / tw))
    phases = {k: {"launches": n, "ms_per_launch": t / n, "share": t / total_ms} for k, (n, t) in rep.items()}

    # end to end through the C ABI, host buffers in pinned memory: every step the boundary
    # forcing (the Q/Z and inflow-concentration tables of the open edges) in through
    # hyd_update_boundary, hyd_step(1), and the water level z out (the reference's data
    # flow: forcing in, levels out; the state stays on the device).  The levels reach the
    # host through the library's mirror (hyd_mirror_update_async: a full host copy of z
    # after every step, of which only the box of cells a step can change crosses PCIe);
    # e2e_full_field copies every cell of z every step instead (hyd_get_field_async)
    e2e_steps = max(10, min(args.steps, 100))

    def pinned(a):
        t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
        t.numpy()[...] = a
        return t

    tabs = [pinned(np.asarray(t, dtype=np.float64)) for t in case.tables]
    ccs = [pinned(np.asarray(t, dtype=np.float64)) for t in case.cc]
    # two pinned level buffers: step k's levels copy out (hyd_get_field_async, on the
    # library's copy stream) while step k + 1 runs
    z_host = [torch.empty((N + 3, M + 3), dtype=torch.float64, pin_memory=True) for _ in range(2)]

    def timed_max(fn):
        """Run fn between events on the library's stream; (device ms, max over ranks, and
        fn's result)."""
        torch.cuda.synchronize()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(ext)
        res = fn()
        a1.record(ext)
        a1.synchronize()
        t = torch.tensor([a0.elapsed_time(a1)], device="cuda")
        if world > 1:
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item()), res

    def mirror_loop(n):
        moved = 0
        view = None
        for _ in range(n):
            sim.update_boundary([t.numpy() for t in tabs], [t.numpy() for t in ccs])
            sim.step(1, sync=False)
            view, b = sim.mirror_update()
            moved += b
        sim.wait_fields()
        return view, moved

    def full_loop(n):
        for k in range(n):
            sim.update_boundary([t.numpy() for t in tabs], [t.numpy() for t in ccs])
            sim.step(1, sync=False)
            sim.get_async("z", z_host[k % 2].numpy())
        sim.wait_fields()

    h2d_bytes = sum(t.numel() * 8 for t in tabs + ccs)
    sim.mirror_open("z")
    # untimed warm-up of the same loops (first use of the snapshots and host buffers)
    mirror_loop(max(args.warmup, 3))
    e2e_ms, (view, moved) = timed_max(lambda: mirror_loop(e2e_steps))
    mirror_exact = bool(np.array_equal(view, sim.get("z")))
    sim.mirror_close()
    d2h_bytes = moved / e2e_steps
    e2e_value = world * cells * e2e_steps / (e2e_ms / 1e3)
    full_value = rt_value = None
    field_bytes = (N + 3) * (M + 3) * 8 * 4
    if not secondary:
        full_loop(max(args.warmup, 3))
        full_ms, _ = timed_max(lambda: full_loop(e2e_steps))
        full_value = world * cells * e2e_steps / (full_ms / 1e3)

        # the heavier round trip for reference: the whole state (z, u, v, FS) in and out
        names = ("z", "u", "v", "FS")
        host = {f: torch.empty((N + 3, M + 3), dtype=torch.float64, pin_memory=True) for f in names}
        for f in names:
            sim.get(f, out=host[f].numpy())

        def roundtrip_loop(n):
            for _ in range(n):
                for f in names:
                    sim.set(f, host[f].numpy())
                sim.step(1, sync=False)
                for f in names:
                    sim.get(f, out=host[f].numpy())

        roundtrip_loop(max(args.warmup, 3))
        rt_ms, _ = timed_max(lambda: roundtrip_loop(e2e_steps))
        rt_value = world * cells * e2e_steps / (rt_ms / 1e3)

    result = None
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline:
            st_t = sim.t
            hmax = sim.get("hmax")
            snap = {f: sim.get(f) for f in __import__("oracle").OracleSim.STATE_FIELDS}
            budget = args.cpu_seconds if not secondary else min(args.cpu_seconds, 6.0)
            n_cpu, el = cpu_port_sample(case, lambda f: snap[f], st_t, hmax, budget_s=budget)
            cpu = {"value": cells * n_cpu / el, "unit": "cell-updates/s", "cores": os.cpu_count(),
                   "kind": "port",
                   "sample": "%d ADI steps of the %dx%d reach from t=%.0f s (the GPU state), oracle port "
                             "(OpenMP, %d threads), %.1f s wall" % (n_cpu, N, M, st_t, os.cpu_count(), el)}
        ref_gpu = None
        if world == 1 and not args.no_reference_gpu and not secondary:
            # sediment active from t = 1800 s, as in the timed steps
            ref_gpu = reference_kernels_sample(case, int(round(1800 / case.params.dT)) + 5, 20)
        clocks = clk.summary()
        result = {
            "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": WORKLOADS[workload][2],
            "config": {"workload": "%s, t=%d..%d s" % (WORKLOADS[workload][1], args.spinup + 2 * args.warmup,
                                                        args.spinup + 2 * args.warmup + args.steps),
                       "grid": [N, M], "cells": cells, "wet_cells": wet,
                       "parallelism": "replicas%d" % world if world > 1 else "single",
                       "core_cells": core, "span_cells": span,
                       "touched_fraction": span / cells,
                       "l2": "256 MB written before every timed step (flush); steps timed one by one"},
            "back_to_back": {"value": world * cells * args.steps / (warm_ms / 1e3), "ms_per_step": warm_ms / args.steps,
                             "l2": "no flush between steps"},
            "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": h2d_bytes,
                    "d2h_bytes_per_step": d2h_bytes, "steps": e2e_steps,
                    "api": "hyd_update_boundary(Q/Z + concentration tables) + hyd_step(1) + "
                           "hyd_mirror_update_async(z): a full host copy of z after every step (checked equal "
                           "to hyd_get_field at the end: %s), only the box of cells a step can change copied, "
                           "while the next step runs" % mirror_exact},
            "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "bytes_per_launch": bytes_per_launch, "bytes_unit": "%d B x %d %s cells" % (
                             per_unit, units[unit], unit),
                         "ms_per_launch": avg_ms, "timed": "events around this phase alone, L2 flushed per step"},
            "step_roofline": {"bytes_per_cell_update": 208, "achieved": value * 208 / 1e9 / world, "peak": peak,
                              "frac": value * 208 / 1e9 / world / peak},
            "mixed": mixed,
            "morpho": morpho,
            "phases": phases,
            "cpu_baseline": cpu,
            "reference_kernels_gpu": ref_gpu,
            "clocks": clocks,
            "gpu_launches": launches,
        }
        if full_value is not None:
            result.update({
                    "e2e_full_field": {"value": full_value, "unit": "cell-updates/s", "h2d_bytes_per_step": h2d_bytes,
                                       "d2h_bytes_per_step": (N + 3) * (M + 3) * 8, "steps": e2e_steps,
                                       "api": "as e2e, with every cell of z copied every step (hyd_get_field_async into "
                                              "two pinned buffers in turn)"},
                    "e2e_state_roundtrip": {"value": rt_value, "unit": "cell-updates/s", "h2d_bytes_per_step": field_bytes,
                                            "d2h_bytes_per_step": field_bytes, "steps": e2e_steps,
                                            "api": "hyd_set_field(z,u,v,FS) + hyd_step(1) + hyd_get_field(z,u,v,FS), "
                                                   "pinned host buffers"},
            })
        dram = STEP_DRAM.get(workload)
        if dram:
            # the whole step's DRAM bytes as ncu counted them (every launch of a timed step),
            # against the step time of this run: what the step moves, not what it models
            b = dram["bytes_per_step"]
            result["step_dram"] = {"bytes_per_step": b, "achieved": b / (ms / args.steps / 1e3) / 1e9,
                                   "peak": peak, "unit": "GB/s",
                                   "frac": b / (ms / args.steps / 1e3) / 1e9 / peak,
                                   "source": dram["source"]}
        result["step_roofline"]["note"] = (
            "modelled: 208 B per cell-update charged to all %d cells, while the step's kernels touch "
            "%d cells (%.1f %%, touched_fraction); step_dram is the measured traffic" % (cells, span, 100.0 * span / cells))
        result["roofline"]["traffic_kind"] = "modelled from the ncu capture in NCU_TRAFFIC, scaled by wet cells"
    sim.close()
    return result


def run_ensemble(args, local_rank):
    """Config 3: the 96-reach ensemble on one GPU as one batch, stepped with batched
    launches (every phase one launch for all reaches, the batch step one CUDA graph),
    member by member (one graph and stream per reach), and as the autotuner chooses
    between those and the members' sweep shapes (`value`).  Spun up past the discharge
    ramp and the sediment start, then timed by CUDA events back to back."""
    import torch
    from hydist import cases
    from hydist.lib import Batch
    cs = cases.config3_cases()
    cells = sum(c.N * c.M for c in cs)
    b = Batch(cs, device=local_rank)
    b.set_fused(True)
    b.step(1805, sync=True)  # past the 0.5 h ramp; sediment active from 1800 s
    streams = [torch.cuda.ExternalStream(m.stream_ptr(), device=local_rank) for m in b.members]

    def timed(n):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(streams[0])
        for st in streams[1:]:
            st.wait_event(e0)
        b.step(n, sync=False)
        for st in streams[1:]:
            ev = torch.cuda.Event()
            ev.record(st)
            streams[0].wait_event(ev)
        e1.record(streams[0])
        e1.synchronize()
        return e0.elapsed_time(e1)

    out = {"workload": "config3 ensemble: 96 reaches (nx 128-1024, ny 64-512, dx=5m), dt=1s, FP64 "
                       "hydraulics+sediment, t=1810.. s", "reaches": len(cs), "cells": cells,
           "l2": "no flush (the reaches' fields, %d cells, exceed L2)" % cells}
    for label, fused in (("batched", True), ("per_member", False)):
        b.set_fused(fused)
        b.step(max(args.warmup, 3), sync=True)
        f0 = b.fused_steps()
        ms = timed(args.steps)
        out[label] = {"value": cells * args.steps / (ms / 1e3), "unit": "cell-updates/s",
                      "ms_per_step": ms / args.steps, "batched_steps": b.fused_steps() - f0}
    out["speedup_vs_per_member"] = out["per_member"]["ms_per_step"] / out["batched"]["ms_per_step"]
    # the autotuner's choice among per-member sweep shapes and the batched launches
    from hydist.tune import DEFAULT_CANDIDATES, tune_batch
    best, times = tune_batch(b, DEFAULT_CANDIDATES, steps=10)
    b.step(max(args.warmup, 3), sync=True)
    ms = timed(args.steps)
    out["tuned"] = {"policy": "batched" if best == ("fused",) else "per_member d=%d wide=%d" % tuple(best),
                    "value": cells * args.steps / (ms / 1e3), "unit": "cell-updates/s",
                    "ms_per_step": ms / args.steps,
                    "candidates_ms": {("batched" if k == ("fused",) else "d=%d wide=%d" % k): v * 1e3
                                      for k, v in times.items()}}
    out["value"] = out["tuned"]["value"]
    b.close()
    return out


def run_config5(args, local_rank, hours=12.0, seeds=8, snapshots=64, iters=800, warm=20, min_warm=1):
    """Config 5, the morphodynamic reach (1048 x 980, bed fed back every 10 min, 30 days
    stated): simulated hours per wall second of the plain FP64 run and of the quasi-steady
    form (FP32-bulk mixed steps; each 10-min period replaced by the surrogate's jump and at
    most `warm` plain steps judged by the steady residual; a rejected jump retried from the
    previous state, then the fallback to plain stepping),
    and the quasi-steady form's bed and level differences from the plain FP64 run, on a
    bounded sample of `hours` hours after a 2 h spin-up (the spin-up and the surrogate's
    data generation and training are not timed).  Timed by the host clock around
    synchronised calls: each period's decisions are taken on the host CPU, inside the
    library (hyd_quasi_steady_period)."""
    import numpy as np
    import torch
    from hydist import cases, morpho as MO, surrogate as S
    from hydist.lib import Simulation
    from hydist.params import PRECISION_MIXED
    spin = 7200
    days = (spin / 3600 + hours) / 24 + 0.05
    t0 = time.perf_counter()
    X, Y, W, crop, dropped = MO.generate(list(range(500, 500 + seeds)), snapshots, every=600, device=local_rank)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    net = S.Surrogate(device=local_rank, seed=0)
    t0 = time.perf_counter()
    L = MO.train(net, X, Y, W, iters=iters, batch=8, lr=2e-3)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    nsnap = int(X.shape[0])
    del X, Y, W

    def make(mixed):
        c = cases.config5_case(days=days)
        if mixed:
            p = c.params.copy()
            p.precision_mode = PRECISION_MIXED
            c.params = p
        sim = Simulation.from_case(c, device=local_rank)
        sim.step(spin)
        sim.synchronize()
        return sim, c

    ref, _ = make(False)
    t0 = time.perf_counter()
    ref.step(int(round(hours * 3600)))
    plain_s = time.perf_counter() - t0
    zr, dHr, wet = ref.get("z"), ref.get("dH"), ref.get("khouot") == 0
    ref_nonfinite = int((~np.isfinite(zr)).sum() + (~np.isfinite(dHr)).sum())
    ref.close()
    out = {"workload": "config5 morphodynamic reach 1048x980 dx=5m dt=1s, bed fed back every 600 s (morfac 1); "
                       "sample of %.0f h after a 2 h spin-up (30 days stated)" % hours,
           "sim_hours": hours,
           "plain_fp64": {"sim_h_per_wall_s": hours / plain_s, "wall_s": plain_s,
                          "steps": int(round(hours * 3600)), "bed_change_max_m": float(np.nanmax(np.abs(dHr))),
                          "nonfinite_cells": ref_nonfinite},
           "surrogate": {"snapshots": nsnap, "reaches_dropped": dropped, "iters": iters,
                         "loss_first": L[0], "loss_last": float(np.mean(L[-20:])), "generate_s": gen_s,
                         "train_s": train_s}}
    for label, use_net in (("quasi_steady_surrogate", True), ("quasi_steady_no_network", False)):
        sim, c = make(True)
        jump = MO.SurrogateJump(net, c, crop) if use_net else None
        q = MO.QuasiSteady(sim, c, warm=warm, gate=1e-4, jump=jump, min_warm=min_warm)
        t0 = time.perf_counter()
        q.run_until(spin + hours * 3600)
        wall = time.perf_counter() - t0
        z, dH = sim.get("z"), sim.get("dH")
        out[label] = {"sim_h_per_wall_s": hours / wall, "wall_s": wall, "speedup_vs_plain_fp64": plain_s / wall,
                      "periods_accepted": q.accepted, "periods_accepted_with_jump": q.jump_accepted,
                      "periods_fallback": q.fallbacks, "steps": q.steps,
                      "max_level_diff_m": float(np.nanmax(np.abs(z - zr)[wet])),
                      "max_bed_diff_m": float(np.nanmax(np.abs(dH - dHr))),
                      "nonfinite_cells": int((~np.isfinite(z)).sum() + (~np.isfinite(dH)).sum())}
        sim.close()
    return out


def run_surrogate(args, local_rank, B=16, H=1048, W=89, reps=30):
    """The surrogate's tensor-core kernels on a batch of B crops of the config-5 channel band
    (H x W cells; the activations of one 48-channel layer, 16 x 1048 x 89 x 48 BF16, are
    143 MB, above L2): the full-resolution 48 -> 48 convolution (`k_conv_tc`) alone, then
    the network's forward pass and one training iteration (forward, loss, backward through
    the data- and weight-gradient kernels, Adam), each timed with CUDA events on the
    stream the kernels run on.  The convolution's roofline: its MMA FLOPs (2 x pixels x
    9 taps x 48 x 48) against the measured BF16 peak and its activation bytes (48 channels
    in, 48 out, BF16) against the measured HBM copy bandwidth."""
    import torch
    from hydist import surrogate as S
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    net = S.Surrogate(device=local_rank, seed=0)
    g = torch.Generator(device="cpu").manual_seed(1)
    x = torch.zeros((B, H, W, S.CIN_PAD), dtype=torch.bfloat16)
    x[..., :S.IN_CH] = torch.randn((B, H, W, S.IN_CH), generator=g).to(torch.bfloat16)
    x = x.to(dev)
    y = torch.randn((B, H, W, S.OUT_CH), generator=g).to(dev)
    wgt = torch.ones((B, H, W), device=dev)
    l = 4  # full resolution, 48 -> 48, ReLU
    mode, cin, cout, relu = S.LAYERS[l]
    act = (torch.randn((B, H, W, cin), generator=g) * 0.5).to(torch.bfloat16).to(dev)
    wpk = S.pack_weights(net.w[l], S.pad16(cout), S.pad16(cin))
    stream = torch.cuda.current_stream(dev)

    def timed(fn, n):
        for _ in range(3):
            fn()
        torch.cuda.synchronize(dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(n):
            fn()
        b.record(stream)
        torch.cuda.synchronize(dev)
        return a.elapsed_time(b) / n

    conv_ms = timed(lambda: net.conv(act, B, H, W, cin, wpk, net.b[l], S.pad16(cout), cout, mode, relu, H, W), reps)
    fwd_ms = timed(lambda: net.forward(x), reps)

    def train_iter():
        pred, saved = net.forward(x)
        loss, dy = net.loss_grad(pred, y, wgt)
        gw, gb = net.backward(saved, dy)
        net.adam(gw + gb, lr=1e-4)

    train_ms = timed(train_iter, max(5, reps // 3))
    net.check_errors()
    npix = B * H * W
    flops = 2.0 * npix * 9 * cin * cout
    nbytes = npix * (cin + cout) * 2
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        peaks = {"tflops": float(d["bf16_tflops"]), "gbs": float(d["hbm_gbs"]), "kind": "measured"}
    except Exception:
        peaks = {"tflops": 1590.0, "gbs": 6650.0, "kind": "fallback"}
    tf = flops / (conv_ms * 1e-3) / 1e12
    gbs = nbytes / (conv_ms * 1e-3) / 1e9
    t_tensor = flops / (peaks["tflops"] * 1e12)
    t_hbm = nbytes / (peaks["gbs"] * 1e9)
    bound = "tensor" if t_tensor >= t_hbm else "hbm"
    return {"workload": "BF16 surrogate, batch %d x %d x %d cells (config-5 channel band), 6 conv layers width 48"
                        % (B, H, W),
            "conv_48x48": {"kernel": "k_conv_tc (SAME, 48 -> 48, ReLU)", "ms_per_launch": conv_ms,
                           "tflops": tf, "gbs": gbs, "mma_flops_per_launch": flops, "bytes_per_launch": nbytes,
                           "roofline": {"bound": bound, "achieved": tf if bound == "tensor" else gbs,
                                        "peak": peaks["tflops"] if bound == "tensor" else peaks["gbs"],
                                        "unit": "TFLOP/s" if bound == "tensor" else "GB/s",
                                        "frac": (tf / peaks["tflops"]) if bound == "tensor" else (gbs / peaks["gbs"]),
                                        "frac_tensor": tf / peaks["tflops"], "frac_hbm": gbs / peaks["gbs"],
                                        "speed_of_light_ms": 1e3 * max(t_tensor, t_hbm),
                                        "peak_kind": peaks["kind"]}},
            "forward": {"ms": fwd_ms, "cells_per_s": npix / (fwd_ms * 1e-3)},
            "train_iteration": {"ms": train_ms, "cells_per_s": npix / (train_ms * 1e-3)}}


def run_reference(args, rank):
    if rank != 0:
        return None
    import numpy as np
    import oracle
    from hydist import cases
    case = getattr(cases, WORKLOADS[args.workload][0])()
    cells = case.N * case.M
    ora = oracle.OracleSim(case, threads=os.cpu_count() or 1)
    ora.init()
    # the sample starts from the oracle's own spin-up state; spin-up is not timed
    spin = min(SPINUP_STEPS, args.ref_spinup)
    if spin:
        ora.step(spin)
    ora.step(max(1, args.warmup))
    per_step = []
    budget = args.cpu_seconds
    t_all = time.perf_counter()
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ora.step(1)
        per_step.append(time.perf_counter() - t0)
        if time.perf_counter() - t_all > budget:
            break
    n = len(per_step)
    el = sum(per_step)
    value = cells * n / el
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": 0,
        "steps": n, "warmup": args.warmup, "ms_per_step": el / n * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": WORKLOADS[args.workload][2],
        "config": {"workload": WORKLOADS[args.workload][1],
                   "grid": [case.N, case.M], "cells": cells},
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": "%d ADI steps after %d spin-up steps, oracle port (OpenMP)" % (n, spin)},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def relaunch_under_torchrun(n):
    """--gpus N > 1 without a launcher: run this command under torch.distributed.run with N
    ranks (one per GPU), so that the flag is never silently ignored."""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(n),
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--ref-spinup", type=int, default=200)
    ap.add_argument("--spinup", type=int, default=SPINUP_STEPS,
                    help="untimed steps before the warm-up (default: to t = 3590 s, sediment active)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own kernels on the GPU (oracle/_ref/libhydref_gpu.so)")
    ap.add_argument("--workload", default="config2", choices=sorted(WORKLOADS),
                    help="config2 (the default: the 1048x980 reach) or config4 (the 4096x2048 reach)")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the config-3 ensemble line")
    ap.add_argument("--no-config5", action="store_true", help="skip the config-5 morphodynamic line")
    ap.add_argument("--no-surrogate", action="store_true", help="skip the surrogate kernels' line")
    ap.add_argument("--surrogate-only", action="store_true",
                    help="time only the surrogate kernels (one JSON line; for profiling them)")
    ap.add_argument("--timed-only", action="store_true",
                    help="profiling runs: spin up, warm up, run the timed steps, print a short line and stop")
    ap.add_argument("--config5-hours", type=float, default=12.0,
                    help="simulated hours of the config-5 sample (720 = the stated 30 days)")
    ap.add_argument("--secondary", default="config4", choices=sorted(WORKLOADS) + ["none"],
                    help="a second workload measured in the same run and printed under 'workloads' "
                         "(default config4; 'none' skips it)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        sys.exit(relaunch_under_torchrun(args.gpus))
    if args.gpus != world:
        sys.stderr.write("bench.py: --gpus %d but WORLD_SIZE=%d ranks; launch one rank per GPU\n" % (args.gpus, world))
        sys.exit(2)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        res = run_reference(args, rank)
        if res is not None:
            print(json.dumps(res))
        return
    if args.surrogate_only:
        print(json.dumps(run_surrogate(args, local_rank)))
        return
    if world > 1:
        import datetime
        import torch
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        res = run_ours(args, rank, world, local_rank, args.workload)
        if args.secondary not in ("none", args.workload):
            res2 = run_ours(args, rank, world, local_rank, args.secondary, secondary=True)
            if res is not None:
                res.setdefault("workloads", {})[args.secondary] = res2
        if not args.no_ensemble and args.secondary != "none":
            ens = run_ensemble(args, local_rank)
            if res is not None:
                res.setdefault("workloads", {})["config3"] = ens
        if not args.no_config5 and args.secondary != "none" and world == 1:
            c5 = run_config5(args, local_rank, hours=args.config5_hours)
            if res is not None:
                res.setdefault("workloads", {})["config5"] = c5
        if not args.no_surrogate and args.secondary != "none" and world == 1:
            sg = run_surrogate(args, local_rank)
            if res is not None:
                res.setdefault("workloads", {})["surrogate"] = sg
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()
    if res is not None:
        print(json.dumps(res))


if __name__ == "__main__":
    main()
