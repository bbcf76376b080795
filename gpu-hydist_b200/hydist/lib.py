"""ctypes binding of libhydist_b200.so (the C ABI declared in include/hydist_b200.h).

There is no CPU fallback: if the library or a CUDA device is missing, every call
raises.  The shared object is built in-tree by ``make -C gpu-hydist_b200``.
"""
import ctypes
import os

import numpy as np

from .params import HydCaseParams

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhydist_b200.so")
SEGL = 20

_lib = None

# int (*hyd_run_callback)(hyd_handle h, double t, void* user)
RUN_CALLBACK = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p)


class HydError(RuntimeError):
    pass


def load():
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise HydError("libhydist_b200.so not built (run: make -C gpu-hydist_b200)")
    lib = ctypes.CDLL(LIB_PATH)
    H = ctypes.c_void_p
    sig = {
        "hyd_last_error": (ctypes.c_char_p, []),
        "hyd_version": (ctypes.c_char_p, []),
        "hyd_params_default": (None, [ctypes.POINTER(HydCaseParams)]),
        "hyd_params_derive": (None, [ctypes.POINTER(HydCaseParams)]),
        "hyd_create": (ctypes.c_int, [ctypes.POINTER(HydCaseParams), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.POINTER(H)]),
        "hyd_destroy": (ctypes.c_int, [H]),
        "hyd_set_field": (ctypes.c_int, [H, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t]),
        "hyd_get_field": (ctypes.c_int, [H, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t]),
        "hyd_set_boundary": (ctypes.c_int, [H, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_int]),
        "hyd_init": (ctypes.c_int, [H, ctypes.c_double]),
        "hyd_get_field_async": (ctypes.c_int, [H, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t]),
        "hyd_wait_fields": (ctypes.c_int, [H]),
        "hyd_mirror_open": (ctypes.c_int, [H, ctypes.c_char_p]),
        "hyd_mirror_update_async": (ctypes.c_int, [H, ctypes.POINTER(ctypes.POINTER(ctypes.c_double)),
                                                   ctypes.POINTER(ctypes.c_size_t)]),
        "hyd_mirror_close": (ctypes.c_int, [H]),
        "hyd_update_boundary": (ctypes.c_int, [H, ctypes.c_void_p, ctypes.c_void_p]),
        "hyd_init_pickup": (ctypes.c_int, [H, ctypes.c_double]),
        "hyd_step": (ctypes.c_int, [H, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
        "hyd_run": (ctypes.c_int, [H, ctypes.c_double, ctypes.c_double, RUN_CALLBACK, ctypes.c_void_p,
                                   ctypes.POINTER(ctypes.c_double)]),
        "hyd_get_time": (ctypes.c_int, [H, ctypes.POINTER(ctypes.c_double)]),
        "hyd_set_params": (ctypes.c_int, [H, ctypes.POINTER(HydCaseParams)]),
        "hyd_synchronize": (ctypes.c_int, [H]),
        "hyd_mass_balance": (ctypes.c_int, [H, ctypes.c_void_p, ctypes.c_int]),
        "hyd_mass_budget": (ctypes.c_int, [H, ctypes.c_void_p, ctypes.c_int]),
        "hyd_checkpoint": (ctypes.c_int, [H, ctypes.c_int]),
        "hyd_quasi_steady_period": (ctypes.c_int, [H, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_longlong,
                                                   ctypes.c_int, ctypes.c_void_p]),
        "hyd_get_field_device": (ctypes.c_int, [H, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t]),
        "hyd_set_time": (ctypes.c_int, [H, ctypes.c_double]),
        "hyd_steady_residual": (ctypes.c_int, [H, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]),
        "hyd_add_levels": (ctypes.c_int, [H, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_longlong]),
        "hyd_state_size": (ctypes.c_int, [H, ctypes.POINTER(ctypes.c_size_t)]),
        "hyd_get_state": (ctypes.c_int, [H, ctypes.c_void_p, ctypes.c_size_t]),
        "hyd_set_state": (ctypes.c_int, [H, ctypes.c_void_p, ctypes.c_size_t]),
        "hyd_launch_count": (ctypes.c_int, [H, ctypes.POINTER(ctypes.c_longlong)]),
        "hyd_get_stream": (ctypes.c_int, [H, ctypes.POINTER(ctypes.c_void_p)]),
        "hyd_device_status": (ctypes.c_int, [H, ctypes.POINTER(ctypes.c_uint)]),
        "hyd_set_timing": (ctypes.c_int, [H, ctypes.c_int]),
        "hyd_set_timing_phases": (ctypes.c_int, [H, ctypes.c_uint]),
        "hyd_phase_name": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p)]),
        "hyd_timing_report": (ctypes.c_int, [H, ctypes.c_char_p, ctypes.c_size_t]),
        "hyd_batch_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_void_p)]),
        "hyd_batch_size": (ctypes.c_int, [H, ctypes.POINTER(ctypes.c_int)]),
        "hyd_batch_member": (ctypes.c_int, [H, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
        "hyd_batch_step": (ctypes.c_int, [H, ctypes.c_int, ctypes.c_int]),
        "hyd_batch_destroy": (ctypes.c_int, [H]),
        "hyd_batch_set_fused": (ctypes.c_int, [H, ctypes.c_int]),
        "hyd_batch_fused_steps": (ctypes.c_int, [H, ctypes.POINTER(ctypes.c_longlong)]),
        "hyd_set_sweep_shape": (ctypes.c_int, [H, ctypes.c_int, ctypes.c_int]),
        "hyd_get_sweep_shape": (ctypes.c_int, [H, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(rc):
    if rc != 0:
        raise HydError("hydist error %d: %s" % (rc, _lib.hyd_last_error().decode()))


def phase_ids(lib):
    """{phase name: bit index} of the library's step phases."""
    out, k = {}, 0
    name = ctypes.c_char_p()
    while lib.hyd_phase_name(k, ctypes.byref(name)) == 0:
        out[name.value.decode()] = k
        k += 1
    return out


def field_shape(name, N, M):
    if name in ("daui", "cuoii"):
        return (N + 2, SEGL), np.int32
    if name in ("dauj", "cuoij"):
        return (M + 2, SEGL), np.int32
    if name == "moci":
        return (N + 2,), np.int32
    if name == "mocj":
        return (M + 2,), np.int32
    if name in ("ubt", "ubp"):
        return (M + 2,), np.float64
    if name in ("vbt", "vbd"):
        return (N + 2,), np.float64
    if name == "hi":
        return (2 * (N + 3) + 2 * (M + 3),), np.float64
    if name == "hmax":
        return (4,), np.float64
    if name == "khouot":
        return (N + 3, M + 3), np.int32
    return (N + 3, M + 3), np.float64


class Simulation:
    """One device-resident simulation (a hyd_handle)."""

    def __init__(self, params, N, M, device=0):
        lib = load()
        self.lib = lib
        self.N, self.M = int(N), int(M)
        self._p = params.copy()
        h = ctypes.c_void_p()
        _check(lib.hyd_create(ctypes.byref(self._p), self.N, self.M, int(device), ctypes.byref(h)))
        self.h = h

    @classmethod
    def from_case(cls, case, device=0, init=True):
        sim = cls(case.params, case.N, case.M, device)
        sim.load_case(case, init)
        return sim

    @classmethod
    def _member(cls, lib, handle, params, N, M):
        """A view of a batch member's handle (owned by the batch, not closed by the view)."""
        sim = cls.__new__(cls)
        sim.lib, sim.h, sim.N, sim.M, sim._p = lib, handle, int(N), int(M), params.copy()
        sim._owned = False
        return sim

    def load_case(self, case, init=True):
        """Fields and boundary tables of `case` (and hyd_init unless init is False)."""
        for name in ("h", "hsnham", "VISCOIDX", "Fw", "Tsxw", "Tsyw", "u", "v", "z", "FS"):
            self.set(name, case.fields[name])
        self.set_boundary(case.boundary_type, case.tables, case.cc, case.total_time)
        if init:
            self.init(case.t_start)

    def set(self, name, arr):
        shape, dt = field_shape(name, self.N, self.M)
        a = np.ascontiguousarray(arr, dtype=dt)
        if a.shape != shape:
            raise ValueError("%s: expected shape %s, got %s" % (name, shape, a.shape))
        _check(self.lib.hyd_set_field(self.h, name.encode(), a.ctypes.data, a.size))

    def get(self, name, out=None):
        shape, dt = field_shape(name, self.N, self.M)
        a = out if out is not None else np.empty(shape, dtype=dt)
        _check(self.lib.hyd_get_field(self.h, name.encode(), a.ctypes.data, a.size))
        return a

    def set_boundary(self, boundary_type, tables, cc, total_time):
        bt = np.ascontiguousarray(boundary_type, dtype=np.int32)
        tabs = [np.ascontiguousarray(t, dtype=np.float64) for t in tables]
        ccs = [np.ascontiguousarray(t, dtype=np.float64) for t in cc]
        PD = ctypes.POINTER(ctypes.c_double)
        tp = (PD * 4)(*[t.ctypes.data_as(PD) for t in tabs])
        cp = (PD * 4)(*[t.ctypes.data_as(PD) for t in ccs])
        ns = (ctypes.c_int * 4)(*[int(t.shape[0]) for t in tabs])
        _check(self.lib.hyd_set_boundary(self.h, bt.ctypes.data, tp, cp, ns, int(total_time)))

    def get_async(self, name, out):
        """Start reading a grid field of doubles into `out` (a C-contiguous (N+3)x(M+3)
        float64 array, ideally a view of pinned memory) while later steps run; complete
        after wait_fields() or once the second get_async() after it has returned."""
        shape, dt = field_shape(name, self.N, self.M)
        if out.shape != shape or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("%s: expected a C-contiguous float64 array of shape %s" % (name, shape))
        _check(self.lib.hyd_get_field_async(self.h, name.encode(), out.ctypes.data, out.size))

    def wait_fields(self):
        _check(self.lib.hyd_wait_fields(self.h))

    def mirror_open(self, name="z"):
        """Keep a host mirror of z, u or v (two library-owned pinned copies, in turn)."""
        _check(self.lib.hyd_mirror_open(self.h, name.encode()))
        self._mirror_name = name

    def mirror_update(self):
        """Bring the next mirror copy up to date after the queued steps; returns (view,
        bytes moved).  The (N+3)x(M+3) view is complete once the next mirror_update() (or
        wait_fields()) has returned, and valid until the second later mirror_update()."""
        ptr = ctypes.POINTER(ctypes.c_double)()
        n = ctypes.c_size_t()
        _check(self.lib.hyd_mirror_update_async(self.h, ctypes.byref(ptr), ctypes.byref(n)))
        return np.ctypeslib.as_array(ptr, shape=(self.N + 3, self.M + 3)), n.value

    def mirror_close(self):
        _check(self.lib.hyd_mirror_close(self.h))

    def set_sweep_shape(self, ctas, wide):
        """Sweep CTAs (0: one per SM) and whether warps take every line up to 288 rows."""
        _check(self.lib.hyd_set_sweep_shape(self.h, int(ctas), int(wide)))

    def sweep_shape(self):
        c, w = ctypes.c_int(), ctypes.c_int()
        _check(self.lib.hyd_get_sweep_shape(self.h, ctypes.byref(c), ctypes.byref(w)))
        return c.value, w.value

    def update_boundary(self, tables, cc):
        """New values for the boundary tables of set_boundary (same shapes); uploaded in
        order with the steps (the arrays are free again on return)."""
        PD = ctypes.POINTER(ctypes.c_double)
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in list(tables) + list(cc)]
        tp = (PD * 4)(*[a.ctypes.data_as(PD) for a in arrs[:4]])
        cp = (PD * 4)(*[a.ctypes.data_as(PD) for a in arrs[4:]])
        _check(self.lib.hyd_update_boundary(self.h, tp, cp))

    def set_params(self, params):
        self._p = params.copy()
        _check(self.lib.hyd_set_params(self.h, ctypes.byref(self._p)))

    @property
    def params(self):
        return self._p.copy()

    def init(self, t_start=0.0):
        _check(self.lib.hyd_init(self.h, float(t_start)))

    def init_pickup(self, t_start=0.0):
        """hyd_init keeping the mask set with set("khouot", ...) (rep.py:126-131)."""
        _check(self.lib.hyd_init_pickup(self.h, float(t_start)))

    def step(self, n=1, sync=True):
        t = ctypes.c_double()
        _check(self.lib.hyd_step(self.h, int(n), 1 if sync else 0, ctypes.byref(t)))
        return t.value

    def synchronize(self):
        _check(self.lib.hyd_synchronize(self.h))

    def run(self, Tmax, interval=0.0, callback=None):
        """hyd_run: step while t < Tmax; at every whole multiple of `interval` s (and at the
        end) check for non-finite values (HydError if any) and call callback(t), whose true
        return ends the run.  Returns the time reached."""
        t = ctypes.c_double()
        if callback is None:
            cb = RUN_CALLBACK()
        else:
            cb = RUN_CALLBACK(lambda h, tt, user: 1 if callback(tt) else 0)
        _check(self.lib.hyd_run(self.h, float(Tmax), float(interval), cb, None, ctypes.byref(t)))
        return t.value

    @property
    def t(self):
        t = ctypes.c_double()
        _check(self.lib.hyd_get_time(self.h, ctypes.byref(t)))
        return t.value

    def mass_balance(self):
        out = np.zeros(5)
        _check(self.lib.hyd_mass_balance(self.h, out.ctypes.data, 5))
        return {"volume": out[0], "suspended": out[1], "bed_change": out[2], "wet_cells": int(out[3]),
                "nonfinite": int(out[4])}

    def mass_budget(self):
        """The water volume budget since init (hyd_mass_budget), m^3: net, gross in and out
        through the edges, volumes of the cells opened and closed by the wet/dry resets, the
        volume fed-back bed changes added to the depths, and the net per edge (up, down,
        left, right)."""
        out = np.zeros(12)
        _check(self.lib.hyd_mass_budget(self.h, out.ctypes.data, 12))
        return {"net_in": out[0], "gross_in": out[1], "gross_out": out[2], "opened": out[3], "closed": out[4],
                "bed": out[5], "edge_net": out[6:10].copy(), "added": out[10], "leak": out[11]}

    # quasi-steady support: device checkpoint, time, steady residual, level increments
    def checkpoint(self):
        """Save the whole device state in the handle's device slot (hyd_checkpoint)."""
        _check(self.lib.hyd_checkpoint(self.h, 0))

    def restore(self):
        """Restore the state and time of the last checkpoint()."""
        _check(self.lib.hyd_checkpoint(self.h, 1))

    def get_device(self, name, out):
        """Copy field `name` into the device tensor `out` (its packed shape and dtype)."""
        shape, dtype = field_shape(name, self.N, self.M)
        if tuple(out.shape) != shape or not out.is_contiguous() or not out.is_cuda or \
                out.element_size() != np.dtype(dtype).itemsize:
            raise ValueError("get_device needs a contiguous device tensor of shape %s" % (shape,))
        _check(self.lib.hyd_get_field_device(self.h, name.encode(), out.data_ptr(), int(np.prod(shape))))
        return out

    def quasi_steady_period(self, period, warm=20, min_warm=1, gate=1e-4, jump=None, i0=0, j0=0, retry=True):
        """One bed period of the quasi-steady form in the library (hyd_quasi_steady_period);
        jump: (du, dv, dz) FP32 device tensors of one shape, added at grid cell (i0, j0), or
        None.  Returns (accepted, accepted with the jump, steps taken)."""
        res = (ctypes.c_int * 3)()
        if jump is None:
            args = (None, None, None, 0, 0, 0, 0, 0)
        else:
            du, dv, dz = jump
            rows, cols = du.shape
            for a in (du, dv, dz):
                if tuple(a.shape) != (rows, cols) or not a.is_contiguous() or not a.is_cuda or a.element_size() != 4:
                    raise ValueError("the jump takes three contiguous FP32 device tensors of one shape")
            args = (du.data_ptr(), dv.data_ptr(), dz.data_ptr(), int(i0), int(j0), rows, cols, cols)
        _check(self.lib.hyd_quasi_steady_period(self.h, float(period), int(warm), int(min_warm), float(gate), *args,
                                                1 if retry else 0, ctypes.cast(res, ctypes.c_void_p)))
        return bool(res[0]), bool(res[1]), int(res[2])

    def set_time(self, t):
        _check(self.lib.hyd_set_time(self.h, float(t)))

    def steady_residual(self, snapshot=True):
        """(momentum, continuity) relative change since the last snapshot (hyd_steady_residual):
        ||d(u, v)|| / ||(u, v)|| and ||dz|| / ||H|| over the wet cells; inf before the first."""
        out = np.zeros(2)
        _check(self.lib.hyd_steady_residual(self.h, 1 if snapshot else 0, out.ctypes.data, 2))
        return float(out[0]), float(out[1])

    def add_levels(self, du, dv, dz, i0, j0):
        """Add FP32 device tensors du, dv, dz (rows x cols, contiguous) to u, v, z on the wet
        cells of the rectangle starting at grid cell (i0, j0) (hyd_add_levels)."""
        rows, cols = du.shape
        for a in (du, dv, dz):
            if tuple(a.shape) != (rows, cols) or not a.is_contiguous() or not a.is_cuda or a.element_size() != 4:
                raise ValueError("add_levels takes three contiguous FP32 device tensors of one shape")
        _check(self.lib.hyd_add_levels(self.h, du.data_ptr(), dv.data_ptr(), dz.data_ptr(), int(i0), int(j0), rows,
                                       cols, cols))

    def get_state(self):
        n = ctypes.c_size_t()
        _check(self.lib.hyd_state_size(self.h, ctypes.byref(n)))
        buf = np.zeros(n.value, dtype=np.uint8)
        _check(self.lib.hyd_get_state(self.h, buf.ctypes.data, buf.size))
        return buf

    def set_state(self, buf):
        b = np.ascontiguousarray(buf, dtype=np.uint8)
        _check(self.lib.hyd_set_state(self.h, b.ctypes.data, b.size))

    def launch_count(self):
        c = ctypes.c_longlong()
        _check(self.lib.hyd_launch_count(self.h, ctypes.byref(c)))
        return c.value

    def device_status(self):
        st = ctypes.c_uint()
        _check(self.lib.hyd_device_status(self.h, ctypes.byref(st)))
        return st.value

    def stream_ptr(self):
        """The library stream (cudaStream_t as an integer) for torch.cuda.ExternalStream."""
        p = ctypes.c_void_p()
        _check(self.lib.hyd_get_stream(self.h, ctypes.byref(p)))
        return p.value or 0

    def set_timing(self, enable, phases=None):
        """Bracket the step's phases with events: every phase, or only those named in
        `phases` (names as in timing_report)."""
        if not enable:
            _check(self.lib.hyd_set_timing(self.h, 0))
        elif phases is None:
            _check(self.lib.hyd_set_timing(self.h, 1))
        else:
            ids = phase_ids(self.lib)
            mask = 0
            for name in phases:
                mask |= 1 << ids[name]
            _check(self.lib.hyd_set_timing_phases(self.h, mask))

    def timing_report(self):
        buf = ctypes.create_string_buffer(8192)
        _check(self.lib.hyd_timing_report(self.h, buf, len(buf)))
        out = {}
        for line in buf.value.decode().splitlines():
            name, n, ms = line.split()
            out[name] = (int(n), float(ms))
        return out

    def close(self):
        if getattr(self, "h", None) and getattr(self, "_owned", True):
            self.lib.hyd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Independent reaches on one device (hyd_batch_*): member k is a Simulation view of
    the batch's handle k; step() advances all of them, side by side on the device."""

    def __init__(self, cases, device=0, init=True):
        lib = load()
        self.lib = lib
        n = len(cases)
        params = (HydCaseParams * n)(*[c.params.copy() for c in cases])
        dims = (ctypes.c_int * (2 * n))(*[v for c in cases for v in (c.N, c.M)])
        b = ctypes.c_void_p()
        _check(lib.hyd_batch_create(n, ctypes.cast(params, ctypes.c_void_p), ctypes.cast(dims, ctypes.c_void_p),
                                    int(device), ctypes.byref(b)))
        self.b = b
        self.members = []
        for k, c in enumerate(cases):
            h = ctypes.c_void_p()
            _check(lib.hyd_batch_member(b, k, ctypes.byref(h)))
            self.members.append(Simulation._member(lib, h, c.params, c.N, c.M))
        for sim, c in zip(self.members, cases):
            sim.load_case(c, init)

    def step(self, n=1, sync=True):
        _check(self.lib.hyd_batch_step(self.b, int(n), 1 if sync else 0))

    def set_fused(self, on=True):
        """Batched launches: every phase of a batch step one launch for all members, the
        step one CUDA graph (hyd_batch_set_fused)."""
        _check(self.lib.hyd_batch_set_fused(self.b, 1 if on else 0))

    def fused_steps(self):
        n = ctypes.c_longlong()
        _check(self.lib.hyd_batch_fused_steps(self.b, ctypes.byref(n)))
        return n.value

    def synchronize(self):
        for s in self.members:
            s.synchronize()

    def close(self):
        if getattr(self, "b", None):
            self.lib.hyd_batch_destroy(self.b)
            self.b = None
            self.members = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
