"""ctypes front-ends of the parity checkers (test infrastructure only).

``OracleSim``  — the C restatement (liboracle.so), CPU, OpenMP.
``RefSim``     — the reference's own kernel sources run launch for launch
                 (_ref/libhydref_cpu.so on the CPU, _ref/libhydref_gpu.so on a B200).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and reference arms
import this module.  Both classes take a ``hydist.cases.Case``.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SEGL = 20

_libs = {}


def build(targets=("oracle", "ref_cpu")):
    """Build the checkers with oracle/Makefile (the _ref targets need the reference tree)."""
    subprocess.run(["make", "-s", "-C", HERE] + list(targets), check=True)


def _load(path):
    if path not in _libs:
        _libs[path] = ctypes.CDLL(path)
    return _libs[path]


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


def _boundary_args(case):
    bt = np.ascontiguousarray(case.boundary_type, dtype=np.int32)
    tabs = [np.ascontiguousarray(t, dtype=np.float64) for t in case.tables]
    ccs = [np.ascontiguousarray(t, dtype=np.float64) for t in case.cc]
    PD = ctypes.POINTER(ctypes.c_double)
    tp = (PD * 4)(*[t.ctypes.data_as(PD) for t in tabs])
    cp = (PD * 4)(*[t.ctypes.data_as(PD) for t in ccs])
    ns = (ctypes.c_int * 4)(*[int(t.shape[0]) for t in tabs])
    keep = (bt, tabs, ccs)
    return bt, tp, cp, ns, keep


class OracleSim:
    """The C restatement of the reference kernels."""

    def __init__(self, case, threads=0):
        from hydist.params import HydCaseParams  # noqa: F401  (struct layout)
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build(("oracle",))
        lib = _load(path)
        lib.ora_create.restype = ctypes.c_void_p
        lib.ora_create.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        lib.ora_field.restype = ctypes.c_void_p
        lib.ora_field.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int),
                                  ctypes.POINTER(ctypes.c_size_t)]
        lib.ora_set_boundary.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        lib.ora_init.argtypes = [ctypes.c_void_p, ctypes.c_double]
        lib.ora_init_pickup.argtypes = [ctypes.c_void_p, ctypes.c_double]
        lib.ora_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.ora_time.restype = ctypes.c_double
        lib.ora_time.argtypes = [ctypes.c_void_p]
        lib.ora_destroy.argtypes = [ctypes.c_void_p]
        lib.ora_set_threads.argtypes = [ctypes.c_int]
        lib.ora_tridiag.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 8
        lib.ora_derived_constants.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        lib.ora_set_time.argtypes = [ctypes.c_void_p, ctypes.c_double]
        lib.ora_set_hmax.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        self.lib = lib
        self.case = case
        self.N, self.M = case.N, case.M
        self._p = case.params.copy()
        if threads:
            lib.ora_set_threads(int(threads))
        self.h = lib.ora_create(ctypes.byref(self._p), case.N, case.M)
        if not self.h:
            raise RuntimeError("ora_create failed")
        for name in ("h", "hsnham", "VISCOIDX", "Fw", "Tsxw", "Tsyw", "u", "v", "z", "FS"):
            self.view(name)[...] = case.fields[name]
        bt, tp, cp, ns, keep = _boundary_args(case)
        if lib.ora_set_boundary(self.h, bt.ctypes.data, tp, cp, ns, int(case.total_time)) != 0:
            raise RuntimeError("ora_set_boundary failed")

    def view(self, name):
        is_int = ctypes.c_int()
        cnt = ctypes.c_size_t()
        ptr = self.lib.ora_field(self.h, name.encode(), ctypes.byref(is_int), ctypes.byref(cnt))
        if not ptr:
            raise KeyError(name)
        shape, dt = field_shape(name, self.N, self.M)
        ct = ctypes.c_int if is_int.value else ctypes.c_double
        arr = np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ct)), shape=(cnt.value,))
        return arr.reshape(shape)

    def get(self, name):
        return self.view(name).copy()

    def init(self):
        self.lib.ora_init(self.h, float(self.case.t_start))

    def init_pickup(self):
        """Initialise keeping the mask written into view("khouot") (rep.py:126-131)."""
        self.lib.ora_init_pickup(self.h, float(self.case.t_start))

    def step(self, n):
        self.lib.ora_step(self.h, int(n))

    STATE_FIELDS = ("u", "v", "z", "t_u", "t_v", "t_z", "Htdu", "Htdv", "H_moi", "htaiz", "htaiz_bd", "Kx1", "Ky1",
                    "FS", "tFS", "VTH", "Kx", "Ky", "Qbx", "Qby", "dH", "khouot", "daui", "cuoii", "moci", "dauj",
                    "cuoij", "mocj", "ubt", "ubp", "vbt", "vbd", "hi")

    def load_state(self, get, t, hmax4):
        """Resume from another implementation's state: `get(name)` returns each field."""
        for f in self.STATE_FIELDS:
            self.view(f)[...] = get(f)
        self.lib.ora_set_time(self.h, float(t))
        hm = np.ascontiguousarray(hmax4, dtype=np.float64)
        self.lib.ora_set_hmax(self.h, hm.ctypes.data)

    @property
    def t(self):
        return self.lib.ora_time(self.h)

    def close(self):
        if self.h:
            self.lib.ora_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RefSim:
    """The reference's own kernels, compiled by oracle/Makefile and run launch for launch."""

    def __init__(self, case, gpu=False):
        path = os.path.join(HERE, "_ref", "libhydref_gpu.so" if gpu else "libhydref_cpu.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        lib = _load(path)
        lib.ref_create.restype = ctypes.c_void_p
        lib.ref_create.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        lib.ref_set_field.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t]
        lib.ref_get_field.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t]
        lib.ref_set_boundary.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        lib.ref_init.argtypes = [ctypes.c_void_p, ctypes.c_double]
        lib.ref_init_pickup.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p]
        lib.ref_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.ref_time.restype = ctypes.c_double
        lib.ref_time.argtypes = [ctypes.c_void_p]
        lib.ref_last_ms.restype = ctypes.c_double
        lib.ref_last_ms.argtypes = [ctypes.c_void_p]
        lib.ref_destroy.argtypes = [ctypes.c_void_p]
        lib.ref_last_error.restype = ctypes.c_char_p
        self.lib = lib
        self.case = case
        self.N, self.M = case.N, case.M
        self._p = case.params.copy()
        self.h = lib.ref_create(ctypes.byref(self._p), case.N, case.M)
        if not self.h:
            raise RuntimeError("ref_create failed: %s" % lib.ref_last_error())
        for name in ("h", "hsnham", "VISCOIDX", "Fw", "Tsxw", "Tsyw", "u", "v", "z", "FS"):
            a = np.ascontiguousarray(case.fields[name], dtype=np.float64)
            self._check(lib.ref_set_field(self.h, name.encode(), a.ctypes.data, a.size))
        bt, tp, cp, ns, keep = _boundary_args(case)
        self._check(lib.ref_set_boundary(self.h, bt.ctypes.data, tp, cp, ns, int(case.total_time)))

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError("reference harness error %d: %s" % (rc, self.lib.ref_last_error()))

    def get(self, name):
        shape, dt = field_shape(name, self.N, self.M)
        a = np.zeros(shape, dtype=dt)
        self._check(self.lib.ref_get_field(self.h, name.encode(), a.ctypes.data, a.size))
        return a

    def init(self):
        self._check(self.lib.ref_init(self.h, float(self.case.t_start)))

    def init_pickup(self, mask):
        """Initialise with a pick-up mask loaded after Onetime_init (rep.py:126-131)."""
        m = np.ascontiguousarray(mask, dtype=np.int32)
        self._check(self.lib.ref_init_pickup(self.h, float(self.case.t_start), m.ctypes.data))

    def step(self, n):
        self._check(self.lib.ref_step(self.h, int(n)))

    @property
    def t(self):
        return self.lib.ref_time(self.h)

    @property
    def last_ms(self):
        return self.lib.ref_last_ms(self.h)

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
