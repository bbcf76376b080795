"""Case parameters: a ctypes mirror of ``HydCaseParams`` (include/hydist_b200.h).

The reference selects its case by copying a ``constant_<case>.cuh`` over
``constant.cuh`` and recompiling (readme.md:13-15); here the same constants
(constant.cuh:31-118) are a run-time struct.  :func:`default_params` returns the
values of the reference's ``constant.cuh`` and the keyword defaults of
``Engine.hydraulic_Calculation`` (Engine.py:49-50).
"""
import ctypes
import math

PI_REF = 3.14159265359  # constant.cuh:3

_DOUBLE_FIELDS = [
    "dX", "dY", "dT",
    "dXbp", "dX2", "dYbp", "dY2", "dTchia2dX", "dTchia2dY", "QuyDoiTime", "QuyDoiPi", "HaiChiadT",
    "NANGDAY", "H_TINH", "Wind", "huonggio", "Zbandau", "heso", "mu_mn",
    "NDnen", "NDbphai", "NDbtrai", "NDbtren", "NDbduoi",
    "Tod", "Toe", "hstoe", "ghtoe", "Mbochat", "ro", "ros", "dm", "d90", "muy", "Dorong", "Sx",
    "sohn", "soha", "sohn1", "CORIOLIS_FORCE", "g", "Ks",
    "sediment_start", "bed_change_start",
]
_INT_FIELDS = ["ketdinh", "kenhhepd", "kenhhepng", "precision_mode"]
# morphodynamic feedback (no reference counterpart), after the reference's constants
_MORPHO_FIELDS = [("morfac", ctypes.c_double), ("bed_period", ctypes.c_double), ("bed_feedback", ctypes.c_int),
                  ("bed_fixed", ctypes.c_int), ("bed_min_depth", ctypes.c_double)]

PRECISION_FP64 = 0
PRECISION_MIXED = 1


class HydCaseParams(ctypes.Structure):
    _fields_ = ([(n, ctypes.c_double) for n in _DOUBLE_FIELDS] + [(n, ctypes.c_int) for n in _INT_FIELDS] +
                _MORPHO_FIELDS)

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}

    def copy(self):
        c = HydCaseParams()
        ctypes.pointer(c)[0] = self
        return c


def derive(p):
    """Recompute the derived constants from dX, dY, dT (constant.cuh:36-47)."""
    p.dXbp = p.dX * p.dX
    p.dX2 = 2 * p.dX
    p.dYbp = p.dY * p.dY
    p.dY2 = 2 * p.dY
    p.dTchia2dX = p.dT / (2 * p.dX)
    p.dTchia2dY = p.dT / (2 * p.dY)
    p.QuyDoiTime = 1.0 / 3600
    p.QuyDoiPi = 1.0 / PI_REF
    p.HaiChiadT = 2.0 / p.dT
    return p


def default_params(**overrides):
    """Values of the reference constant.cuh (constant.cuh:31-118) plus Engine defaults."""
    p = HydCaseParams()
    vals = dict(
        dX=10.0, dY=10.0, dT=2.0,
        NANGDAY=0.0, H_TINH=0.02, Wind=0.0, huonggio=0.0, Zbandau=0.0, heso=0.94, mu_mn=0.2,
        NDnen=0.0, NDbphai=0.5, NDbtrai=0.5, NDbtren=0.5, NDbduoi=0.5,
        Tod=0.06, Toe=0.15, hstoe=0.0, ghtoe=3.0, Mbochat=0.00001, ro=1000.0, ros=2000.0,
        dm=0.00001, d90=0.002, muy=1.01e-06, Dorong=0.5, Sx=2.0,
        sohn=8.0, soha=3.0, sohn1=3.0, CORIOLIS_FORCE=0.0, g=9.81, Ks=2.5 * 0.00001,
        sediment_start=36000.0, bed_change_start=72000.0,
        ketdinh=1, kenhhepd=0, kenhhepng=0, precision_mode=PRECISION_FP64,
        morfac=1.0, bed_period=0.0, bed_feedback=0, bed_fixed=0, bed_min_depth=0.0,
    )
    vals.update(overrides)
    for k, v in vals.items():
        setattr(p, k, v)
    derive(p)
    return p


def settling_velocity(p):
    """wss() of constant.cuh:131-133 evaluated on the host."""
    return 10 * p.muy / p.dm * (math.sqrt(1 + 0.01 * (p.Sx - 1) * 9.81 * p.dm ** 3 / p.muy ** 2) - 1)
