"""The C-ABI library loads and exports every entry point include/hydist_b200.h declares."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hydist_b200.h")
LIB = os.path.join(ROOT, "gpu-hydist_b200", "hydist", "libhydist_b200.so")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hyd_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_api():
    syms = declared_symbols()
    for s in ("hyd_create", "hyd_step", "hyd_set_field", "hyd_get_field", "hyd_init", "hyd_destroy"):
        assert s in syms


def test_library_exports_all_symbols():
    if not os.path.exists(LIB):
        subprocess = __import__("subprocess")
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "gpu-hydist_b200")], check=True)
    lib = ctypes.CDLL(LIB)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_params_struct_layout():
    """The Python mirror of HydCaseParams has the C layout (44 doubles + 4 ints of the
    reference's constants and run options, then 2 doubles + 2 ints of the morphodynamic
    feedback)."""
    from hydist.params import HydCaseParams, default_params
    assert ctypes.sizeof(HydCaseParams) == 47 * 8 + 6 * 4
    assert HydCaseParams.morfac.offset == 44 * 8 + 4 * 4
    p = default_params()
    assert p.dXbp == p.dX * p.dX and p.HaiChiadT == 2.0 / p.dT


def test_params_default_matches_library():
    from hydist.params import HydCaseParams, default_params
    lib = ctypes.CDLL(LIB)
    c = HydCaseParams()
    lib.hyd_params_default(ctypes.byref(c))
    p = default_params()
    for name, _ in HydCaseParams._fields_:
        assert getattr(c, name) == getattr(p, name), name


def test_no_device_fails_loudly():
    """Without a GPU, creating a simulation is an error (there is no CPU path)."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    from hydist import lib as hl
    from hydist.params import default_params
    with pytest.raises(hl.HydError):
        hl.Simulation(default_params(), 16, 16)
