"""hyd_mass_balance_noalloc against hyd_mass_balance, through the C ABI (GPU).

The new entry point takes its partial sums from a fixed device array instead of a
per-call allocation; it must return the same domain sums.  Collected last so that it
also runs after every other test in the same process.
"""
import ctypes

import numpy as np
import pytest

import golden
from hydist import lib as hlib
from hydist.lib import Simulation

pytestmark = pytest.mark.gpu

REL = 1e-12  # block-order summation differences only


def _noalloc(lib):
    fn = lib.hyd_mass_balance_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
    return fn


def _allocating(sim):
    out = np.zeros(5)
    assert sim.lib.hyd_mass_balance(sim.h, out.ctypes.data, 5) == 0
    return out


def _close(a, b):
    for k in range(3):
        assert abs(a[k] - b[k]) <= REL * max(abs(a[k]), abs(b[k]), 1e-300), (k, a[k], b[k])
    assert a[3] == b[3] and a[4] == b[4]


def test_noalloc_mass_balance_matches_allocating_entry_point():
    case, _ = golden.load("islands")
    sim = Simulation.from_case(case)
    sim.step(case.nsteps)
    fn = _noalloc(hlib.load())
    ref = _allocating(sim)
    assert ref[0] > 0 and ref[3] > 0
    for _ in range(2):  # two calls in a row
        for nblocks in (148, 37):
            out = np.zeros(5)
            rc = fn(sim.h, nblocks, out.ctypes.data, 5)
            assert rc == 0, hlib.load().hyd_last_error()
            _close(out, ref)
    # and after the state moves on, both entry points again agree
    sim.step(10)
    ref2 = _allocating(sim)
    out = np.zeros(5)
    assert fn(sim.h, 148, out.ctypes.data, 5) == 0
    _close(out, ref2)
    sim.close()


def test_noalloc_mass_balance_rejects_oversize():
    case, _ = golden.load("channel_small")
    sim = Simulation.from_case(case)
    lib = hlib.load()
    fn = _noalloc(lib)
    out = np.zeros(5)
    for bad in (0, 1025):
        assert fn(sim.h, bad, out.ctypes.data, 5) == -1
        assert b"1..1024" in lib.hyd_last_error()
    assert fn(sim.h, 1024, out.ctypes.data, 5) == 0
    sim.close()


_PROBE = r"""
import ctypes, sys
import numpy as np
sys.path[:0] = sys.argv[1:]
import torch
import golden
from hydist import lib as hlib
from hydist.lib import Simulation
case, _ = golden.load("islands")
sim = Simulation.from_case(case)
sim.step(case.nsteps)
torch.cuda.synchronize()
fn = hlib.load().hyd_mass_balance_noalloc
fn.restype = ctypes.c_int
fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
free0 = torch.cuda.mem_get_info()[0]
out = np.zeros(5)
for _ in range(5):
    assert fn(sim.h, 148, out.ctypes.data, 5) == 0, hlib.load().hyd_last_error()
torch.cuda.synchronize()
free1 = torch.cuda.mem_get_info()[0]
print("FREE", free0, free1, out[0])
"""


def test_noalloc_first_calls_allocate_nothing_with_lazy_loading():
    """With CUDA's lazy module loading, the module holding the fixed array would load at
    its first use and take device memory then; the handle's creation loads it, so calls
    made afterwards, with no hyd_mass_balance call before them, leave the device's free
    memory unchanged.  Run in a fresh process with CUDA_MODULE_LOADING=LAZY."""
    import os
    import subprocess
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    paths = [os.path.join(root, "gpu-hydist_b200"), here, os.path.join(here, "golden")]
    env = dict(os.environ, CUDA_MODULE_LOADING="LAZY")
    r = subprocess.run([sys.executable, "-c", _PROBE] + paths, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("FREE")][-1]
    _, free0, free1, vol = line.split()
    assert int(free0) == int(free1), "free device memory changed across the no-allocation calls: %s -> %s" % (
        free0, free1)
    assert float(vol) > 0
