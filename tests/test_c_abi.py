"""A C host against include/hydist_b200.h alone (tests/c_abi/forcing_loop.c): it compiles
with gcc here, and on the GPU it sets up a reach, runs the forcing-in / levels-out loop,
the reference's time loop (hyd_run) with an output callback, and closes the water budget."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c_abi", "forcing_loop.c")
LIBDIR = os.path.join(ROOT, "gpu-hydist_b200", "hydist")


def _build(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libhydist_b200.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "gpu-hydist_b200")], check=True)
    exe = str(tmp_path / "forcing_loop")
    r = subprocess.run(["gcc", "-std=c99", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                        SRC, "-o", exe, "-L", LIBDIR, "-lhydist_b200", "-Wl,-rpath," + LIBDIR, "-lm"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_c_host_compiles(tmp_path):
    _build(tmp_path)


@pytest.mark.gpu
def test_c_host_runs(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "forcing_loop ok" in r.stdout
