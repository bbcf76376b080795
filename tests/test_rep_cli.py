"""The rep.py-compatible command line (rep.py:23-40, 145-173): its flags on the CPU, and a
short run of the channel case on the GPU."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ENV = dict(os.environ, PYTHONPATH=os.path.join(ROOT, "gpu-hydist_b200"))


def _rep(*args, timeout=600):
    return subprocess.run([sys.executable, "-m", "hydist.rep"] + list(args), capture_output=True, text=True,
                          timeout=timeout, env=ENV, cwd=ROOT)


def test_rep_flags():
    r = _rep("--help")
    assert r.returncode == 0
    for flag in ("--Device", "--hours", "--mins", "--sediment", "--bed_change", "--pick_up", "--pickup_dirs",
                 "--kenhhepng", "--kenhhepd", "--plot"):
        assert flag in r.stdout, flag


def test_rep_needs_a_case(tmp_path):
    r = subprocess.run([sys.executable, "-m", "hydist.rep", "--hours", "0"], capture_output=True, text=True,
                       timeout=120, env=ENV, cwd=str(tmp_path))
    assert r.returncode != 0 and "DirsOfInputs_1.txt" in r.stderr + r.stdout


def test_channel_flag_strings_follow_the_reference():
    sys.path.insert(0, os.path.join(ROOT, "gpu-hydist_b200"))
    from hydist.engine import _channel_flag
    assert _channel_flag(False) == 0 and _channel_flag(1) == 1 and _channel_flag(0) == 0
    # rep.py passes argparse strings: true, but never equal to 1 (no range shift)
    assert _channel_flag("True") == 2 and _channel_flag("1") == 2


@pytest.mark.gpu
def test_rep_runs_the_channel_case():
    r = _rep("--case", "config1", "--hours", "0", "--mins", "30")
    assert r.returncode == 0, r.stdout + r.stderr
    assert "total running time of  0 hours is" in r.stdout
