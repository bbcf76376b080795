"""Shared test set-up: import paths, the `gpu` marker, built checkers."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "gpu-hydist_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests"),
          os.path.join(ROOT, "tests", "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)

# the reference tree (read-only, absent on GPU machines): $HYDIST_REFERENCE, default below
REFERENCE_TREE = os.environ.get("HYDIST_REFERENCE", "/root/reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        oracle.build(("oracle",))
    return oracle


@pytest.fixture(scope="session")
def ref_cpu_lib():
    """The reference's own kernels, compiled for the CPU by oracle/Makefile."""
    import oracle
    path = os.path.join(ROOT, "oracle", "_ref", "libhydref_cpu.so")
    if not os.path.exists(path):
        if not os.path.isdir(REFERENCE_TREE):
            pytest.skip("reference tree absent and oracle/_ref/libhydref_cpu.so not built")
        oracle.build(("ref_cpu",))
    return oracle
