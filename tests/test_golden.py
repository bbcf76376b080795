"""The oracle against the committed golden fixtures (outputs of the reference's kernels).

The fixtures were produced by tests/golden/make_golden.py from the reference's own
kernel sources; this test needs neither the reference tree nor a GPU."""
import numpy as np
import pytest

import golden


@pytest.mark.parametrize("name", golden.names())
def test_oracle_matches_golden(oracle_lib, name):
    import oracle
    case, out = golden.load(name)
    a = oracle.OracleSim(case)
    a.init()
    a.step(case.nsteps)
    for f, ref in out.items():
        got = a.get(f)
        assert np.array_equal(got, ref, equal_nan=True), "%s: oracle differs from the reference kernels" % f


def test_golden_fixtures_present():
    assert len(golden.names()) >= 4
