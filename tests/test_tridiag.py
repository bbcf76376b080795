"""Known-answer tests of the reference Thomas solver restated in the oracle."""
import ctypes

import numpy as np


def _solve(oracle_lib, a, b, c, d):
    import oracle
    lib = oracle._load(oracle.os.path.join(oracle.HERE, "liboracle.so"))
    lib.ora_tridiag.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 8
    n = len(b)
    x = np.zeros(n)
    ap, bp, ep = np.zeros(n), np.zeros(n), np.zeros(n)
    arrs = [np.ascontiguousarray(v, dtype=np.float64) for v in (a, b, c, d)]
    lib.ora_tridiag(n - 1, *[v.ctypes.data for v in arrs], x.ctypes.data, ap.ctypes.data, bp.ctypes.data,
                    ep.ctypes.data)
    return x


def test_thomas_random_dominant(oracle_lib):
    rng = np.random.default_rng(3)
    for n in (1, 2, 3, 17, 200):
        a = rng.uniform(-1, 1, n)
        c = rng.uniform(-1, 1, n)
        b = np.abs(a) + np.abs(c) + rng.uniform(0.5, 2, n)
        d = rng.uniform(-5, 5, n)
        A = np.diag(b) + np.diag(a[1:], -1) + np.diag(c[:-1], 1)
        x = _solve(oracle_lib, a, b, c, d)
        assert np.allclose(x, np.linalg.solve(A, d), rtol=1e-12, atol=1e-12)


def test_thomas_interleaved_wave_rows(oracle_lib):
    """Rows alternating continuity (a2, 1, c2) and momentum (a1, b1, c1) like the UZ sweep."""
    rng = np.random.default_rng(5)
    n = 41
    a = np.empty(n); b = np.empty(n); c = np.empty(n)
    for r in range(n):
        if r % 2 == 0:
            a[r], b[r], c[r] = -0.2 * rng.uniform(2, 8), 1.0, 0.2 * rng.uniform(2, 8)
        else:
            a[r], b[r], c[r] = 3.92 + rng.uniform(0, 0.1), -2.0 - rng.uniform(0, 0.5), -3.92 - rng.uniform(0, 0.1)
    d = rng.uniform(-1, 1, n)
    A = np.diag(b) + np.diag(a[1:], -1) + np.diag(c[:-1], 1)
    x = _solve(oracle_lib, a, b, c, d)
    assert np.allclose(A @ x, d, rtol=1e-10, atol=1e-10)
