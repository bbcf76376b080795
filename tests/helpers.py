"""Comparison helpers shared by the parity tests."""
import numpy as np

# parity tolerance of the plain FP64 form: relative L-infinity against the reference
REL_TOL = 1e-9
PARITY_FIELDS = ("z", "u", "v", "t_z", "t_u", "t_v", "FS", "dH", "H_moi", "Htdu", "Htdv")
EXACT_FIELDS = ("khouot", "moci", "mocj", "daui", "cuoii", "dauj", "cuoij")


def rel_linf(a, b):
    """max |a-b| / max |b| over entries finite in both; NaN positions must coincide."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    na, nb = ~np.isfinite(a), ~np.isfinite(b)
    if not np.array_equal(na, nb):
        return np.inf
    m = ~na
    if not m.any():
        return 0.0
    scale = np.max(np.abs(b[m]))
    d = np.max(np.abs(a[m] - b[m]))
    if scale == 0:
        return float(d)
    return float(d / scale)


def compare(sim_a, get_b, fields=PARITY_FIELDS, exact=EXACT_FIELDS, tol=REL_TOL):
    """Return {field: rel_linf}; raise AssertionError listing the fields over `tol`."""
    errs = {}
    bad = []
    for f in fields:
        e = rel_linf(sim_a.get(f), get_b(f))
        errs[f] = e
        if not e <= tol:
            bad.append((f, e))
    for f in exact:
        a, b = sim_a.get(f), get_b(f)
        if not np.array_equal(a, b):
            bad.append((f, "mismatch at %s" % (np.argwhere(a != b)[:3].tolist(),)))
    assert not bad, "parity failure: %s" % bad
    return errs
