"""The library's span-limited stepping rests on one property of the reference's scheme:
after the first step's whole-grid passes, z, u and v change only within the extended
spans (every cell within 4 rows and columns of a cell whose mask is not 2; such masks
never change).  The level mirror copies only the box of those spans for the same reason.
Checked here on the oracle (the reference's arithmetic) over the golden cases, config 1
and a reach with sediment and bed change: no cell outside the spans changes."""
import numpy as np
import pytest

HALO = 4  # kSpanHalo of the library's span kernels


def extended_spans(kh, halo=HALO):
    """(elo, ehi) per row, empty rows as (1, 0), as k_spans + k_ext_spans compute them."""
    n, m = kh.shape
    act = kh != 2
    rlo = np.where(act.any(1), act.argmax(1), 1 << 30)
    rhi = np.where(act.any(1), m - 1 - act[:, ::-1].argmax(1), -1)
    elo = np.ones(n, dtype=np.int64)
    ehi = np.zeros(n, dtype=np.int64)
    for i in range(n):
        a, b = max(0, i - halo), min(n - 1, i + halo)
        ok = rhi[a:b + 1] >= rlo[a:b + 1]
        if ok.any():
            elo[i] = max(int((rlo[a:b + 1][ok] - halo).min()), 0)
            ehi[i] = min(int((rhi[a:b + 1][ok] + halo).max()), m - 1)
    return elo, ehi


def outside_mask(kh):
    elo, ehi = extended_spans(kh)
    j = np.arange(kh.shape[1])[None, :]
    return (j < elo[:, None]) | (j > ehi[:, None])


def _cases():
    import golden
    from hydist import cases
    out = [(n, lambda n=n: golden.load(n)[0]) for n in golden.names()]
    out.append(("config1", cases.config1_case))
    out.append(("islands_bed", lambda: cases.islands_case(N=60, M=44, seed=5, bed_change_start=6.0)))
    return out


@pytest.mark.parametrize("name,make", _cases(), ids=[c[0] for c in _cases()])
def test_fields_change_only_inside_spans(name, make, oracle_lib):
    import oracle
    c = make()
    ora = oracle.OracleSim(c)
    ora.init()
    ora.step(1)
    kh0 = ora.get("khouot")
    out = outside_mask(kh0)
    ref = {f: ora.get(f) for f in ("z", "u", "v")}
    changed_inside = False
    for _ in range(12):
        ora.step(2)
        kh = ora.get("khouot")
        assert np.array_equal(kh == 2, kh0 == 2), "%s: a mask-2 cell changed" % name
        for f, r in ref.items():
            a = ora.get(f)
            diff = out & ~((a == r) | (np.isnan(a) & np.isnan(r)))
            assert not diff.any(), "%s t=%g: %s changed outside the spans at %s" % (
                name, ora.t, f, np.argwhere(diff)[:3].tolist())
            changed_inside |= bool((~out & (a != r)).any())
    assert changed_inside, "%s: nothing moved (the check would be empty)" % name
