"""The quasi-steady support entry points (GPU): device checkpoint and restore, the clock,
the steady residual and the level increments, each against host-side arithmetic on the
fields read back; then the quasi-steady morphodynamic loop (hydist.morpho.QuasiSteady):
its fallback path equal to plain stepping, and a sample of the morphodynamic reach against
the plain FP64 run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# the quasi-steady form's stated difference from the plain FP64 run over the six-hour
# sample (m): its approximation error, not rounding
QS_LEVEL_TOL = 2e-2
QS_BED_TOL = 5e-2


def _case():
    from hydist import cases
    return cases.islands_case()


def test_checkpoint_restore_is_exact():
    """A restored checkpoint gives back every field, the time and the budget, and the run
    continues bit for bit as it did from the saved state."""
    from hydist.lib import Simulation
    sim = Simulation.from_case(_case())
    sim.step(30)
    st0 = sim.get_state()
    b0 = sim.mass_budget()
    sim.checkpoint()
    sim.step(25)
    a = {f: sim.get(f) for f in ("z", "u", "v", "FS", "khouot")}
    t_a = sim.t
    sim.restore()
    assert sim.t == 30 * sim.params.dT
    assert np.array_equal(sim.get_state(), st0)
    b1 = sim.mass_budget()
    assert all(np.array_equal(np.asarray(b0[k]), np.asarray(b1[k])) for k in b0)
    sim.step(25)
    assert sim.t == t_a
    for f, v in a.items():
        assert np.array_equal(sim.get(f), v), f
    sim.close()


def test_steady_residual_matches_host():
    from hydist.lib import Simulation
    sim = Simulation.from_case(_case())
    sim.step(20)
    r = sim.steady_residual(snapshot=True)
    assert r == (np.inf, np.inf) or (np.isinf(r[0]) and np.isinf(r[1]))
    N, M = sim.N, sim.M
    u0, v0, z0 = sim.get("u"), sim.get("v"), sim.get("z")
    sim.step(1)
    u, v, z, H, kh = sim.get("u"), sim.get("v"), sim.get("z"), sim.get("H_moi"), sim.get("khouot")
    r = sim.steady_residual(snapshot=False)
    w = np.zeros_like(kh, dtype=bool)
    w[2:N + 1, 2:M + 1] = kh[2:N + 1, 2:M + 1] == 0
    mom = np.sqrt(((u - u0)[w] ** 2 + (v - v0)[w] ** 2).sum() / (u[w] ** 2 + v[w] ** 2).sum())
    con = np.sqrt(((z - z0)[w] ** 2).sum() / (H[w] ** 2).sum())
    assert abs(r[0] - mom) <= 1e-12 * mom and abs(r[1] - con) <= 1e-12 * con, (r, mom, con)
    # without a snapshot the reference state stays: the same residual again
    assert sim.steady_residual(snapshot=False) == r
    sim.close()


def test_add_levels_and_set_time():
    import torch
    from hydist.lib import Simulation
    sim = Simulation.from_case(_case())
    sim.step(20)
    N, M = sim.N, sim.M
    before = {f: sim.get(f) for f in ("z", "u", "v", "t_z", "H_moi", "htaiz", "khouot", "h", "Htdu", "Htdv")}
    b0 = sim.mass_budget()["added"]
    i0, j0, rows, cols = 3, 4, N - 6, M - 8
    g = torch.Generator().manual_seed(0)
    du = (torch.randn((rows, cols), generator=g) * 0.01).float().cuda()
    dv = (torch.randn((rows, cols), generator=g) * 0.01).float().cuda()
    dz = (torch.randn((rows, cols), generator=g) * 0.005).float().cuda()
    sim.add_levels(du, dv, dz, i0, j0)
    after = {f: sim.get(f) for f in before}
    kh = before["khouot"]
    sl = (slice(i0, i0 + rows), slice(j0, j0 + cols))
    wet = np.zeros_like(kh, dtype=bool)
    wet[sl] = kh[sl] == 0
    wet[:2, :] = False
    wet[:, :2] = False
    wet[N + 1:, :] = False
    wet[:, M + 1:] = False
    dz_full = np.zeros_like(before["z"])
    dz_full[sl] = dz.double().cpu().numpy()
    dz_full[~wet] = 0
    keep = wet & (before["htaiz"] + (before["z"] + dz_full) <= sim.params.H_TINH)
    dz_full[keep] = 0
    assert np.array_equal(after["z"], before["z"] + dz_full)
    assert np.array_equal(after["t_z"][wet], after["z"][wet])
    assert np.array_equal(after["H_moi"][wet], (before["htaiz"] + after["z"])[wet])
    du_full = np.zeros_like(before["u"])
    du_full[sl] = du.double().cpu().numpy()
    assert np.array_equal(after["u"][wet], (before["u"] + du_full)[wet])
    assert np.array_equal(after["u"][~wet], before["u"][~wet])
    # face depths of the changed rows (Htuongdoi)
    h, z = after["h"], after["z"]
    i, j = i0 + 2, j0 + 2
    assert after["Htdu"][i, j] == (h[i, j - 1] + h[i, j] + z[i + 1, j] + z[i, j]) * 0.5
    added = sim.mass_budget()["added"] - b0
    area = sim.params.dX * sim.params.dY
    assert abs(added - dz_full[wet].sum() * area) <= 1e-9 * max(1.0, abs(added))
    # the clock: a step after set_time ends at the new time + dT
    sim.set_time(100.0)
    sim.step(1)
    assert sim.t == 100.0 + sim.params.dT
    assert np.isfinite(sim.get("z")).all()
    sim.close()


def _config5(hours):
    from hydist import cases
    from hydist.params import PRECISION_MIXED
    c = cases.config5_case(days=(2.0 + hours) / 24 + 0.05)
    p = c.params.copy()
    p.precision_mode = PRECISION_MIXED
    c.params = p
    return c


def test_quasi_steady_fallback_is_plain_stepping():
    """With a gate no state can pass, every period falls back: restored from the device
    checkpoint and stepped plainly, which must give the plain run bit for bit."""
    from hydist import morpho as MO
    from hydist.lib import Simulation
    c = _config5(1.0)
    a = Simulation.from_case(c)
    a.step(7200)
    b = Simulation.from_case(c)
    b.step(7200)
    q = MO.QuasiSteady(b, c, warm=20, gate=0.0)
    q.run_until(7200 + 3600)
    a.step(3600)
    assert q.fallbacks == 6 and q.accepted == 0
    assert a.t == b.t
    for f in ("z", "u", "v", "FS", "dH", "h"):
        assert np.array_equal(a.get(f), b.get(f)), f
    a.close()
    b.close()


def test_quasi_steady_config5_sample():
    """Six hours of the morphodynamic reach (bed fed back every 10 min) after a 2 h spin-up:
    the quasi-steady form (FP32-bulk steps, no network: the previous state is the warm
    start) against the plain FP64 run.  Most periods pass the gate within the warm steps,
    the steps taken fall by more than 5x, and the level and bed stay within the stated
    bounds of the FP64 run (QS_LEVEL_TOL, QS_BED_TOL: the quasi-steady approximation's own
    error, the flow and the suspended sediment not following the period's forcing and bed
    changes step by step)."""
    from hydist import morpho as MO
    from hydist.lib import Simulation
    hours = 6.0
    c = _config5(hours)
    from hydist import cases
    cref = cases.config5_case(days=(2.0 + hours) / 24 + 0.05)
    ref = Simulation.from_case(cref)
    ref.step(7200 + int(hours * 3600))
    sim = Simulation.from_case(c)
    sim.step(7200)
    q = MO.QuasiSteady(sim, c, warm=20, gate=1e-4)
    q.run_until(7200 + hours * 3600)
    assert sim.t == ref.t
    wet = ref.get("khouot") == 0
    dz = float(np.abs(sim.get("z") - ref.get("z"))[wet].max())
    db = float(np.abs(sim.get("dH") - ref.get("dH")).max())
    nplain = int(hours * 3600)
    print("quasi-steady %.0f h: %d of %d periods accepted, %d steps (plain %d), level diff %.2e m, bed diff %.2e m "
          "(bed change up to %.3f m)" % (hours, q.accepted, q.accepted + q.fallbacks, q.steps, nplain, dz, db,
                                         float(np.abs(ref.get("dH")).max())))
    assert q.accepted >= 0.75 * (q.accepted + q.fallbacks)
    assert q.steps * 5 < nplain
    assert dz <= QS_LEVEL_TOL and db <= QS_BED_TOL
    assert sim.mass_balance()["nonfinite"] == 0
    sim.close()
    ref.close()


class _AlternatingJump:
    """A fixed level increment over the reach's crop, large on odd periods (for the gate
    to reject, and the retry without it to run) and small on even ones."""

    def __init__(self, crop):
        self.crop = crop
        self.k = 0

    def increments(self, sim, Q, stage):
        import torch
        _, rows, _, cols = self.crop
        self.k += 1
        amp = 5e-2 if self.k % 2 else 1e-4
        g = torch.Generator().manual_seed(self.k)
        dz = (amp * torch.rand((rows, cols), generator=g)).float().cuda()
        zero = torch.zeros_like(dz)
        return zero, zero.clone(), dz


def test_native_period_matches_the_host_loop():
    """hyd_quasi_steady_period makes the calls of the host loop in the same order: both
    give the same fields bit for bit and the same counters, with a jump that is accepted
    on some periods and retried without on others."""
    from hydist import morpho as MO
    from hydist.lib import Simulation
    c = _config5(1.0)
    crop = MO.reach_crop(c)
    out = []
    for native in (False, True):
        sim = Simulation.from_case(c)
        sim.step(7200)
        q = MO.QuasiSteady(sim, c, warm=20, gate=1e-4, jump=_AlternatingJump(crop), native=native)
        assert q.native == native
        q.run_until(7200 + 3600)
        out.append(((q.accepted, q.jump_accepted, q.fallbacks, q.steps, sim.t),
                    {f: sim.get(f) for f in ("z", "u", "v", "FS", "dH", "h")}))
        sim.close()
    (ca, fa), (cb, fb) = out
    print("host loop: accepted %d (jump %d), fallbacks %d, steps %d" % ca[:4])
    assert ca == cb
    assert ca[0] + ca[2] == 6
    for f in fa:
        assert np.array_equal(fa[f], fb[f]), f
