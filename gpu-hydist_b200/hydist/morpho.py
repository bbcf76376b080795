"""Quasi-steady morphodynamics with the surrogate's jump: the fast form of a long
morphodynamic run (the 30-day, 10-minute bed-update workload).

The plain run steps the hydraulics and the sediment every dT and feeds the bed change
back every bed period (bed_feedback).  Between two bed updates the flow of a slowly
forced reach stays close to the equilibrium of the current bed and forcing, and the bed
update only reads the state at the period's end.  The quasi-steady form therefore
replaces the period's steps by a jump to that equilibrium and a few plain steps:

  1. checkpoint the device state (hyd_checkpoint);
  2. the jump: the surrogate's predicted change of (u, v, z) from the last period's
     (bed, forcing) to this one's, added on the wet cells (hyd_add_levels), or no jump
     (the method without the network: the previous state is the warm start);
  3. the clock moved to `warm` steps before the period's end (hyd_set_time) and plain
     ADI steps taken, the steady residual (hyd_steady_residual: relative velocity change
     per step, and level change per depth) read after each;
  4. once both residuals are below the gate (read from the `min_warm`-th warm step on)
     and the state is finite,
     the clock is moved to the last step of the period and that step taken, which makes
     the period's bed update on the accepted state; if the residual has not fallen below
     the gate within `warm` - 1 steps, the checkpoint is restored and the period stepped
     plainly (the fallback).

No reference counterpart (the reference steps every dT, Engine.py:144-366, and never
feeds the bed back).  The surrogate's data are plain-solver snapshots of config-5-style
reaches (other seeds of the same generator) along their slowly varying forcing.
"""
import math
import time

import numpy as np

from . import cases
from . import surrogate as S
from .lib import HydError, Simulation

H_REF, N_REF, Q_REF, STAGE_REF, DZ_REF = 8.0, 0.025, 700.0, 0.3, 0.1
# trust region of one jump: the surrogate's increments are clipped to these (m/s, m/s, m)
JUMP_MAX = (0.1, 0.1, 0.05)
# snapshot cells with a faster flow are left out of the training loss (a reach about to
# fail the run's checks can carry a few runaway cells before it is dropped)
TRAIN_MAX_SPEED = 3.0


def forcing_at(case, t):
    """(upstream discharge, downstream stage) of the case's hourly tables at time t
    (linear between the hourly knots, as the library interpolates them)."""
    k = int(t // 3600)
    w = (t - 3600.0 * k) / 3600.0
    q = case.tables[cases.EDGE_LEFT][0]
    z = case.tables[cases.EDGE_RIGHT][0]
    return float(q[k] + w * (q[k + 1] - q[k])), float(z[k] + w * (z[k + 1] - z[k]))


def reach_crop(case, margin=6):
    """Rows 1..N and the columns of the channel band (every column holding a bed cell below
    the datum in any row, widened by `margin`): (i0, rows, j0, cols) in grid indices."""
    N, M = case.N, case.M
    h = case.fields["h"][1:N + 1, 1:M + 1] - case.params.NANGDAY
    cols = np.nonzero((h > 0.0).any(axis=0))[0]
    j0 = max(1, int(cols.min()) + 1 - margin)
    j1 = min(M, int(cols.max()) + 1 + margin)
    return 1, N, j0, j1 - j0 + 1


class Features:
    """The network's input of one reach on its crop, built on the device: bed depth,
    roughness, upstream Q, downstream stage and the along-flow and cross coordinates
    (normalised), padded to the first layer's 16 channels (BF16)."""

    def __init__(self, case, crop, device):
        import torch
        self.crop = crop
        self.dev = device
        i0, rows, j0, cols = crop
        N, M = case.N, case.M
        self.nangday = case.params.NANGDAY
        self.hbuf = torch.empty((N + 3, M + 3), dtype=torch.float64, device=device)
        n = torch.from_numpy(np.ascontiguousarray(case.fields["hsnham"][i0:i0 + rows, j0:j0 + cols]))
        self.static = torch.zeros((rows, cols, 3), dtype=torch.float32)
        self.static[..., 0] = ((n - N_REF) / 0.01).float()
        self.static[..., 1] = torch.linspace(0.0, 1.0, rows)[:, None]
        self.static[..., 2] = torch.linspace(0.0, 1.0, cols)[None, :]
        self.static = self.static.to(device)

    def build(self, sim, Q, stage, out=None):
        """(rows, cols, 16) BF16 on the device; written into `out` when given."""
        import torch
        i0, rows, j0, cols = self.crop
        sim.get_device("h", self.hbuf)
        h = (self.hbuf[i0:i0 + rows, j0:j0 + cols] - self.nangday) / H_REF
        x = out if out is not None else torch.empty((rows, cols, 16), dtype=torch.bfloat16, device=self.dev)
        x.zero_()
        x[..., 0] = h.to(torch.bfloat16)
        x[..., 1] = self.static[..., 0].to(torch.bfloat16)
        x[..., 2] = Q / Q_REF
        x[..., 3] = stage / STAGE_REF
        x[..., 4] = self.static[..., 1].to(torch.bfloat16)
        x[..., 5] = self.static[..., 2].to(torch.bfloat16)
        return x


class Targets:
    """The state on the crop as network targets, on the device: u, v, (z - stage) / DZ_REF
    and the wet mask."""

    def __init__(self, case, crop, device):
        import torch
        N, M = case.N, case.M
        self.crop = crop
        self.buf = {f: torch.empty((N + 3, M + 3), dtype=torch.float64, device=device) for f in ("u", "v", "z")}
        self.kh = torch.empty((N + 3, M + 3), dtype=torch.int32, device=device)

    def build(self, sim, stage, y_out, w_out):
        i0, rows, j0, cols = self.crop
        for f, b in self.buf.items():
            sim.get_device(f, b)
        sim.get_device("khouot", self.kh)
        sl = (slice(i0, i0 + rows), slice(j0, j0 + cols))
        u, v, z = self.buf["u"][sl], self.buf["v"][sl], self.buf["z"][sl]
        y_out[..., 0] = u
        y_out[..., 1] = v
        y_out[..., 2] = (z - stage) / DZ_REF
        ok = (self.kh[sl] == 0) & (u.abs() <= TRAIN_MAX_SPEED) & (v.abs() <= TRAIN_MAX_SPEED) & z.isfinite()
        y_out.nan_to_num_(0.0, 0.0, 0.0)
        w_out.copy_(ok.float())


def generate(seeds, snapshots, every=600, settle_h=2.0, device=0, crop=None, log=None):
    """Plain-solver quasi-steady snapshots of config-5-style reaches (config5_case with
    each seed, the bed not fed back): every reach on its own handle and stream, all queued
    together so that they step side by side on the device, spun up for `settle_h` hours,
    then a snapshot of every reach every `every` seconds, `snapshots` per reach.  A reach
    whose run fails (a device check, e.g. a line with more than 20 wet segments once its
    floodplain starts to flood in patches) keeps the snapshots it gave and drops out.
    Returns device tensors X (S, rows, cols, 16) BF16, Y (S, rows, cols, 3) FP32,
    W (S, rows, cols) FP32, the crop and the number of reaches that dropped out."""
    import torch
    from .lib import HydError
    dev = torch.device("cuda", device)
    days = (settle_h * 3600 + snapshots * every) / 86400.0 + 0.1
    cs = [cases.config5_case(seed=s, days=days, feedback=False) for s in seeds]
    crop = crop or reach_crop(cs[0])
    i0, rows, j0, cols = crop
    n = len(cs) * snapshots
    X = torch.empty((n, rows, cols, 16), dtype=torch.bfloat16, device=dev)
    Y = torch.empty((n, rows, cols, 3), dtype=torch.float32, device=dev)
    W = torch.empty((n, rows, cols), dtype=torch.float32, device=dev)
    sims = [Simulation.from_case(c, device=device) for c in cs]
    feats = [Features(c, crop, dev) for c in cs]
    tgts = [Targets(c, crop, dev) for c in cs]
    alive = list(range(len(cs)))

    def advance(nsteps):
        for m in alive:
            sims[m].step(nsteps, sync=False)
        ok = []
        for m in alive:
            try:
                sims[m].synchronize()
                ok.append(m)
            except HydError as e:
                if log:
                    log("reach %d dropped at t = %.0f s: %s" % (seeds[m], sims[m].t, e))
        alive[:] = ok

    advance(int(round(settle_h * 3600)))
    k = 0
    t0 = time.perf_counter()
    for s in range(snapshots):
        advance(every)
        for m in alive:
            Q, st = forcing_at(cs[m], sims[m].t)
            feats[m].build(sims[m], Q, st, out=X[k])
            tgts[m].build(sims[m], st, Y[k], W[k])
            k += 1
        if log and s % max(1, snapshots // 5) == 0:
            log("snapshot %d/%d, %d reaches, %.1f s" % (s + 1, snapshots, len(alive), time.perf_counter() - t0))
    for sim in sims:
        sim.close()
    return X[:k], Y[:k], W[:k], crop, len(cs) - len(alive)


def train(net, X, Y, W, iters=1500, batch=8, lr=2e-3, seed=0, log_every=0):
    """Minibatch Adam on device tensors (as from generate), the forward and backward passes
    on the tensor-core kernels.  Returns the loss of every iteration."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    losses = []
    for it in range(iters):
        idx = torch.randint(0, X.shape[0], (batch,), generator=g).to(X.device)
        xb = X.index_select(0, idx).contiguous()
        yb = Y.index_select(0, idx).contiguous()
        wb = W.index_select(0, idx).contiguous()
        pred, saved = net.forward(xb)
        loss, dy = net.loss_grad(pred, yb, wb)
        gw, gb = net.backward(saved, dy)
        net.adam(gw + gb, lr=lr * 0.5 * (1 + math.cos(math.pi * it / iters)))
        losses.append(loss)
        if log_every and it % log_every == 0:
            print("train %d loss %.4e" % (it, float(loss.item())))
    net.check_errors()
    return [float(l.item()) for l in losses]


class SurrogateJump:
    """The jump of the quasi-steady form: the network's predicted equilibrium for the
    current (bed, forcing) minus its prediction for the previous period's, as FP32
    increments of u, v, z on the crop."""

    def __init__(self, net, case, crop, clip=True):
        self.net = net
        self.crop = crop
        self.clip = clip
        self.feat = Features(case, crop, net.dev)
        self.prev = None

    def predict(self, sim, Q, stage):
        x = self.feat.build(sim, Q, stage)[None]
        y, _ = self.net.forward(x)
        y = y[0]
        return y[..., 0], y[..., 1], y[..., 2] * DZ_REF + stage

    def increments(self, sim, Q, stage):
        """(du, dv, dz) contiguous FP32 device tensors, or None on the first call; the
        prediction is kept as the next call's reference.  Each increment is clipped to
        JUMP_MAX (the jump's trust region; the gate judges the rest)."""
        cur = self.predict(sim, Q, stage)
        prev, self.prev = self.prev, cur
        if prev is None:
            return None
        return tuple((a - b).nan_to_num(0.0, 0.0, 0.0).clamp(-m if self.clip else -1e30, m if self.clip else 1e30)
                     .contiguous() for a, b, m in zip(cur, prev, JUMP_MAX))

    def reset(self, sim, Q, stage):
        """Take the prediction for (Q, stage) as the reference of the next increments."""
        self.prev = self.predict(sim, Q, stage)


class QuasiSteady:
    """The quasi-steady morphodynamic loop on one Simulation (see the module docstring).

    period(): advance one bed period; returns (accepted, plain steps taken).  The gate is
    read after each of the first `warm` - 1 warm steps from the `min_warm`-th on.  With a
    jump, a rejected jump is followed by one more try from the checkpoint without it
    (`retry`), before the period is stepped plainly.  Counters: accepted (of them
    jump_accepted with the jump), fallbacks, steps.

    native: the period's calls are made inside the library (hyd_quasi_steady_period: no
    host round trip between the warm steps) when the simulation offers it; the same calls
    in the same order as the loop written here, which runs otherwise."""

    def __init__(self, sim, case, warm=20, gate=1e-4, jump=None, min_warm=1, retry=True, native=True):
        self.sim = sim
        self.case = case
        self.warm = int(warm)
        self.min_warm = max(1, min(int(min_warm), self.warm - 1))
        self.gate = float(gate)
        self.jump = jump
        self.retry = retry
        self.native = bool(native) and hasattr(sim, "quasi_steady_period")
        self.period_s = float(case.params.bed_period)
        self.accepted = 0
        self.jump_accepted = 0
        self.fallbacks = 0
        self.steps = 0

    def _warm(self, t_end):
        """The warm steps from the current state; True (and the period's last step taken)
        once the gate passes; the residual reached otherwise."""
        sim = self.sim
        dT = sim.params.dT
        sim.set_time(t_end - self.warm * dT)
        sim.steady_residual(snapshot=True)
        r = (math.inf, math.inf)
        try:
            for k in range(1, self.warm):
                sim.step(1)
                r = sim.steady_residual(snapshot=True)
                if k >= self.min_warm and max(r) < self.gate and sim.mass_balance()["nonfinite"] == 0:
                    sim.set_time(t_end - dT)
                    sim.step(1)  # the period's last step: the bed update on the accepted state
                    self.steps += k + 1
                    return True, r
        except HydError:
            # a device check failed on the warm-started state (e.g. jumped levels flooded a
            # bank in patches and a line passed 20 wet segments): rejected like a state that
            # is not steady; the checkpoint holds the device status of before the jump
            r = (math.inf, math.inf)
        self.steps += self.warm - 1
        return False, r

    def period(self):
        sim = self.sim
        dT = sim.params.dT
        t_end = sim.t + self.period_s
        nper = int(round(self.period_s / dT))
        steps0 = self.steps
        inc = None
        if self.jump is not None:
            Q, st = forcing_at(self.case, t_end)
            inc = self.jump.increments(sim, Q, st)
        if self.native:
            i0 = j0 = 0
            if inc is not None:
                i0, _, j0, _ = self.jump.crop
            ok, jumped, n = sim.quasi_steady_period(self.period_s, self.warm, self.min_warm, self.gate, jump=inc,
                                                    i0=i0, j0=j0, retry=self.retry)
            self.steps += n
            self.accepted += 1 if ok else 0
            self.jump_accepted += 1 if jumped else 0
            self.fallbacks += 0 if ok else 1
            return ok, n
        sim.checkpoint()
        jumped = False
        if inc is not None:
            i0, _, j0, _ = self.jump.crop
            sim.add_levels(*inc, i0, j0)
            jumped = True
        ok, r = self._warm(t_end)
        if not ok and jumped and self.retry:
            sim.restore()  # the jump rejected: the previous state as the warm start
            ok, r = self._warm(t_end)
            jumped = False
        if ok:
            self.accepted += 1
            self.jump_accepted += 1 if jumped else 0
            return True, self.steps - steps0
        # not steady within the warm steps: back to the checkpoint, the period stepped plainly
        sim.restore()
        sim.step(nper)
        self.fallbacks += 1
        self.steps += nper
        return False, self.steps - steps0

    def run_until(self, t_stop):
        while self.sim.t + self.period_s <= t_stop + 1e-9:
            self.period()
