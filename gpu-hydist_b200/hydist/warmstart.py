"""Surrogate-assisted quasi-steady hydraulics: the learned part in use.

The plain ADI reaches the equilibrium flow of a new forcing or a new bed by stepping
through the transient, thousands of steps.  The surrogate (hydist.surrogate) predicts
that equilibrium (u, v, z) from the bed, the roughness, the upstream discharge and the
downstream stage; the prediction replaces the state ("the jump"), the plain ADI then
runs a few warm-start steps, and the state is kept only if its steady residual, the
relative change of the velocity field per step, has fallen below the gate by then.
Otherwise the run falls back to the last accepted state and steps plainly.  No
reference counterpart (the reference has no learned part).

  reach_case(seed)          a seeded meandering reach (192 x 96 cells, 5 m) for data
  generate(...)             quasi-steady snapshots from the plain solver (a hyd_batch of
                            reaches, each taken through a sequence of forcings)
  train(net, data, ...)     minibatch training on the tensor-core kernels
  GatedWarmStart            the jump, the warm-start steps, the residual gate, fallback
"""
import math

import numpy as np

from . import cases
from . import surrogate as S
from .lib import Batch, Simulation

REACH_N, REACH_M, REACH_DX = 192, 96, 5.0
FEATURES = 6  # bed, roughness, upstream Q, downstream stage, along-flow and cross coordinates
Q_REF, H_REF, N_REF, DZ_REF = 100.0, 4.0, 0.025, 0.1


def reach_case(seed, Q=60.0, hours=40.0):
    """A small meandering reach of the config-2 generator (channel 60 m wide and 4 m deep,
    floodplain at +1.5 m, bed noise, lognormal roughness): discharge in on the left edge,
    stage on the right, hydraulics only, the discharge ramped up over the first 15 min."""
    rng = np.random.default_rng(seed)
    amp = rng.uniform(0.0, 80.0)
    wavelength = rng.uniform(500.0, 1200.0)
    c = cases.meander_case(N=REACH_N, M=REACH_M, dX=REACH_DX, dT=1.0, hours=hours, seed=seed, amp=amp,
                           wavelength=wavelength, width=60.0, depth=4.0, floodplain=1.5, noise_sigma=0.15,
                           noise_len=25.0, manning=0.025, manning_spread=0.10, Q0=Q, Q1=Q, tide_amp=0.0,
                           spinup_h=0.25, sediment_start=1e12, bed_change_start=1e12, end_cells=8,
                           name="reach%d" % seed)
    c.notes.update({"amp": amp, "wavelength": wavelength})
    return c


def forcing_tables(case, Q, stage):
    """Boundary tables holding discharge Q and stage `stage` at every hour."""
    tabs = [np.array(t, dtype=np.float64, copy=True) for t in case.tables]
    tabs[cases.EDGE_LEFT][:] = Q
    tabs[cases.EDGE_RIGHT][:] = stage
    return tabs, [np.array(t, dtype=np.float64, copy=True) for t in case.cc]


def features(case, Q, stage):
    """The network input of a reach under a forcing: (N, M, FEATURES) FP32, channels bed,
    roughness, Q, stage, x, y (normalised); the network pads them to 16 with zeros."""
    N, M = case.N, case.M
    x = np.zeros((N, M, FEATURES), dtype=np.float32)
    x[..., 0] = case.fields["h"][1:N + 1, 1:M + 1] / H_REF
    x[..., 1] = (case.fields["hsnham"][1:N + 1, 1:M + 1] - N_REF) / 0.01
    x[..., 2] = Q / Q_REF
    x[..., 3] = stage
    x[..., 4] = np.linspace(0.0, 1.0, N, dtype=np.float32)[:, None]
    x[..., 5] = np.linspace(0.0, 1.0, M, dtype=np.float32)[None, :]
    return x


def targets(sim, stage):
    """The state as network targets: u, v, (z - stage) / DZ_REF on the interior, and the wet
    mask."""
    N, M = sim.N, sim.M
    u = sim.get("u")[1:N + 1, 1:M + 1]
    v = sim.get("v")[1:N + 1, 1:M + 1]
    z = sim.get("z")[1:N + 1, 1:M + 1]
    wet = (sim.get("khouot")[1:N + 1, 1:M + 1] == 0).astype(np.float32)
    y = np.stack([u, v, (z - stage) / DZ_REF], axis=-1).astype(np.float32)
    return y, wet


def steady_residual(u0, v0, u1, v1, wet):
    """Relative change of the velocity field over one step on the wet cells."""
    du = (u1 - u0)[wet > 0]
    dv = (v1 - v0)[wet > 0]
    num = math.sqrt(float((du * du).sum() + (dv * dv).sum()))
    den = math.sqrt(float((u1[wet > 0] ** 2).sum() + (v1[wet > 0] ** 2).sum()))
    return num / max(den, 1e-30)


def forcing_levels(rng, n):
    """n (Q, stage) pairs: discharge 30-150 m3/s, stage -0.5..0.5 m."""
    return [(float(rng.uniform(30.0, 150.0)), float(rng.uniform(-0.5, 0.5))) for _ in range(n)]


def generate(seeds, levels_per_reach, settle=1500, device=0, seed=11):
    """Quasi-steady snapshots: every reach of `seeds` (run side by side as a batch) is taken
    through `levels_per_reach` forcings, each held for `settle` steps, and its state taken
    at the end of each.  Returns X (S, N, M, 16), Y (S, N, M, 3), W (S, N, M) and the
    residual at each snapshot."""
    rng = np.random.default_rng(seed)
    cs = [reach_case(s) for s in seeds]
    batch = Batch(cs, device=device)
    batch.set_fused(True)  # the reaches share sizes and schedule: batched launches
    batch.step(int(round(0.25 * 3600)) + 300)  # the ramp, then a settling margin
    X, Y, W, R = [], [], [], []
    plans = [forcing_levels(rng, levels_per_reach) for _ in cs]
    for k in range(levels_per_reach):
        for sim, c, plan in zip(batch.members, cs, plans):
            tabs, cc = forcing_tables(c, *plan[k])
            sim.update_boundary(tabs, cc)
        batch.step(settle - 1)
        prev = [(m.get("u"), m.get("v")) for m in batch.members]
        batch.step(1)
        for sim, c, plan, (u0, v0) in zip(batch.members, cs, plans, prev):
            Q, stage = plan[k]
            y, wet = targets(sim, stage)
            X.append(features(c, Q, stage))
            Y.append(y)
            W.append(wet)
            N, M = c.N, c.M
            R.append(steady_residual(u0[1:N + 1, 1:M + 1], v0[1:N + 1, 1:M + 1], y[..., 0], y[..., 1], wet))
    batch.close()
    return np.stack(X), np.stack(Y), np.stack(W), np.array(R)


def train(net, X, Y, W, iters=1500, batch=16, lr=2e-3, seed=0, log_every=0):
    """Minibatch Adam on (X, Y, W) (numpy, as from generate), the forward and backward
    passes on the tensor-core kernels.  Returns the loss of every iteration."""
    import torch
    rng = np.random.default_rng(seed)
    Xd = pad_input(torch.from_numpy(X).to(net.dev))
    Yd = torch.from_numpy(Y).to(net.dev)
    Wd = torch.from_numpy(W).to(net.dev)
    losses = []
    for it in range(iters):
        idx = torch.from_numpy(rng.integers(0, X.shape[0], size=batch)).to(net.dev)
        xb = Xd.index_select(0, idx).contiguous()
        yb = Yd.index_select(0, idx).contiguous()
        wb = Wd.index_select(0, idx).contiguous()
        pred, saved = net.forward(xb)
        loss, dy = net.loss_grad(pred, yb, wb)
        gw, gb = net.backward(saved, dy)
        # cosine decay of the step size
        net.adam(gw + gb, lr=lr * 0.5 * (1 + math.cos(math.pi * it / iters)))
        losses.append(loss)
        if log_every and it % log_every == 0:
            print("train %d loss %.4e" % (it, float(loss.item())))
    net.check_errors()
    return [float(l.item()) for l in losses]


def pad_input(x):
    """FP32 (..., FEATURES) -> BF16 (..., 16), the first layer's padded input channels."""
    import torch
    out = torch.zeros(x.shape[:-1] + (16,), dtype=torch.bfloat16, device=x.device)
    out[..., :x.shape[-1]] = x.to(torch.bfloat16)
    return out


def predict(net, case, Q, stage):
    """The network's equilibrium (u, v, z) of `case` under (Q, stage), interior N x M."""
    import torch
    x = pad_input(torch.from_numpy(features(case, Q, stage)[None]).to(net.dev))
    y, _ = net.forward(x)
    y = y[0].float().cpu().numpy()
    return y[..., 0], y[..., 1], y[..., 2] * DZ_REF + stage


class GatedWarmStart:
    """The surrogate's jump with the plain ADI as the judge.

    apply(sim, case, Q, stage): checkpoint the state, set (u, v, z) to the network's
    equilibrium on the wet cells (the depths and face depths re-derived), run up to
    `gate_steps` plain ADI steps, and keep the result if the steady residual has fallen
    below `gate` by then; otherwise restore the checkpoint (the run continues from the
    last accepted state with plain stepping).  Returns (accepted, residual, steps run)."""

    def __init__(self, net, gate=1e-4, gate_steps=20):
        self.net = net
        self.gate = gate
        self.gate_steps = gate_steps

    def jump(self, sim, case, Q, stage):
        N, M = sim.N, sim.M
        up, vp, zp = predict(self.net, case, Q, stage)
        wet = sim.get("khouot")[1:N + 1, 1:M + 1] == 0
        h = sim.get("h")
        fields = {}
        for name, pred in (("u", up), ("v", vp), ("z", zp)):
            a = sim.get(name)
            inner = a[1:N + 1, 1:M + 1]
            inner[wet] = pred[wet]
            fields[name] = a
        z = fields["z"]
        # the state update's derived fields for the new levels (update_h_moi, Htuongdoi)
        htaiz = sim.get("htaiz")
        Hn = sim.get("H_moi")
        kh = sim.get("khouot")
        inner = (kh == 0)[1:N + 1, 1:M + 1]
        Hn[1:N + 1, 1:M + 1][inner] = (htaiz + z)[1:N + 1, 1:M + 1][inner]
        Htdu, Htdv = sim.get("Htdu"), sim.get("Htdv")
        Htdu[1:N + 1, 1:M + 1] = (h[1:N + 1, 0:M] + h[1:N + 1, 1:M + 1] + z[2:N + 2, 1:M + 1] + z[1:N + 1, 1:M + 1]) * 0.5
        Htdv[1:N + 1, 1:M + 1] = (h[0:N, 1:M + 1] + h[1:N + 1, 1:M + 1] + z[1:N + 1, 2:M + 2] + z[1:N + 1, 1:M + 1]) * 0.5
        for name, a in (("u", fields["u"]), ("v", fields["v"]), ("z", z), ("t_u", fields["u"]),
                        ("t_v", fields["v"]), ("t_z", z), ("H_moi", Hn), ("Htdu", Htdu), ("Htdv", Htdv)):
            sim.set(name, a)

    def apply(self, sim, case, Q, stage):
        N, M = sim.N, sim.M
        saved = sim.get_state()
        self.jump(sim, case, Q, stage)
        r = float("inf")
        wet = (sim.get("khouot")[1:N + 1, 1:M + 1] == 0).astype(np.float32)
        u0, v0 = sim.get("u")[1:N + 1, 1:M + 1], sim.get("v")[1:N + 1, 1:M + 1]
        steps = 0
        for _ in range(self.gate_steps):
            sim.step(1)
            steps += 1
            u1, v1 = sim.get("u")[1:N + 1, 1:M + 1], sim.get("v")[1:N + 1, 1:M + 1]
            r = steady_residual(u0, v0, u1, v1, wet)
            u0, v0 = u1, v1
            if r < self.gate:
                break
        if r < self.gate:
            return True, r, steps
        sim.set_state(saved)
        return False, r, steps


def steps_to_steady(sim, tau, cap, N, M):
    """Plain steps until the steady residual falls below tau (at most cap); the count."""
    wet = (sim.get("khouot")[1:N + 1, 1:M + 1] == 0).astype(np.float32)
    u0, v0 = sim.get("u")[1:N + 1, 1:M + 1], sim.get("v")[1:N + 1, 1:M + 1]
    for k in range(1, cap + 1):
        sim.step(1)
        u1, v1 = sim.get("u")[1:N + 1, 1:M + 1], sim.get("v")[1:N + 1, 1:M + 1]
        if steady_residual(u0, v0, u1, v1, wet) < tau:
            return k
        u0, v0 = u1, v1
    return cap
