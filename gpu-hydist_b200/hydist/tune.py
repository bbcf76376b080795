"""Online autotuner of the line sweeps' launch shape for a batch of reaches.

A batch's members run side by side on one GPU, so the best sweep shape depends on the
whole batch, not on one reach: how many persistent CTAs each member's sweeps take (a
member's CTAs hold whole SMs while they run) and whether warps sweep every line of up to
288 rows or only those of up to 96 (the rest by the whole CTA, one after another).  The
tuner steps the batch under each candidate policy for a few steps, times them, and keeps
the fastest.  The tuning steps are ordinary steps of the simulation (every shape gives
the same results up to rounding, within the parity tolerance), so nothing is saved or
restored.

    tune_batch(batch, candidates, steps) -> (best policy, {policy: seconds per step})

A policy (d, wide) steps every member on its own stream and graph and gives member k
ceil((max(N_k, M_k) + 3) / d) sweep CTAs (d lines per CTA: one per warp at d = 16) and
the warp-tier choice `wide`.  The policy FUSED steps the batch by batched launches
(hyd_batch_set_fused: every phase one launch for all members, the lines of all members
in one persistent sweep of one CTA per SM).  Which is faster depends on the batch: the
batched launches wait, phase by phase, for the member with the longest chain, while the
members' own streams overlap their phases.
"""
import math
import time

FUSED = ("fused",)
DEFAULT_CANDIDATES = ((16, 1), (8, 1), (32, 1), (16, 0), FUSED)


def apply_policy(batch, policy):
    """Set the batch's stepping from the policy: FUSED, or (d, wide) for every member."""
    if tuple(policy) == FUSED:
        batch.set_fused(True)
        return
    if hasattr(batch, "set_fused"):
        batch.set_fused(False)
    d, wide = policy
    for sim in batch.members:
        sim.set_sweep_shape(max(1, math.ceil((max(sim.N, sim.M) + 3) / d)), wide)


def tune_batch(batch, candidates=DEFAULT_CANDIDATES, steps=20, warm=2, clock=time.perf_counter):
    """Step the batch `warm` untimed steps (new graphs are captured then) and `steps` timed
    steps under each candidate policy; leave the batch on the fastest and return it with
    the measured seconds per step of every candidate.  Timed by the host clock around
    synchronised batch steps (the batch is device-bound: the host queues a member step in
    a few microseconds)."""
    if not candidates:
        raise ValueError("no candidate policies")
    times = {}
    for pol in candidates:
        apply_policy(batch, pol)
        batch.step(warm, sync=True)
        t0 = clock()
        batch.step(steps, sync=True)
        times[tuple(pol)] = (clock() - t0) / steps
    best = min(times, key=times.get)
    apply_policy(batch, best)
    return best, times
