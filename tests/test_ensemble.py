"""Ensembles of independent reaches split across ranks (hydist.ensemble).

CPU: the cost partition, and two ranks over torch.distributed's gloo backend (processes
on 127.0.0.1) whose reaches step through the oracle: the gathered fields equal one
process stepping every reach, and the max-over-ranks reduction returns the largest
rank's value.  GPU: the same reaches stepped through the library on one device, each
handle on its own stream, equal bit for bit to handles stepped one at a time."""
import os
import socket

import numpy as np
import pytest

STEPS = 6


def _small_cases(n=5):
    from hydist import cases
    return cases.config3_cases(n=n, seed=11, nx_range=(24, 48), ny_range=(16, 32), hours=1.0, spinup_h=0.1)


class _OracleStepper:
    """The stepping interface of a library handle, on the CPU oracle (test only)."""

    def __init__(self, case):
        import oracle
        self.o = oracle.OracleSim(case, threads=1)
        self.o.init()

    def step(self, n=1, sync=True):
        self.o.step(n)

    def synchronize(self):
        pass

    def get(self, name):
        return self.o.get(name)

    def close(self):
        self.o.close()


def test_partition_covers_and_balances():
    from hydist import cases
    from hydist.ensemble import partition, reach_cost
    cs = cases.config3_cases(n=96)
    costs = [reach_cost(c) for c in cs]
    for world in (1, 2, 4, 8):
        parts = partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(cs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) <= sum(costs) / world + max(costs)
        assert parts == partition(costs, world)  # deterministic
    # a reach never splits: world larger than the ensemble leaves ranks empty
    assert sum(len(p) == 0 for p in partition(costs[:3], 5)) == 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    import datetime
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    for p in (root, os.path.join(root, "gpu-hydist_b200"), os.path.join(root, "oracle"), here):
        if p not in sys.path:
            sys.path.insert(0, p)
    import torch.distributed as dist
    from hydist.ensemble import Ensemble, checksum, max_over_ranks
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ens = Ensemble(_small_cases(), rank=rank, world=world, factory=_OracleStepper)
        ens.step(STEPS)
        got = ens.gather(("z", "u", "v"))
        mx = max_over_ranks(float(rank + 1) * 1.5)
        upd = max_over_ranks(ens.cell_updates(STEPS))
        if rank == 0:
            np.save(os.path.join(out_dir, "result.npy"),
                    {"owned": ens.owned, "sums": checksum(got), "max": mx, "upd": upd,
                     "fields": got}, allow_pickle=True)
        ens.close()
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_match_one_process(tmp_path, oracle_lib):
    import torch.multiprocessing as mp
    from hydist.ensemble import Ensemble, partition, reach_cost
    world, port = 2, _free_port()
    mp.spawn(_rank_main, args=(world, port, str(tmp_path)), nprocs=world, join=True)
    res = np.load(tmp_path / "result.npy", allow_pickle=True).item()
    cs = _small_cases()
    parts = partition([reach_cost(c) for c in cs], world)
    assert res["owned"] == parts[0]
    assert res["max"] == 3.0
    assert res["upd"] == max(STEPS * sum(reach_cost(cs[i]) for i in p) for p in parts)
    ref = Ensemble(cs, rank=0, world=1, factory=_OracleStepper)
    ref.step(STEPS)
    want = ref.fields(("z", "u", "v"))
    ref.close()
    assert sorted(res["fields"]) == list(range(len(cs)))
    for i, d in want.items():
        for f, a in d.items():
            assert np.array_equal(res["fields"][i][f], a), (i, f)
            assert np.isfinite(a).all()


@pytest.mark.gpu
def test_gpu_ensemble_streams_match_single_handles(oracle_lib):
    from helpers import REL_TOL, rel_linf
    from hydist.ensemble import Ensemble
    from hydist.lib import Simulation
    import oracle
    cs = _small_cases()
    ens = Ensemble(cs, rank=0, world=1)
    ens.step(STEPS)
    got = ens.fields(("z", "u", "v", "FS"))
    ens.close()
    for i, c in enumerate(cs):
        s = Simulation.from_case(c)
        s.step(STEPS)
        for f in ("z", "u", "v", "FS"):
            assert np.array_equal(got[i][f], s.get(f)), (i, f)
        s.close()
        o = oracle.OracleSim(c)
        o.init()
        o.step(STEPS)
        for f in ("z", "u", "v"):
            e = rel_linf(got[i][f], o.get(f))
            assert e <= REL_TOL, "reach %d %s rel L-inf %.3e" % (i, f, e)


@pytest.mark.gpu
def test_gpu_batch_realistic_reaches_vs_oracle(oracle_lib):
    """Batch members sized for throughput sweep every line of up to 288 rows by a warp,
    where a lone handle hands lines over 96 rows to the whole CTA: reaches of config 3's
    sizes (lines of a few hundred rows) against the oracle within 1e-9."""
    from helpers import REL_TOL, rel_linf
    from hydist import cases
    from hydist.ensemble import Ensemble
    import oracle
    cs = cases.config3_cases(n=3, seed=17, nx_range=(300, 500), ny_range=(150, 260), hours=1.0, spinup_h=0.1)
    ens = Ensemble(cs, rank=0, world=1)
    ens.step(20)
    got = ens.fields(("z", "u", "v", "FS"))
    ens.close()
    for i, c in enumerate(cs):
        o = oracle.OracleSim(c)
        o.init()
        o.step(20)
        for f in ("z", "u", "v", "FS"):
            e = rel_linf(got[i][f], o.get(f))
            assert e <= REL_TOL, "reach %d %s rel L-inf %.3e" % (i, f, e)


def test_tune_policy_shapes_on_cpu_fake():
    """The tuner's bookkeeping with a fake batch: each candidate sets every member's shape,
    the fastest (by the injected clock) is applied last and returned."""
    from hydist import tune

    class FakeSim:
        def __init__(self, N, M):
            self.N, self.M, self.shape = N, M, None

        def set_sweep_shape(self, ctas, wide):
            self.shape = (ctas, wide)

    class FakeBatch:
        def __init__(self):
            self.members = [FakeSim(100, 60), FakeSim(40, 300)]
            self.log = []

        def step(self, n, sync=True):
            self.log.append((n, self.members[0].shape))

    costs = {(16, 1): 3.0, (8, 1): 1.0, (16, 0): 2.0}
    b = FakeBatch()
    t = [0.0]

    def clock():
        # advance by the cost of the shape the last timed step ran with
        if b.log and b.log[-1][0] == 5:
            d = next(p for p in costs if b.members[0].shape == (max(1, -(-103 // p[0])), p[1]))
            t[0] += costs[d] * 5
        return t[0]

    best, times = tune.tune_batch(b, candidates=list(costs), steps=5, warm=1, clock=clock)
    assert best == (8, 1)
    assert b.members[0].shape == (13, 1) and b.members[1].shape == (38, 1)  # ceil(103/8), ceil(303/8)
    assert abs(times[(8, 1)] - 1.0) < 1e-12 and abs(times[(16, 1)] - 3.0) < 1e-12


@pytest.mark.gpu
def test_gpu_tuned_batch_vs_oracle(oracle_lib):
    """The online tuner steps the batch under several sweep shapes and keeps one; the
    reaches still match the oracle within 1e-9 after the tuning steps and more."""
    from helpers import REL_TOL, rel_linf
    from hydist import cases
    from hydist.ensemble import Ensemble
    import oracle
    cs = cases.config3_cases(n=3, seed=17, nx_range=(300, 500), ny_range=(150, 260), hours=1.0, spinup_h=0.1)
    ens = Ensemble(cs, rank=0, world=1)
    from hydist.tune import FUSED
    best, times = ens.tune(steps=3, candidates=((16, 1), (4, 0), FUSED))
    assert best in times and len(times) == 3
    n_tuned = 3 * (2 + 3)  # warm + timed steps per candidate
    ens.step(4)
    got = ens.fields(("z", "u", "v", "FS"))
    shapes = [m.sweep_shape() for m in ens.batch.members]
    print("tuner: %s" % ", ".join("%s %.3f ms" % (k, v * 1e3) for k, v in times.items()))
    ens.close()
    if best != FUSED:
        d, wide = best
        for c, sh in zip(cs, shapes):
            assert sh == (min(sh[0], -(-(max(c.N, c.M) + 3) // d)), wide)
    for i, c in enumerate(cs):
        o = oracle.OracleSim(c)
        o.init()
        o.step(n_tuned + 4)
        for f in ("z", "u", "v", "FS"):
            e = rel_linf(got[i][f], o.get(f))
            assert e <= REL_TOL, "reach %d %s rel L-inf %.3e" % (i, f, e)


def _batched_cases():
    """Six reaches of config 3's generator (uneven sizes), sediment from t = 60 s and the
    Exner update every 120 s, so that the batched steps cover every step variant."""
    from hydist import cases
    cs = cases.config3_cases(n=6, seed=23, nx_range=(128, 420), ny_range=(64, 220), hours=1.0, spinup_h=0.02)
    for c in cs:
        p = c.params.copy()
        p.sediment_start = 60.0
        p.bed_change_start = 120.0
        c.params = p
    return cs


@pytest.mark.gpu
def test_gpu_batched_launches_match_member_steps():
    """The batched form (every phase one launch for all members, one graph per batch step)
    against the same batch stepped member by member: every field, the mask and the segment
    tables bit for bit after 300 steps (sediment from 60 s, two Exner updates)."""
    from hydist.lib import Batch
    cs = _batched_cases()
    a = Batch(cs)
    a.set_fused(True)
    a.step(300)
    assert a.fused_steps() >= 290  # the first step and the first sediment step run per member
    b = Batch(cs)
    b.step(300)
    for k, (ma, mb) in enumerate(zip(a.members, b.members)):
        assert ma.t == mb.t == 300.0
        for f in ("z", "u", "v", "t_z", "t_u", "t_v", "FS", "dH", "H_moi", "Htdu", "Htdv", "khouot", "daui", "cuoii",
                  "moci", "dauj", "cuoij", "mocj"):
            assert np.array_equal(ma.get(f), mb.get(f), equal_nan=True), (k, f)
        ba, bb = ma.mass_budget(), mb.mass_budget()
        assert abs(ba["net_in"] - bb["net_in"]) <= 1e-9 * max(abs(bb["net_in"]), 1.0)
    a.close()
    b.close()


@pytest.mark.gpu
def test_gpu_batched_launches_vs_oracle(oracle_lib):
    """Two reaches of the batched form against the oracle within 1e-9."""
    from helpers import REL_TOL, rel_linf
    from hydist.lib import Batch
    import oracle
    cs = _batched_cases()[:2]
    a = Batch(cs)
    a.set_fused(True)
    a.step(150)
    for m, c in zip(a.members, cs):
        o = oracle.OracleSim(c)
        o.init()
        o.step(150)
        for f in ("z", "u", "v", "FS", "dH"):
            e = rel_linf(m.get(f), o.get(f))
            assert e <= REL_TOL, "%s rel L-inf %.3e" % (f, e)
    a.close()
