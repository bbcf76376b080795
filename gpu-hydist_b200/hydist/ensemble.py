"""Ensembles of independent reaches across GPUs (one process per GPU).

Reaches share nothing, so an ensemble is sharded by reach with no data-path collective:
every rank owns a subset, balanced by cost (cells), and steps its reaches on its own
GPU, one library handle per reach.  Each handle launches on its own CUDA stream, so the
steps of a rank's reaches run concurrently on its GPU.  The only collectives are host
bookkeeping: the maximum device time over ranks and, when asked, the reaches' results
gathered on rank 0.

    partition(costs, world)        -> per-rank lists of reach indices (largest first,
                                      each to the least loaded rank)
    Ensemble(cases, rank, world)   -> the rank's reaches (one library batch); .step(n),
                                      .cell_updates(n), .tune(steps) (hydist.tune)
    max_over_ranks(x)              -> max of a host float over the process group
"""
import heapq

import numpy as np


def reach_cost(case):
    """Work of one step of a reach: its interior cells."""
    return case.N * case.M


def partition(costs, world):
    """Longest-processing-time assignment: reaches in decreasing cost, each to the rank
    with the least total so far (ties to the lower rank).  Returns `world` lists of reach
    indices, each in increasing order; deterministic for given costs."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(v) for v in out]


class Ensemble:
    """The reaches of one rank.  By default they form one library batch on `device`
    (hyd_batch_*: one handle and stream per reach, stepped side by side); `factory(case)`
    instead builds one stepping object per reach with step(n, sync), synchronize(),
    get(name) and close()."""

    def __init__(self, cases, rank=0, world=1, device=0, factory=None):
        self.cases = list(cases)
        self.rank, self.world = rank, world
        self.owned = partition([reach_cost(c) for c in self.cases], world)[rank]
        self.sims = {}
        self.batch = None
        try:
            if factory is None:
                if self.owned:
                    from .lib import Batch
                    self.batch = Batch([self.cases[i] for i in self.owned], device=device)
                    self.sims = dict(zip(self.owned, self.batch.members))
            else:
                for i in self.owned:
                    self.sims[i] = factory(self.cases[i])
        except Exception:
            self.close()
            raise

    def tune(self, steps=20, candidates=None):
        """Pick the batch's sweep launch shape by timing (hydist.tune.tune_batch); the
        tuning steps advance the reaches like step().  Returns (policy, timings)."""
        if self.batch is None:
            return None, {}
        from .tune import DEFAULT_CANDIDATES, tune_batch
        return tune_batch(self.batch, candidates or DEFAULT_CANDIDATES, steps)

    def step(self, n=1, sync=True):
        """Advance every owned reach n steps (their launches queued on one stream per
        reach, so the reaches run side by side), then, with sync, wait for all."""
        if self.batch is not None:
            self.batch.step(n, sync)
            return
        for i in self.owned:
            self.sims[i].step(n, sync=False)
        if sync:
            self.synchronize()

    def synchronize(self):
        for i in self.owned:
            self.sims[i].synchronize()

    def cell_updates(self, n=1):
        """Cell-updates of n steps of the owned reaches."""
        return n * sum(reach_cost(self.cases[i]) for i in self.owned)

    def fields(self, names=("z", "u", "v")):
        """{reach index: {name: array}} of the owned reaches."""
        return {i: {f: self.sims[i].get(f) for f in names} for i in self.owned}

    def gather(self, names=("z", "u", "v")):
        """Every rank's fields on rank 0 (torch.distributed object gather; other ranks
        get None)."""
        import torch.distributed as dist
        mine = self.fields(names)
        if self.world == 1 or not dist.is_initialized():
            return mine
        parts = [None] * self.world if self.rank == 0 else None
        dist.gather_object(mine, parts, dst=0)
        if self.rank != 0:
            return None
        out = {}
        for p in parts:
            out.update(p)
        return out

    def close(self):
        if self.batch is not None:
            self.batch.close()
            self.batch = None
        else:
            for s in self.sims.values():
                s.close()
        self.sims = {}


def max_over_ranks(x):
    """Maximum of a host float over the default process group (x itself without one).
    A CPU tensor carries it, so the gloo and nccl backends both work (nccl moves it
    through the rank's current CUDA device)."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def checksum(fields):
    """Order-independent summary of gathered fields for comparisons: per reach and field
    the sum and the sum of squares."""
    return {i: {f: (float(np.sum(a)), float(np.sum(a * a))) for f, a in d.items()} for i, d in fields.items()}
