"""Multi-GPU replicas of the flow workflow: one process per GPU.

The Wilson flow of one configuration does not shard (one 48^4 lattice fits a
single B200), so N GPUs run N independent replicas.  The reference's
configuration loop (LGF/LGF.cpp:169, ``for i in [start..stop]``) is split
across ranks; each rank flows its own configurations through the drop-in on
its own device, and the only collective is a gather of the small
per-configuration status records.  There is no data-path collective.

Failure detection is host-side: a rank whose flow raises still takes part in
the gather (its records carry the error), and a rank that never arrives makes
the gather fail after the process group's timeout instead of hanging.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable


@dataclass
class ConfigRecord:
    config: int
    rank: int
    status: int          # 0 = flowed, < 0 = LGF_E* status
    error: str = ""


def assign(start: int, stop: int, world: int, cost: Callable[[int], float] | None = None) -> list[list[int]]:
    """Split configurations start..stop (inclusive, like FlowParameters) over
    world ranks.  Equal costs: round robin.  With a cost function: longest
    processing time first onto the least-loaded rank."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    cfgs = list(range(start, stop + 1))
    out: list[list[int]] = [[] for _ in range(world)]
    if cost is None:
        for k, c in enumerate(cfgs):
            out[k % world].append(c)
        return out
    load = [0.0] * world
    for c in sorted(cfgs, key=lambda c: -cost(c)):
        r = min(range(world), key=lambda i: (load[i], i))
        out[r].append(c)
        load[r] += cost(c)
    for o in out:
        o.sort()
    return out


def run_replicas(start: int, stop: int, flow_one: Callable[[int], int], rank: int = 0, world: int = 1,
                 group=None, cost: Callable[[int], float] | None = None) -> list[ConfigRecord]:
    """Flow this rank's share of start..stop with ``flow_one(config) -> status``
    and gather every rank's records (all ranks receive the full, sorted list).
    ``group`` is a torch.distributed process group (None with world == 1)."""
    mine = assign(start, stop, world, cost)[rank]
    recs: list[ConfigRecord] = []
    for c in mine:
        try:
            st = int(flow_one(c))
            recs.append(ConfigRecord(c, rank, st))
        except Exception as e:  # report, keep the collective schedule identical on every rank
            recs.append(ConfigRecord(c, rank, -1, f"{type(e).__name__}: {e}"))
    if world == 1:
        return sorted(recs, key=lambda r: r.config)
    import torch.distributed as dist
    gathered: list = [None] * world
    dist.all_gather_object(gathered, recs, group=group)
    allrecs = [r for part in gathered for r in part]
    return sorted(allrecs, key=lambda r: r.config)


def flow_saved_on_replicas(params, flowParams, rank: int = 0, world: int = 1, group=None) -> list[ConfigRecord]:
    """FlowSavedGaugeConfigurations over N GPUs: rank r flows its configurations
    on its local device (the caller sets LGF_DEVICE / the CUDA device)."""
    from .lgf import FlowParameters, FlowSavedGaugeConfigurations

    def one(c: int) -> int:
        fp = FlowParameters(c, c, flowParams.flowSteps, flowParams.epsilon, flowParams.measureEvery,
                            flowParams.dataFolder)
        return FlowSavedGaugeConfigurations(params, fp)

    return run_replicas(flowParams.start, flowParams.stop, one, rank, world, group)
