"""Multi-GPU replica routing on CPU: world-size-2 gloo process groups (no GPU).
The flow itself is replaced by a host-side fake; what is tested is the split
of the configuration loop, the gather, and host-side failure reporting."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from msc_project_b200.replicas import ConfigRecord, assign, run_replicas


def test_assign_covers_every_config_once():
    for world in (1, 2, 3, 8):
        parts = assign(3, 20, world)
        flat = sorted(c for p in parts for c in p)
        assert flat == list(range(3, 21))
        assert max(map(len, parts)) - min(map(len, parts)) <= 1


def test_assign_balances_costs():
    cost = {c: (10.0 if c < 2 else 1.0) for c in range(10)}
    parts = assign(0, 9, 2, cost=lambda c: cost[c])
    loads = [sum(cost[c] for c in p) for p in parts]
    assert abs(loads[0] - loads[1]) <= 2.0
    assert sorted(c for p in parts for c in p) == list(range(10))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, fail_cfg, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))

    def flow_one(c):
        if c == fail_cfg:
            raise RuntimeError("input file unreadable")
        return 0

    recs = run_replicas(0, 6, flow_one, rank, world)
    q.put((rank, [(r.config, r.rank, r.status, r.error) for r in recs]))
    dist.destroy_process_group()


@pytest.mark.parametrize("fail_cfg", [None, 3])
def test_two_ranks_gather_all_records(fail_cfg):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, fail_cfg, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0] == out[1]  # every rank sees the same full list
    recs = out[0]
    assert [c for c, *_ in recs] == list(range(7))
    assert {c for c, r, *_ in recs if r == 0} == {0, 2, 4, 6}
    for c, r, st, err in recs:
        if c == fail_cfg:
            assert st < 0 and "unreadable" in err
        else:
            assert st == 0


def _silent_worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    if rank == 1:
        q.put((rank, "left"))  # rank 1 leaves between steps, before the gather
        return
    try:
        run_replicas(0, 3, lambda c: 0, rank, world)
        q.put((rank, "no error"))
    except Exception as e:
        q.put((rank, type(e).__name__))


def test_missing_rank_is_detected_by_timeout():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_silent_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    assert out[1] == "left"
    assert out[0] != "no error"  # the gather on rank 0 ended with an error, it did not hang
