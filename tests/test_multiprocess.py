"""Multi-rank host logic on CPU (gloo, world size 2).

The GPU path shards as independent units with no data-path collective; on
the CPU side this checks that every rank derives the same LPT assignment,
that the shards are disjoint and complete, that per-rank results gathered
together equal a single-process run (each rank solves its systems with the
oracle), and the max-over-ranks timing reduction the bench uses.
"""
import os
import sys

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _systems():
    sys.path.insert(0, ROOT)
    from ktplace_b200 import synth, netlist
    import oracle
    out = []
    for k in range(5):
        raw = synth.generate(synth.spec_tiny(seed=40 + k, cells=80 + 30 * k, nets=90 + 33 * k))
        nl = netlist.flatten(raw)
        port = oracle.PortNetlist(nl)
        x, y = synth.seed_positions(raw, nl.num_movable, 7 + k)
        fx, fy = nl.floors()
        out.append((port.b2b_axis(True, x, fx, 0.0), x))
        out.append((port.b2b_axis(False, y, fy, 0.0), y))
    return out


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sys.path.insert(0, ROOT)
        import torch
        from ktplace_b200 import shard
        import oracle
        systems = _systems()
        costs = [s["val"].shape[0] + s["diag"].shape[0] for s, _ in systems]
        owned = shard.lpt_assign(costs, world)
        mine = owned[rank]
        results = {i: oracle.port_pcg_axis(systems[i][0], systems[i][1], 1e-6, 1000)["x"]
                   for i in mine}
        gathered = [None] * world
        dist.all_gather_object(gathered, (owned, results))
        t = torch.tensor([float(rank + 1)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if rank == 0:
            q.put((gathered, float(t.item())))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_sharding(port_built):
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered, tmax = q.get(timeout=100)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert tmax == 2.0
    owned0, _ = gathered[0]
    owned1, _ = gathered[1]
    assert owned0 == owned1  # same assignment on every rank
    all_units = sorted(owned0[0] + owned0[1])
    assert all_units == list(range(10))
    assert not set(owned0[0]) & set(owned0[1])
    sys.path.insert(0, ROOT)
    import oracle
    systems = _systems()
    merged = {}
    for _, res in gathered:
        merged.update(res)
    for i, (s, x0) in enumerate(systems):
        ref = oracle.port_pcg_axis(s, x0, 1e-6, 1000)["x"]
        assert np.array_equal(merged[i], ref)


def test_lpt_is_balanced():
    from ktplace_b200 import shard
    costs = [5, 9, 2, 7, 7, 3, 1, 8]
    owned = shard.lpt_assign(costs, 3)
    assert sorted(i for o in owned for i in o) == list(range(8))
    assert shard.makespan(costs, owned) <= 16
