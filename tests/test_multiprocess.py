"""Multi-rank host logic on CPU (gloo, world size 2).

The GPU path shards as independent units with no data-path collective. Each
rank here runs the product scheduling code (shard.ShardPlan, shard.run_share,
shard.gather_to_root) over a batch of netlist-shaped SPD systems; the solve
itself is a CPU stand-in (a sparse direct solve local to this test, since the
product solver needs a GPU), and the oracle's PCG only checks the assembled
result. Also checked: every rank derives the same LPT assignment, the shares
are disjoint and complete, and the max-over-ranks timing reduction the bench
uses.
"""
import os
import sys

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _units():
    """Five netlist-shaped units: per unit an x and a y system (B2B-like
    Laplacians of random 2-4 pin nets plus anchor weights), in the solver's
    CSR layout (off-diagonal row_ptr/col/val, separate diag)."""
    out = []
    for k in range(5):
        rng = np.random.default_rng(40 + k)
        n = 80 + 30 * k
        pair = []
        for axis in range(2):
            a = np.zeros((n, n))
            for _ in range(int(1.1 * n)):
                pins = rng.choice(n, size=rng.integers(2, 5), replace=False)
                w = 1.0 / (len(pins) - 1)
                for i in pins:
                    for j in pins:
                        if i != j:
                            a[i, j] -= w
                            a[i, i] += w
            anchor = rng.uniform(0.01, 0.2, n)
            diag = np.diag(a) + anchor
            off = a - np.diag(np.diag(a))
            rows, cols = np.nonzero(off)
            row_ptr = np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=n))]).astype(np.int64)
            rhs = anchor * rng.uniform(0, 1000, n)
            pair.append(dict(row_ptr=row_ptr, col=cols.astype(np.int32), val=off[rows, cols],
                             diag=diag, rhs=rhs, x0=rng.uniform(0, 1000, n)))
        out.append(pair)
    return out


def _direct_solve(s):
    """The CPU stand-in for the GPU batch solver (test only)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as sla
    n = s["diag"].shape[0]
    a = sp.csr_matrix((s["val"], s["col"], s["row_ptr"]), shape=(n, n)) + sp.diags(s["diag"])
    return sla.spsolve(a.tocsc(), s["rhs"])


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sys.path.insert(0, ROOT)
        import torch
        from ktplace_b200 import shard
        units = _units()
        sizes = [sum(s["diag"].shape[0] for s in pair) for pair in units]
        costs = [sum(s["val"].shape[0] + s["diag"].shape[0] for s in pair) for pair in units]
        plan = shard.ShardPlan(sizes, costs, world)
        out = np.full(plan.total, np.nan)
        solved = []

        def solve_units(us):
            solved.extend(us)
            return [np.concatenate([_direct_solve(s) for s in units[u]]) for u in us]

        mine = shard.run_share(plan, rank, solve_units, out)
        full = shard.gather_to_root(plan, rank, out)
        t = torch.tensor([float(rank + 1)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        owned = [None] * world
        dist.all_gather_object(owned, (plan.owned, mine, sorted(solved)))
        if rank == 0:
            q.put((owned, full, float(t.item())))
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
    owned, full, tmax = q.get(timeout=100)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert tmax == 2.0
    (plan0, mine0, solved0), (plan1, mine1, solved1) = owned
    assert plan0 == plan1  # same assignment on every rank
    assert sorted(mine0) == solved0 == sorted(plan0[0])
    assert sorted(mine1) == solved1 == sorted(plan0[1])
    assert sorted(mine0 + mine1) == list(range(5)) and not set(mine0) & set(mine1)
    # checker: the oracle's PCG on every system of the assembled buffer
    sys.path.insert(0, ROOT)
    import oracle
    assert not np.isnan(full).any()
    o = 0
    for pair in _units():
        for s in pair:
            n = s["diag"].shape[0]
            ref = oracle.port_pcg_axis(s, s["x0"], 1e-10, 10000)["x"]
            got = full[o:o + n]
            assert np.linalg.norm(got - ref) <= 1e-7 * np.linalg.norm(ref)
            o += n
    assert o == full.shape[0]


def test_share_layout_errors():
    from ktplace_b200 import shard
    plan = shard.ShardPlan([3, 4], world=2)
    out = np.zeros(plan.total)
    with pytest.raises(RuntimeError):
        shard.run_share(plan, 0, lambda us: [np.zeros(9) for _ in us], out)
    with pytest.raises(RuntimeError):
        shard.run_share(plan, 1, lambda us: [], out)
    with pytest.raises(ValueError):
        plan.share(2)
    empty = shard.ShardPlan([5], world=3)
    assert shard.run_share(empty, 2, lambda us: 1 / 0, np.zeros(5)) == []


def test_lpt_is_balanced():
    from ktplace_b200 import shard
    costs = [5, 9, 2, 7, 7, 3, 1, 8]
    owned = shard.lpt_assign(costs, 3)
    assert sorted(i for o in owned for i in o) == list(range(8))
    assert shard.makespan(costs, owned) <= 16
