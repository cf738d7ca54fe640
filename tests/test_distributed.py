"""Multi-rank host logic on CPU (gloo, world size 2): the ligand shards, the result gather of the sharded screen
and the max-over-ranks timing reduction. The docking call is replaced by a deterministic stand-in, so no GPU is
involved."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from adock_b200.distributed import shard_indices


class _Lig:
    def __init__(self, n):
        self.heavy = np.ones(n, bool)
        self.n = n


def _fake_dock(receptor, box, ligs, **kw):
    # one result per ligand that identifies it (its atom count) and the receptor it was docked against
    return [{"affinity": np.array([-float(l.n)]), "receptor": receptor["name"]} for l in ligs]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, sizes, q):
    import torch.distributed as dist
    from adock_b200.distributed import dock_screen_sharded, max_over_ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ligs = [_Lig(n) for n in sizes]
        out = dock_screen_sharded({"name": "rec"}, {}, ligs, dock_fn=_fake_dock)
        t = max_over_ranks(1.5 + rank)
        q.put((rank, None if out is None else [float(r["affinity"][0]) for r in out], t))
    finally:
        dist.destroy_process_group()


def test_shards_cover_every_ligand_once_and_balance_cost():
    rng = np.random.default_rng(0)
    costs = rng.integers(8, 81, 1001)
    for world in (1, 2, 3, 8):
        shards = [shard_indices(costs, r, world) for r in range(world)]
        allidx = sorted(i for s in shards for i in s)
        assert allidx == list(range(len(costs)))
        tot = [costs[s].sum() for s in shards]
        assert max(tot) - min(tot) <= costs.max()
        assert all(s == sorted(s) for s in shards)


def test_sharded_screen_gathers_in_order_on_two_gloo_ranks():
    sizes = [int(x) for x in np.random.default_rng(1).integers(8, 81, 37)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res = dict((r, (o, t)) for r, o, t in got)
    assert res[1][0] is None
    assert res[0][0] == [-float(n) for n in sizes]
    assert res[0][1] == res[1][1] == 2.5
