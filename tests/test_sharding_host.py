"""Spreading batches and served diagrams over several GPUs (replicas, no
collective), host side: the least-loaded partition, the per-rank split of a
multi-process job (gloo, world size 2), and the routing of a server pool,
driven with stand-in servers."""
import os
import socket

import numpy as np
import pytest

from integer_delauney_b200.sharding import ServerPool, partition, rank_shard


def test_partition_covers_every_item_once_and_balances():
    rng = np.random.default_rng(3)
    w = (rng.lognormal(10, 1.2, 517)).tolist()
    for n in (1, 2, 3, 8):
        parts = partition(w, n)
        assert len(parts) == n
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(w)))
        assert all(p == sorted(p) for p in parts)
        loads = [sum(w[i] for i in p) for p in parts]
        # greedy least-loaded: no part exceeds the lightest by more than one item
        assert max(loads) - min(loads) <= max(w) + 1e-6
    assert partition(w, 4) == partition(list(w), 4)         # deterministic
    assert partition([], 3) == [[], [], []]
    assert partition([5.0, 5.0, 5.0], 2) == [[0, 2], [1]]   # ties: lower index, lower part first
    with pytest.raises(ValueError):
        partition(w, 0)
    with pytest.raises(ValueError):
        rank_shard(w, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from integer_delauney_b200.workloads import batched_images
    imgs = batched_images(count=64, seed=5)
    mine = rank_shard([(w + 33) * (h + 33) for w, h, _ in imgs], rank, world)
    got = [None] * world
    dist.all_gather_object(got, mine)           # for the check only: the split needs no exchange
    out[rank] = got
    dist.destroy_process_group()


def test_ranks_take_disjoint_shares_that_cover_the_batch():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    a, b = out[0]
    assert out[1] == [a, b]
    assert not set(a) & set(b) and sorted(a + b) == list(range(64))


class _FakeTicket:
    def __init__(self, did):
        self.diagram_id = did


class _FakeServer:
    def __init__(self, dev):
        self.dev = dev
        self.new, self.ins = [], []
        self.live = set()
        self.stats = {"groups": 1, "evicted": dev}
        self.closed = False

    def submit_new(self, W, H, seeds, fetch=False, arrival=None):
        did = 100 * self.dev + len(self.new)
        self.new.append((W, H))
        self.live.add(did)
        return _FakeTicket(did)

    def submit_insert(self, did, seeds, fetch=False, arrival=None):
        if did not in self.live:
            raise KeyError(did)
        self.ins.append((did, len(seeds)))
        return _FakeTicket(did)

    def resident(self):
        return sorted(self.live)

    def drain(self):
        pass

    def close(self):
        self.closed = True


def test_pool_routes_new_to_least_loaded_and_inserts_home():
    fakes = {}
    pool = ServerPool(devices=[0, 1, 2], border_padding=0, make_server=lambda d: fakes.setdefault(d, _FakeServer(d)))
    sizes = [(1000, 1000), (100, 100), (100, 100), (500, 500), (10, 10)]
    t = [pool.submit_new(W, H, [(0, 0)]) for W, H in sizes]
    # 1e6 -> dev0; 1e4 -> dev1; 1e4 -> dev2; 2.5e5 -> dev1 (tie with dev2 broken low); 100 -> dev2
    assert [x.device for x in t] == [0, 1, 2, 1, 2]
    assert [x.diagram_id for x in t] == [0, 1, 2, 3, 4]
    assert pool.loads() == [10 ** 6, 10 ** 4 + 250000, 10 ** 4 + 100]
    ins = pool.submit_insert(3, [(1, 1)] * 7)
    assert ins.device == 1 and fakes[1].ins == [(101, 7)]
    assert pool.loads()[1] == 10 ** 4 + 250000 + 7
    with pytest.raises(KeyError):
        pool.submit_insert(99, [(1, 1)])
    fakes[1].live.discard(101)                  # the device server evicted it
    with pytest.raises(KeyError):
        pool.submit_insert(3, [(1, 1)])
    assert pool.resident() == [0, 1, 2, 4]
    assert pool.stats == {"groups": 3, "evicted": 3}
    pool.close()
    assert all(f.closed for f in fakes.values())
