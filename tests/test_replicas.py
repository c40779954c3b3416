"""Replica bookkeeping across ranks: world_size-2 process groups on the CPU (gloo)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from su2_b200 import replicas


def ensemble(n=64, seed=5):
    """Seeded ensemble of SU(2) chains: d=4 with L in 8..24, d=3 with L in 16..48 (even)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        if rng.random() < 0.5:
            L = int(rng.integers(4, 13)) * 2
            out.append(dict(dims=(L, L, L, L), ndims=4, beta=float(rng.uniform(2.0, 2.6)),
                            seed=1000 + i))
        else:
            L = int(rng.integers(8, 25)) * 2
            out.append(dict(dims=(L, L, 1, L), ndims=3, beta=float(rng.uniform(2.0, 2.6)),
                            seed=1000 + i))
    return out


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_partition_covers_every_chain_once_and_balances(world):
    chains = ensemble()
    parts = [replicas.partition_chains(chains, world, r) for r in range(world)]
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(chains)))
    loads = [sum(replicas.chain_cost(chains[i]) for i in p) for p in parts]
    biggest = max(replicas.chain_cost(c) for c in chains)
    assert max(loads) - min(loads) <= biggest


def test_cost_counts_staple_work_not_sites():
    """A d = 4 site carries 4 links of 6 staples, a d = 3 site 3 links of 4."""
    d4 = dict(dims=(8, 8, 8, 8), ndims=4)
    d3 = dict(dims=(16, 16, 1, 16), ndims=3)
    assert replicas.chain_sites(d4) == 8 ** 4 and replicas.chain_sites(d3) == 16 ** 3
    assert replicas.chain_cost(d4) == 8 ** 4 * 4 * 6
    assert replicas.chain_cost(d3) == 16 ** 3 * 3 * 4
    # equal site counts, twice the work per site in d = 4
    assert replicas.chain_cost(d4) == 2 * replicas.chain_cost(d3)


def _mixed_worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        chains = ensemble(64, seed=11)
        owned = replicas.partition_chains(chains, world, rank)
        load = sum(replicas.chain_cost(chains[i]) for i in owned)
        q.put((rank, owned, load, replicas.max_over_ranks(load),
               replicas.sum_over_ranks(load)))
    finally:
        dist.destroy_process_group()


def test_two_ranks_balance_a_mixed_d3_d4_ensemble():
    """Each gloo rank partitions the same mixed ensemble on its own; the two shares cover
    every chain once, and their staple work differs by at most one chain's cost."""
    chains = ensemble(64, seed=11)
    assert {c["ndims"] for c in chains} == {3, 4}
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_mixed_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    owned = [o for _, o, _, _, _ in out]
    assert sorted(owned[0] + owned[1]) == list(range(64))
    loads = [ld for _, _, ld, _, _ in out]
    total = sum(replicas.chain_cost(c) for c in chains)
    assert out[0][4] == total and out[0][3] == max(loads)
    biggest = max(replicas.chain_cost(c) for c in chains)
    assert abs(loads[0] - loads[1]) <= biggest


def test_partition_rejects_bad_rank():
    with pytest.raises(ValueError):
        replicas.partition_chains(ensemble(4), 2, 2)


def test_replica_seeds_distinct():
    assert len({replicas.replica_seed(20240, r) for r in range(64)}) == 64


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        chains = ensemble(16)
        owned = replicas.partition_chains(chains, world, rank)
        results = [{"chain": i, "rank": rank, "plaq": 0.5 + i} for i in owned]
        allres = replicas.gather_chain_results(len(chains), owned, results)
        t = replicas.max_over_ranks(1.0 + rank)
        s = replicas.sum_over_ranks(len(owned))
        q.put((rank, [r["chain"] for r in allres], [r["rank"] for r in allres], t, s))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gather_and_reduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    chains = ensemble(16)
    for rank, order, owners, t, s in out:
        assert order == list(range(16))
        for i, o in enumerate(owners):
            assert i in replicas.partition_chains(chains, 2, o)
        assert t == 2.0
        assert s == 16
