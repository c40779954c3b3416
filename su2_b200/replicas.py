"""Replica plumbing for one process per GPU.

The Monte-Carlo path does not shard a single lattice here: every rank advances its own
chains (independent Markov chains, or its share of an ensemble) and nothing crosses ranks
inside a trajectory.  What crosses ranks is bookkeeping: which chains a rank owns, a seed per
rank, the slowest rank's device time and the gathered per-chain results.  These helpers use
torch.distributed only for that; they work with the gloo backend on the CPU and with NCCL on
the GPUs (tensors then live on the current CUDA device).
"""
from __future__ import annotations

from typing import Any, Sequence


def chain_sites(chain: dict) -> int:
    """Lattice sites of one chain."""
    Lx, Ly, Lz, Lt = chain["dims"]
    return Lx * Ly * Lz * Lt


def chain_cost(chain: dict) -> int:
    """Work of one chain per trajectory, in staple evaluations: V d links with 2(d-1) staples
    each (get_staples.hh:26-80).  The force dominates a trajectory and its cost per site grows
    with d(d-1): a d = 4 site carries four links of six staples, a d = 3 site three links of
    four, so counting sites alone would weigh a d = 3 chain twice as heavy as it is."""
    d = int(chain["ndims"])
    return chain_sites(chain) * d * 2 * (d - 1)


def partition_chains(chains: Sequence[dict], world_size: int, rank: int) -> list[int]:
    """Indices of the chains that rank owns.

    Longest-processing-time assignment: chains sorted by cost (largest first, index as the
    tie-break) go one by one to the rank with the least work so far (lowest rank on ties).
    Deterministic, so every rank computes the same partition without communication; every
    chain lands on exactly one rank.
    """
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError(f"bad rank {rank} of {world_size}")
    load = [0] * world_size
    owner = [0] * len(chains)
    for i in sorted(range(len(chains)), key=lambda k: (-chain_cost(chains[k]), k)):
        r = min(range(world_size), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += chain_cost(chains[i])
    return [i for i in range(len(chains)) if owner[i] == rank]


def replica_seed(base: int, rank: int) -> int:
    """Seed of the chain of one rank: distinct Philox keys per rank."""
    return (int(base) + 1000003 * int(rank)) & 0xFFFFFFFFFFFF


def _device():
    import torch
    import torch.distributed as dist
    if dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(x: float) -> float:
    """The largest value over all ranks (device time of the slowest rank)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_chain_results(n_chains: int, owned: Sequence[int], results: Sequence[Any]) -> list:
    """Per-chain results of all ranks, in chain order (every rank receives the full list).

    ``owned`` are the chain indices of this rank and ``results`` their results (any picklable
    objects), in the same order.
    """
    import torch.distributed as dist
    if len(owned) != len(results):
        raise ValueError("one result per owned chain")
    mine = list(zip(owned, results))
    if not (dist.is_available() and dist.is_initialized()):
        parts = [mine]
    else:
        parts = [None] * dist.get_world_size()
        dist.all_gather_object(parts, mine)
    out: list = [None] * n_chains
    for part in parts:
        for i, r in part:
            if out[i] is not None:
                raise RuntimeError(f"chain {i} reported by two ranks")
            out[i] = r
    missing = [i for i, r in enumerate(out) if r is None]
    if missing:
        raise RuntimeError(f"chains without a result: {missing}")
    return out
