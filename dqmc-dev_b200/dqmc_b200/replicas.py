"""Independent Markov chains spread over ranks, one process per GPU.

The reference runs one chain per process and never exchanges data between
them (src/main_stack.c hands sim files to workers; each runs dqmc_wrapper on
its own).  Multi-GPU here is the same: a job of `n_total` chains is cut into
contiguous per-rank blocks, every rank advances its block on its own device,
and nothing crosses ranks during sweeps.  The only collectives are outside
the data path: the maximum of the ranks' device times (the job takes as long
as its slowest rank) and, at the end of a run, the sum of sign-weighted
accumulators over all chains.

Chain c of a job draws from the stream of the master seed jumped c times by
2^512 (rand_jump, as gen_1band_unified_hub.py:1163-1200 seeds a batch), so
the chains of a job are the same whatever the number of ranks.
"""
from __future__ import annotations

import numpy as np

from . import gen


def shard(n_total: int, rank: int, world: int) -> range:
    """Global chain indices of `rank`: contiguous blocks, sizes differing by
    at most one, the larger blocks first."""
    if world < 1 or not 0 <= rank < world or n_total < 0:
        raise ValueError(f"bad shard request: n_total={n_total} rank={rank} world={world}")
    base, extra = divmod(n_total, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def chain_streams(seed: int, chains: range) -> list[np.ndarray]:
    """Initial xorshift1024* states (16 words + index) of the given global
    chains: the master stream of `seed` jumped `c` times for chain c."""
    if len(chains) == 0:
        return []
    first = gen.chain_rngs(seed, chains.stop)
    return [first[c] for c in chains]


def max_over_ranks(x: float, world: int, device: str = "cpu") -> float:
    """Maximum of a per-rank scalar over all ranks (the job's device time)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(acc: np.ndarray, world: int, device: str = "cpu") -> np.ndarray:
    """Element-wise sum of accumulator arrays over all ranks (real or
    complex; the sign-weighted measurement sums of every chain)."""
    a = np.ascontiguousarray(acc)
    if world == 1:
        return a.copy()
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(a.view(np.float64) if np.iscomplexobj(a) else a.astype(np.float64))
    t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    out = t.cpu().numpy()
    return out.view(np.complex128) if np.iscomplexobj(a) else out
