"""Multi-GPU layout of the batched step: independent replicas.

Envs never exchange data inside a physics step, so N GPUs run N independent
sims (one process per GPU, weak scaling: every rank steps its own batch) and
the only collectives are host-side bookkeeping: a barrier around the timed
region and the max over ranks of the measured time.  No collective touches
the physics state.
"""
from __future__ import annotations

SEED_STATE = 1000
SEED_CTRL = 2000
RANK_STRIDE = 7919


def rank_seeds(rank: int) -> tuple[int, int]:
    """Seeds of the synthetic initial states and controls of one rank, so
    that replicas step different envs."""
    return SEED_STATE + RANK_STRIDE * rank, SEED_CTRL + RANK_STRIDE * rank


def shard(total: int, world: int, rank: int) -> tuple[int, int]:
    """(offset, count) of rank's contiguous slice of `total` envs when a fixed
    batch is split across ranks (strong scaling); slices differ by at most 1."""
    base, extra = divmod(total, world)
    count = base + (1 if rank < extra else 0)
    offset = rank * base + min(rank, extra)
    return offset, count


def reduce_over_ranks(x: float, op: str = "max", device=None) -> float:
    """Host scalar reduced over the process group (identity without one)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op={"max": dist.ReduceOp.MAX, "sum": dist.ReduceOp.SUM, "min": dist.ReduceOp.MIN}[op])
    return float(t.item())
