"""Multi-GPU plumbing for sharded counts: one process per GPU, each counting
an equal slice of the level-1 work queue (gat_executor_count_shard), then one
all-reduce of the raw signed sums (int64) and one of the device times (max).

The slice arithmetic mirrors the C ABI's: shard r of w covers units
[T*r//w, T*(r+1)//w) of T.  No data-path collective is needed: the shards are
independent and only their 8-byte totals are combined.
"""
from __future__ import annotations


def shard_bounds(total: int, rank: int, world: int) -> tuple[int, int]:
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad shard")
    return total * rank // world, total * (rank + 1) // world


def reduce_shards(raws: list[int], divisors: list[int], device_ms: float, group=None,
                  device=None) -> tuple[list[int], float]:
    """Sums each pattern's raw total over ranks, takes the max device time,
    and divides by the plan divisors.  Works on any torch.distributed backend
    (gloo on CPU, nccl on GPU); without an initialised process group it is the
    single-rank identity."""
    import torch
    import torch.distributed as dist

    raw = torch.tensor(raws, dtype=torch.int64, device=device)
    t = torch.tensor([device_ms], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(raw, group=group)
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    counts = []
    for r, d in zip(raw.tolist(), divisors):
        if d <= 0 or r % d != 0:
            raise ValueError(f"shard sum {r} is not a multiple of the divisor {d}")
        counts.append(r // d)
    return counts, float(t.item())
