"""Replica helpers for running the engine as one process per GPU.

The path shards without an exchange step (reads and pairs are independent units), so
the only cross-rank operations are a barrier around a timed region and the maximum of
the per-rank times, which is what a job's wall time is when ranks start together.
Works with any torch.distributed backend (NCCL on GPUs, gloo on CPU)."""


def world():
    import torch.distributed as dist
    return dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1


def barrier():
    import torch.distributed as dist
    if world() > 1:
        dist.barrier()


def max_over_ranks(value, device="cpu"):
    """Largest `value` over all ranks (every rank gets the result)."""
    if world() == 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard(n_units, rank, world_size):
    """Contiguous [begin, end) of `n_units` owned by `rank` (sizes differ by at most one)."""
    base, extra = divmod(n_units, world_size)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)
