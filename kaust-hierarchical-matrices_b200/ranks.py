"""Multi-process plumbing of the benchmark (one process per GPU).

The path shards by cloud: every rank builds and multiplies its own independent
cloud, so the only cross-rank steps are the timing reduction (the slowest
rank sets the step time) and the sum of the work.  Nothing here touches the
data path.
"""


def cloud_seed(base, rank):
    """Seed of rank `rank`'s cloud: independent clouds, reproducible per rank."""
    return int(base) + 7919 * int(rank)


def max_over_ranks(value, world):
    """The maximum of a float over all ranks (identity when world == 1).  Uses
    the initialised process group: a CUDA tensor under NCCL, a CPU tensor
    under gloo."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist

    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_value(bytes_per_rank, ms_max, world):
    """Whole-job throughput in GB/s: every rank moved bytes_per_rank in at most
    ms_max milliseconds."""
    return world * float(bytes_per_rank) / (float(ms_max) * 1e-3) / 1e9
