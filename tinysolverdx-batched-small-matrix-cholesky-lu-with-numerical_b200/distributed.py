"""Host-side helpers for running the batched solvers on several GPUs, one process
per GPU (torch.distributed). Every matrix is an independent unit, so a batch
shards by contiguous index ranges with no exchange step; the only collective is
the max-over-ranks of a timing or a counter. TinySolverDx itself is single-node
CPU code with no multi-device path.
"""
import torch


def shard_range(batch, world, rank):
    """[start, stop) of rank's contiguous share of `batch` matrices (sizes differ by <= 1)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    q, r = divmod(int(batch), int(world))
    start = rank * q + min(rank, r)
    return start, start + q + (1 if rank < r else 0)


def max_over_ranks(value, device=None):
    """Max of a scalar over all ranks of the default process group (the value itself
    when no group is initialised). Uses a CUDA tensor for NCCL, a CPU one for gloo."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_shards(t, batch, world):
    """Reassemble per-rank shards (leading dimension = the rank's shard size, as
    given by shard_range) into the full batch on every rank."""
    import torch.distributed as dist
    sizes = [shard_range(batch, world, r)[1] - shard_range(batch, world, r)[0] for r in range(world)]
    m = max(sizes)
    pad = torch.zeros((m,) + tuple(t.shape[1:]), dtype=t.dtype, device=t.device)
    pad[:t.shape[0]] = t
    outs = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(outs, pad)
    return torch.cat([o[:s] for o, s in zip(outs, sizes)])
