"""Multi-GPU plumbing for the field and arrangement evaluators.

The path shards with no exchange: points (or arrangements) are split into
contiguous slices, one per rank, and every rank evaluates all coils on its own
slice with its own copy of the node tables.  The only collectives are the
optional gather of the results onto every rank and the max-over-ranks of a
timing, both through torch.distributed (NCCL between GPUs; gloo works the same
way on CPU, which is how the tests run two ranks).
"""
import numpy as np
import torch
import torch.distributed as dist


def world():
    """(rank, world size) of the default process group, or (0, 1) without one."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def shard_bounds(n, rank, world_size):
    """Contiguous slice [lo, hi) of n items for `rank`; sizes differ by at most one."""
    if world_size < 1 or not 0 <= rank < world_size or n < 0:
        raise ValueError("need 0 <= rank < world_size and n >= 0")
    base, extra = divmod(n, world_size)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def barrier():
    if world()[1] > 1:
        dist.barrier()


def max_over_ranks(x, device=None):
    """Maximum of a float over all ranks (the step time of a multi-GPU run)."""
    if world()[1] == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def evaluate_sharded(evaluate, points, gather=True, device=None):
    """Evaluates this rank's contiguous slice of `points` (n, 3) with `evaluate`
    (a function of an (m, 3) array returning (m, k) results) and, with gather,
    returns the full (n, k) result on every rank (all_gather of equal-size padded
    slices); without gather, returns (lo, hi, local results)."""
    rank, size = world()
    n = len(points)
    lo, hi = shard_bounds(n, rank, size)
    local = evaluate(points[lo:hi])
    local_t = torch.as_tensor(np.asarray(local) if not torch.is_tensor(local) else local)
    if not gather:
        return lo, hi, local_t
    if size == 1:
        return local_t
    width = local_t.shape[1] if local_t.dim() > 1 else 1
    cap = shard_bounds(n, 0, size)[1]  # the largest slice
    pad = torch.zeros((cap, width), dtype=local_t.dtype, device=device if device is not None else local_t.device)
    pad[: hi - lo] = local_t.reshape(hi - lo, width).to(pad.device)
    parts = [torch.empty_like(pad) for _ in range(size)]
    dist.all_gather(parts, pad)
    out = [parts[r][: shard_bounds(n, r, size)[1] - shard_bounds(n, r, size)[0]] for r in range(size)]
    full = torch.cat(out, dim=0)
    return full if local_t.dim() > 1 else full.reshape(-1)
