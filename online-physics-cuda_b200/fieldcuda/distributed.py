"""Several GPUs, one process each (torch.distributed over NCCL; gloo on the CPU): the instance-sharded forms.

The batched ADI, the learned solves and the calibration are independent instances: each rank takes a contiguous shard
of the options or samples, works on its own GPU with no data-path exchange, and only results meet at the end. Where a
result is a sum over ranks (a calibration loss and gradient), it is summed in rank order after an all-gather, in FP64,
so every rank holds the same bits whatever order the collective itself reduces in. No load on this path uses TMA
multicast; the collectives are NCCL's (or gloo's).
"""
import numpy as np
import torch
import torch.distributed as dist


def world():
    return (dist.get_world_size(), dist.get_rank()) if dist.is_available() and dist.is_initialized() else (1, 0)


def shard_range(n, rank, size):
    """The contiguous [lo, hi) of n items rank `rank` of `size` takes (the first n % size ranks take one more)."""
    base, extra = divmod(n, size)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def fixed_order_sum(values, device=None):
    """The sum over ranks of `values` (a float array or tensor), every rank's contribution gathered and added in rank
    order in FP64: the same bits on every rank and from run to run."""
    size, _ = world()
    v = torch.as_tensor(np.asarray(values, np.float64) if not isinstance(values, torch.Tensor) else values,
                        dtype=torch.float64)
    if size == 1:
        return v.clone()
    if device is not None:
        v = v.to(device)
    parts = [torch.empty_like(v) for _ in range(size)]
    dist.all_gather(parts, v)
    out = torch.zeros_like(parts[0])
    for p in parts:
        out = out + p
    return out.cpu()


def max_over_ranks(value, device=None):
    size, _ = world()
    if size == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def calibration_loss_and_grad(law_text, strikes, common, targets, nx, ny, steps, values):
    """The Heston calibration's loss and gradient with the options sharded over the ranks (each rank's shard on its
    own GPU as the z-planes of its lattice), summed in rank order: the same numbers on every rank."""
    from .heston import Calibration
    size, rank = world()
    lo, hi = shard_range(len(strikes), rank, size)
    cal = Calibration(law_text, strikes[lo:hi], common["maturity"], common["spot"], common["r"], targets[lo:hi], nx, ny, steps)
    loss, grad = cal.loss_and_grad(values)
    cal.close()
    total = fixed_order_sum(np.concatenate([[loss], grad]), device="cuda" if size > 1 and dist.get_backend() == "nccl" else None)
    return float(total[0]), total[1:].numpy()
