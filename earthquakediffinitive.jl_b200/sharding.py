"""Column-sharded K builds over several GPUs (one process per GPU).

The columns of K are independent solves, so a build over N ranks gives each
rank a contiguous block of columns (no exchange while solving). The only
exchange is the optional all-gather that hands every rank the full K, e.g.
for a time loop that multiplies by K on each rank (src/BP8.jl:366). Over
NCCL the blocks are device tensors and the gather runs over NVLink; over
gloo (CPU processes) the same code gathers host tensors.

The reference builds K in one process with Julia threads over columns
(`fault_stiffness(...; threaded=true)`, src/FaultResponse.jl:244-263); the
sharded build gives the same matrix, column for column.
"""
import numpy as np


def shard_range(ncols, rank, world):
    """Contiguous, balanced column block [lo, hi) of `rank` among `world`."""
    if world < 1 or not 0 <= rank < world or ncols < 0:
        raise ValueError(f"bad shard request: ncols={ncols} rank={rank} world={world}")
    return ncols * rank // world, ncols * (rank + 1) // world


def _dist():
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        raise RuntimeError("torch.distributed is not initialised")
    return dist


def max_over_ranks(value, group=None, device="cpu"):
    """Max of a float over all ranks (step times are reported as the max)."""
    import torch
    dist = _dist()
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def gather_columns(block, ncols, group=None):
    """All-gather column blocks into the full (nrows, ncols) matrix on every
    rank. `block` is this rank's (nrows, hi - lo) block as a torch tensor
    (device tensor for NCCL, host tensor for gloo); blocks follow
    `shard_range`. Returns a torch tensor on the block's device."""
    import torch
    dist = _dist()
    world = dist.get_world_size(group)
    nrows = block.shape[0]
    width = max(shard_range(ncols, r, world)[1] - shard_range(ncols, r, world)[0] for r in range(world))
    # Column-major blocks: transpose so each rank's columns are contiguous rows.
    send = torch.zeros((width, nrows), dtype=block.dtype, device=block.device)
    send[: block.shape[1]] = block.T
    recv = torch.empty((world * width, nrows), dtype=block.dtype, device=block.device)
    dist.all_gather_into_tensor(recv, send, group=group)
    out = torch.empty((ncols, nrows), dtype=block.dtype, device=block.device)
    for r in range(world):
        lo, hi = shard_range(ncols, r, world)
        out[lo:hi] = recv[r * width: r * width + (hi - lo)]
    return out.T


def fault_stiffness_sharded(fe, build=None, group=None, gather=True, device=None):
    """Build this rank's column block of K (and, with `gather`, the full K on
    every rank). `build(cols) -> (2nf, len(cols)) ndarray` defaults to the GPU
    column build `stiffness_columns(fe, cols)`. Returns (K or block, (lo, hi))."""
    import torch
    dist = _dist()
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    ncols = 2 * fe.nf
    lo, hi = shard_range(ncols, rank, world)
    cols = np.arange(lo, hi, dtype=np.int32)
    if build is None:
        from . import stiffness_columns
        block = stiffness_columns(fe, cols)[0]
    else:
        block = build(cols)
    block = np.ascontiguousarray(block, dtype=np.float64)
    if block.shape != (ncols, hi - lo):
        raise ValueError(f"column block has shape {block.shape}, expected {(ncols, hi - lo)}")
    if not gather:
        return block, (lo, hi)
    if device is None:
        device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    K = gather_columns(torch.from_numpy(block).to(device), ncols, group=group)
    return K.cpu().numpy(), (lo, hi)
