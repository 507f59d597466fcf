"""Sharding of ray work across ranks (one process per GPU).

Rays and frames are independent, so the path shards without any data-path
collective: a rank takes whole frames (round robin) or a contiguous block of
pixel rows of one frame. The only collectives are the timing ones (a barrier and
the maximum of the elapsed device time over ranks) and, when one frame is split,
the gather of the row blocks to rank 0 (the one exchange of a split frame).
"""


def frames_for_rank(frames, rank, world):
    """Whole frames for this rank: frames rank, rank + world, ..."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    return list(frames[rank::world])


def row_block(height, rank, world):
    """Contiguous pixel rows [r0, r1) of a frame for this rank (sizes differ by at most one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    base, extra = divmod(height, world)
    r0 = rank * base + min(rank, extra)
    return r0, r0 + base + (1 if rank < extra else 0)


def max_over_ranks(value, dist=None, device=None):
    """The maximum of a per-rank scalar (e.g. elapsed device milliseconds) over ranks."""
    import torch
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_rows(block, height, width, dist=None, device=None):
    """Rank 0 assembles the full frame from every rank's row block (row-major
    float32 array of (r1 - r0) * width values); other ranks get None."""
    import torch
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return block
    world, rank = dist.get_world_size(), dist.get_rank()
    rows = [row_block(height, r, world) for r in range(world)]
    longest = max(r1 - r0 for r0, r1 in rows) * width
    pad = torch.zeros(longest, dtype=torch.float32, device=device)
    pad[:block.numel()] = block.reshape(-1)
    parts = [torch.zeros(longest, dtype=torch.float32, device=device) for _ in range(world)]
    dist.all_gather(parts, pad)
    if rank != 0:
        return None
    return torch.cat([parts[r][:(r1 - r0) * width] for r, (r0, r1) in enumerate(rows)])
