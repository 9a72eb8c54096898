"""Multi-GPU sharding of a batched transform: independent column blocks per rank.

The transform has no exchange step (SURVEY: every column is independent), so a global
batch of B columns is split into contiguous blocks, one per rank; each rank plans the same
grids on its own GPU and transforms its block.  `gather_columns` assembles the full result
where a caller needs it on every rank (an all-gather; not part of the timed transform).
"""


def column_block(total_cols, world, rank):
    """[start, stop) of the columns owned by `rank` (blocks differ in size by at most 1)."""
    base, extra = divmod(int(total_cols), int(world))
    start = rank * base + min(rank, extra)
    stop = start + base + (1 if rank < extra else 0)
    return start, stop


def gather_columns(local, total_cols, group=None):
    """All-gather column blocks (each rank's `local` is (rows, its columns)) into
    (rows, total_cols) on every rank."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rows = local.shape[0]
    widths = [column_block(total_cols, world, r)[1] - column_block(total_cols, world, r)[0] for r in range(world)]
    wmax = max(widths)
    pad = torch.zeros((rows, wmax), dtype=local.dtype, device=local.device)
    pad[:, : local.shape[1]] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad.contiguous(), group=group)
    return torch.cat([p[:, :w] for p, w in zip(parts, widths)], dim=1)
