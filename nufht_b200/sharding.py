"""Multi-GPU sharding of a batched transform, one process per GPU.

The transform has no exchange step, so it shards two ways without any collective inside a
transform:

* column blocks (B >= world size): each rank plans the same grids and transforms its own
  contiguous block of the B columns; `gather_columns` assembles the full result where a
  caller needs it on every rank;
* target rows (B < world size, e.g. one or a few columns): the targets k are split into
  contiguous ranges, rank q plans the sub-rectangle [k_q] x [all r] on its GPU and evaluates
  every column at its own targets; the coefficients c are broadcast from one rank, and the
  disjoint row blocks of g are all-gathered.  The adjoint shards the same way with the roles
  of r and k swapped (its targets are r).

`sharding_mode` picks between them.  Collectives go through torch.distributed (NCCL between
GPUs; gloo on the CPU for the tests).
"""


def column_block(total_cols, world, rank):
    """[start, stop) of the columns owned by `rank` (blocks differ in size by at most 1)."""
    base, extra = divmod(int(total_cols), int(world))
    start = rank * base + min(rank, extra)
    stop = start + base + (1 if rank < extra else 0)
    return start, stop


def target_rows(n_targets, world, rank):
    """[start, stop) of the targets owned by `rank`: contiguous ranges of the sorted k whose
    sizes differ by at most 1."""
    return column_block(n_targets, world, rank)


def sharding_mode(batch, world):
    """'columns' when every rank gets at least one column, else 'targets'."""
    return "columns" if int(batch) >= int(world) else "targets"


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


def gather_rows(local, total_rows, group=None):
    """All-gather target-row blocks (each rank's `local` is (B, its rows), column t = row t)
    into (B, total_rows) on every rank."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    B = local.shape[0]
    sizes = [target_rows(total_rows, world, r)[1] - target_rows(total_rows, world, r)[0] for r in range(world)]
    smax = max(sizes)
    pad = torch.zeros((B, smax), dtype=local.dtype, device=local.device)
    pad[:, : local.shape[1]] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad.contiguous(), group=group)
    return torch.cat([p[:, :s] for p, s in zip(parts, sizes)], dim=1)


def broadcast_inputs(c, src=0, group=None):
    """Broadcast the coefficient block c (B, m) from rank `src` to every rank, in place."""
    import torch.distributed as dist
    dist.broadcast(c, src=src, group=group)
    return c


class TargetShardedTransform:
    """g = H c with the targets split across the ranks of `group`.

    Rank q plans its sub-rectangle [k_q] x [all r] once (`make_plan(nu, r, k_q, tol, **kw)`,
    by default a DevicePlan on this rank's GPU); each call broadcasts c (B, m) from `src`,
    transforms it at the rank's own targets and all-gathers the rows, returning (B, n) on
    every rank.  `plan_rows` are this rank's target indices [start, stop).
    """

    def __init__(self, nu, r, k, tol=1e-8, *, group=None, make_plan=None, **plan_kw):
        import numpy as np
        import torch.distributed as dist
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.n = len(k)
        self.m = len(r)
        a, b = target_rows(self.n, self.world, self.rank)
        self.plan_rows = (a, b)
        if make_plan is None:
            from .plan import DevicePlan as make_plan
        k_local = np.ascontiguousarray(np.asarray(k, dtype=np.float64)[a:b])
        self.plan = make_plan(nu, r, k_local, tol, **plan_kw) if b > a else None

    def __call__(self, c_cols, src=0):
        import torch
        c_cols = broadcast_inputs(c_cols.contiguous(), src=src, group=self.group)
        a, b = self.plan_rows
        if self.plan is not None:
            g_local = self.plan.execute_columns(c_cols)
        else:
            g_local = torch.zeros((c_cols.shape[0], 0), dtype=c_cols.dtype, device=c_cols.device)
        return gather_rows(g_local, self.n, group=self.group)
