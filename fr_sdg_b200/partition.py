"""Row-block domain decomposition of the 2D mesh over ranks (one GPU each).

The reference distributes the mesh with a PETSc DMDA and refreshes a ghosted local
view before every residual (DMGlobalToLocal; physics_impl_2D.hpp:646-902 reads the
neighbour traces from it).  Here rank r owns a contiguous block of element rows,
stores one ghost element row on each side that has a neighbour (the periodic wrap
included) and, before every residual, receives those rows from its neighbours over
NCCL (torch.distributed point-to-point).  Element rows are contiguous in the DMDA
layout, so every message is one contiguous slice.  The kernels see the block through
frsdg_set_row_window.
"""
from __future__ import annotations

from dataclasses import dataclass


@dataclass(frozen=True)
class RowBlock:
    rank: int
    ranks: int
    g_begin: int        # first owned global row
    g_end: int          # one past the last owned global row
    ghost_below: bool
    ghost_above: bool
    down: int | None    # rank owning the row below (periodic wrap included), None at a physical edge
    up: int | None

    @property
    def owned(self) -> int:
        return self.g_end - self.g_begin

    @property
    def rows(self) -> int:
        """Element rows held locally (owned + ghosts)."""
        return self.owned + int(self.ghost_below) + int(self.ghost_above)

    @property
    def row_base(self) -> int:
        """Global row of local row 0 (-1 for a periodic wrap below row 0)."""
        return self.g_begin - int(self.ghost_below)

    @property
    def row_begin(self) -> int:
        return int(self.ghost_below)

    @property
    def row_end(self) -> int:
        return self.row_begin + self.owned

    def window(self) -> tuple[int, int, int, int]:
        return self.row_base, self.rows, self.row_begin, self.row_end


def row_blocks(ny: int, ranks: int, periodic_y: bool) -> list[RowBlock]:
    """Split ny element rows into `ranks` contiguous blocks (sizes differ by at most one)."""
    if ranks < 1 or ny < ranks:
        raise ValueError(f"cannot split {ny} element rows over {ranks} ranks")
    out = []
    base, extra = divmod(ny, ranks)
    g = 0
    for r in range(ranks):
        n = base + (1 if r < extra else 0)
        wrap = periodic_y and ranks > 1
        down = r - 1 if r > 0 else (ranks - 1 if wrap else None)
        up = r + 1 if r < ranks - 1 else (0 if wrap else None)
        out.append(RowBlock(r, ranks, g, g + n, down is not None, up is not None, down, up))
        g += n
    return out


def scatter_rows(U_global, blk: RowBlock, nx: int, nd: int):
    """The local vector of block `blk` cut from a global one (ghost rows included), for
    tests and set-up; a copy."""
    import torch

    ny = U_global.numel() // (nx * nd)
    G = U_global.view(ny, nx * nd)
    rows = [(blk.g_begin - 1) % ny] if blk.ghost_below else []
    rows += list(range(blk.g_begin, blk.g_end))
    rows += [blk.g_end % ny] if blk.ghost_above else []
    return G[torch.tensor(rows, device=U_global.device)].reshape(-1).contiguous()


def exchange_ghost_rows(U_local, blk: RowBlock, row_len: int, group=None) -> None:
    """Fill the ghost rows of U_local from the neighbouring ranks (collective over the
    group: every rank calls it).  Messages: each rank sends its last owned row up and
    receives its ghost below from down, then sends its first owned row down and
    receives its ghost above from up -- the same order on every rank, so the pairs
    match also when down == up (two ranks, periodic)."""
    import torch.distributed as dist

    V = U_local.view(blk.rows, row_len)
    ops = []
    if blk.up is not None:
        ops.append(dist.P2POp(dist.isend, V[blk.row_end - 1], blk.up, group))
    if blk.down is not None:
        ops.append(dist.P2POp(dist.irecv, V[0], blk.down, group))
    if blk.down is not None:
        ops.append(dist.P2POp(dist.isend, V[blk.row_begin], blk.down, group))
    if blk.up is not None:
        ops.append(dist.P2POp(dist.irecv, V[blk.rows - 1], blk.up, group))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()


def ghost_hook(blk: RowBlock, row_len: int, group=None):
    """A stage hook for fr_sdg_b200.integrate.Integrator(before_stage=...): refreshes the
    ghost rows of every stage input (and of the state before the post-step limiter)
    from the neighbouring ranks."""
    return lambda V: exchange_ghost_rows(V, blk, row_len, group)


def global_max(x: float, device, group=None) -> float:
    """Max over the ranks of a host scalar (the CFL time step's wave speed)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
