"""CPU: row-block partitions, the ghost-row exchange, the integrator's ghost hook and the
global wave-speed maximum (gloo, 2 and 3 ranks)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from fr_sdg_b200.partition import exchange_ghost_rows, ghost_hook, global_max, row_blocks, scatter_rows


@pytest.mark.parametrize("ny,ranks,periodic", [(10, 1, False), (10, 1, True), (10, 2, False), (10, 2, True),
                                               (11, 3, False), (11, 3, True), (7, 7, True)])
def test_row_blocks_cover_and_link(ny, ranks, periodic):
    blks = row_blocks(ny, ranks, periodic)
    assert blks[0].g_begin == 0 and blks[-1].g_end == ny
    assert all(a.g_end == b.g_begin for a, b in zip(blks, blks[1:]))
    assert max(b.owned for b in blks) - min(b.owned for b in blks) <= 1
    for b in blks:
        if ranks == 1:
            assert not b.ghost_below and not b.ghost_above and b.window() == (0, ny, 0, ny)
            continue
        assert b.ghost_below == (b.rank > 0 or periodic) and b.ghost_above == (b.rank < ranks - 1 or periodic)
        if b.down is not None:
            assert blks[b.down].up == b.rank
        base, rows, rb, re_ = b.window()
        assert base + rb == b.g_begin and base + re_ == b.g_end and re_ - rb == b.owned
    with pytest.raises(ValueError):
        row_blocks(3, 4, False)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, ny, periodic, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        nx, nd = 3, 4
        G = torch.arange(ny * nx * nd, dtype=torch.float64)
        blk = row_blocks(ny, ws, periodic)[rank]
        want = scatter_rows(G, blk, nx, nd)
        got = want.clone().view(blk.rows, nx * nd)
        if blk.ghost_below:
            got[0] = -1.0
        if blk.ghost_above:
            got[-1] = -1.0
        got = got.reshape(-1)
        exchange_ghost_rows(got, blk, nx * nd)
        ok = bool(torch.equal(got, want))
        # the integrator's stage hook does the same refresh
        got2 = want.clone().view(blk.rows, nx * nd)
        if blk.ghost_below:
            got2[0] = -2.0
        if blk.ghost_above:
            got2[-1] = -2.0
        got2 = got2.reshape(-1)
        ghost_hook(blk, nx * nd)(got2)
        ok = ok and bool(torch.equal(got2, want))
        # the CFL wave speed is the max over the ranks
        ok = ok and global_max(rank + 0.5, "cpu") == ws - 0.5
        q.put((rank, ok))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("ws,periodic", [(2, False), (2, True), (3, False), (3, True)])
def test_ghost_exchange_gloo(ws, periodic):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, 8, periodic, q)) for r in range(ws)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = dict(q.get(timeout=5) for _ in range(ws))
    assert all(res.values()), res
