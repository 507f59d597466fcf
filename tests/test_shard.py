"""The multi-rank path on CPU: sharding arithmetic, and the timing maximum and
row gather over a world of two gloo ranks (the collectives the GPU run uses
over NCCL)."""
import os

import pytest

from sirius_b200 import shard


def test_row_blocks_cover_the_frame_once():
    for height in (1, 7, 1024, 2049):
        for world in (1, 2, 3, 8):
            blocks = [shard.row_block(height, r, world) for r in range(world)]
            assert blocks[0][0] == 0 and blocks[-1][1] == height
            for (a0, a1), (b0, b1) in zip(blocks, blocks[1:]):
                assert a1 == b0
            sizes = [r1 - r0 for r0, r1 in blocks]
            assert max(sizes) - min(sizes) <= 1


def test_frames_round_robin():
    frames = list(range(10))
    got = [shard.frames_for_rank(frames, r, 3) for r in range(3)]
    assert sorted(sum(got, [])) == frames
    assert got[0] == [0, 3, 6, 9]
    with pytest.raises(ValueError):
        shard.frames_for_rank(frames, 3, 3)


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        height, width = 9, 4
        r0, r1 = shard.row_block(height, rank, world)
        block = torch.arange(r0 * width, r1 * width, dtype=torch.float32)
        full = shard.gather_rows(block, height, width, dist)
        tmax = shard.max_over_ranks(10.0 + rank, dist)
        q.put((rank, None if full is None else full.tolist(), tmax))
    finally:
        dist.destroy_process_group()


def test_two_rank_gather_and_time_max():
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict()
    for _ in range(2):
        rank, full, tmax = q.get(timeout=120)
        out[rank] = (full, tmax)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][0] == [float(i) for i in range(36)]
    assert out[1][0] is None
    assert out[0][1] == out[1][1] == 11.0
