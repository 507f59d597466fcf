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


def _frame(abi, row_begin=0, row_count=0):
    cam = abi.make_camera(r=60.0, theta_deg=70.0, width=24, height=21, fov=35.0)
    return abi.make_frame(abi.make_metric(a=0.9), cam, 0.0, 25.0, row_begin=row_begin, row_count=row_count)


def _oracle_cfg(abi):
    return abi.default_config(abs_tolerance=1e-8, rel_tolerance=1e-8, min_step=1e-9, max_step=2.0,
                              escape_radius=200.0, horizon_factor=1.01, max_steps=10000,
                              precision=abi.PRECISION_FP64)


def _row_block_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist

    from oracle.pyoracle import Oracle
    from sirius_b200 import abi
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        full = _frame(abi)
        h, w = full.camera.height, full.camera.width
        r0, r1 = shard.row_block(h, rank, world)
        res, _ = Oracle().trace_frame(_frame(abi, r0, r1 - r0), _oracle_cfg(abi))
        img = shard.gather_rows(torch.from_numpy(res["intensity"].copy()), h, w, dist)
        out = shard.gather_rows(torch.from_numpy(res["outcome"].astype("float32")), h, w, dist)
        q.put((rank, None if img is None else (img.numpy().tobytes(), out.numpy().tobytes())))
    finally:
        dist.destroy_process_group()


def test_two_rank_row_blocks_reassemble_the_full_frame(oracle):
    """Each of two gloo ranks traces its row block of one frame (the frame's row
    window) with the CPU oracle; the gathered image equals the full-frame trace
    bit for bit."""
    import socket

    import numpy as np
    import torch.multiprocessing as mp

    from sirius_b200 import abi
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_row_block_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=300) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[1] is None
    ref, _ = oracle.trace_frame(_frame(abi), _oracle_cfg(abi))
    assert got[0][0] == ref["intensity"].tobytes()
    assert got[0][1] == ref["outcome"].astype(np.float32).tobytes()
