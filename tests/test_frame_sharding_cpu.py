"""Frame sharding across ranks (cloudrendering_b200.frame_sharding) with world size 2 on the gloo
backend: each rank renders its frame range with the CPU oracle standing in for its GPU, the FP64
films are all-reduced, and the mean equals a single render of all frames."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from cloudrendering_b200.frame_sharding import frame_range, render_sharded

W, H, FRAMES = 24, 20, 7


def scene():
    from oracle import bridge
    from tests.harness import SceneSpec, cloud_block, oracle_scene
    sp = SceneSpec(grid=cloud_block(8, 8, 8, empty_boundary=True), mode="delta", width=W, height=H, extinction=60.0)
    return oracle_scene(None, sp, FRAMES), bridge


def oracle_film(first, count):
    sc, _ = scene()
    sc.set("frame_count", first)
    sc.set("num_frames", count)
    film, _, _ = sc.render()
    return torch.from_numpy(film.reshape(H, W, 3).transpose(2, 0, 1).astype(np.float64).copy())


def worker(rank, world, port, out_path):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mean = render_sharded(FRAMES, W, H, render_fn=oracle_film)
        if rank == 0:
            np.save(out_path, mean.numpy())
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_frame_range_partitions_the_frames():
    for world in (1, 2, 3, 8):
        for total in (0, 1, 7, 64, 65):
            ranges = [frame_range(r, world, total) for r in range(world)]
            covered = [f for first, n in ranges for f in range(first, first + n)]
            assert covered == list(range(total))


def test_two_ranks_equal_one_render(tmp_path):
    out = str(tmp_path / "mean.npy")
    mp.start_processes(worker, args=(2, free_port(), out), nprocs=2, start_method="spawn", join=True)
    sharded = np.load(out)
    single = oracle_film(0, FRAMES).numpy() / FRAMES
    assert np.abs(single).sum() > 0
    assert np.allclose(sharded, single, rtol=1e-12, atol=1e-14)
