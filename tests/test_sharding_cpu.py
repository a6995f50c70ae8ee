"""Scene sharding (cloudrendering_b200.scene_sharding) and data-parallel training's gradient averaging
(cloudrendering_b200.learned_denoiser.average_gradients) with world size 2 on the gloo backend; the CPU
oracle stands in for each rank's GPU renderer."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from cloudrendering_b200.scene_sharding import assign_lpt, rank_loads, render_scenes_sharded, scene_cost


def test_lpt_assignment_covers_every_scene_once_and_balances():
    rng = np.random.default_rng(1000)
    costs = [scene_cost(int(r), int(r), int(s), float(e)) for r, s, e in
             zip(rng.integers(128, 1025, 64), rng.integers(1, 65, 64), rng.uniform(100, 2000, 64))]
    for world in (1, 2, 3, 8):
        a = assign_lpt(costs, world)
        assert sorted(i for lst in a for i in lst) == list(range(64))
        loads = rank_loads(costs, a)
        # LPT bound: the largest load is at most 4/3 of the optimum, which is >= max(mean, largest job)
        lower = max(sum(costs) / world, max(costs))
        assert max(loads) <= 4.0 / 3.0 * lower + 1e-6
        assert a == assign_lpt(costs, world)  # deterministic: every rank computes the same split


def test_lpt_rejects_bad_input():
    with pytest.raises(ValueError):
        assign_lpt([1.0], 0)
    with pytest.raises(ValueError):
        scene_cost(0, 8, 1, 100.0)


SCENES = [(16, 12, 3, 40.0), (24, 20, 2, 120.0), (8, 8, 5, 300.0), (20, 16, 1, 60.0), (12, 12, 4, 200.0)]


def oracle_image(i):
    from tests.harness import SceneSpec, cloud_block, oracle_scene
    w, h, spp, ext = SCENES[i]
    sp = SceneSpec(grid=cloud_block(8, 8, 8, empty_boundary=True), mode="delta", width=w, height=h, extinction=ext,
                   seed_offset=1000 + i)
    sc = oracle_scene(None, sp, spp)
    film, _, _ = sc.render()
    return film.reshape(h, w, 3) / spp


def worker(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        costs = [scene_cost(w, h, s, e) for w, h, s, e in SCENES]
        seen = []

        def render(indices):
            seen.extend(indices)
            return {i: oracle_image(i) for i in indices}

        merged = render_scenes_sharded(costs, render, gather=True)
        np.save(os.path.join(out_dir, f"seen{rank}.npy"), np.array(sorted(seen), np.int64))
        if rank == 0:
            np.savez(os.path.join(out_dir, "merged.npz"), **{str(k): v for k, v in merged.items()})
        else:
            assert merged is None
        # data-parallel gradient averaging: each rank's gradient differs, the average is their mean
        from cloudrendering_b200.learned_denoiser import average_gradients
        g = torch.arange(10, dtype=torch.float32) * (rank + 1)
        average_gradients(g)
        np.save(os.path.join(out_dir, f"grad{rank}.npy"), g.numpy())
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_scene_sharding_and_gradient_average_world2(tmp_path):
    mp.spawn(worker, args=(2, free_port(), str(tmp_path)), nprocs=2, join=True)
    seen = [np.load(tmp_path / f"seen{r}.npy").tolist() for r in range(2)]
    assert sorted(seen[0] + seen[1]) == list(range(len(SCENES)))  # every scene on exactly one rank
    assert seen[0] and seen[1]
    merged = np.load(tmp_path / "merged.npz")
    for i in range(len(SCENES)):
        assert np.array_equal(merged[str(i)], oracle_image(i))  # same image as a single-process render
    want = np.arange(10, dtype=np.float32) * 1.5
    for r in range(2):
        assert np.array_equal(np.load(tmp_path / f"grad{r}.npy"), want)
