"""The N>1 host logic of bench.py on two CPU ranks (gloo).

Multi-GPU runs are weak scaling with no data-path collective: every rank renders
the same frame over its own block of sample indices, and the only collectives are
the timing reductions (maximum over ranks). These tests run that logic as two
gloo processes on 127.0.0.1, with the oracle's estimator standing in for the
GPU render, and check that the ranks' frames add up to one render of all their
samples and that the job time is the slowest rank's.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORLD = 2
SPP = 2
STEPS = 3


def _free_port() -> int:
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, port: int, out_dir: str):
    sys.path.insert(0, ROOT)
    import datetime

    import torch
    import torch.distributed as dist

    import bench
    import oracle
    from rednoise_b200 import scenes

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=WORLD,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # sample blocks of every (step, rank)
        mine = torch.tensor([bench.shard_sample_offset(k, rank, WORLD, SPP) for k in range(STEPS)], dtype=torch.int64)
        every = [torch.zeros_like(mine) for _ in range(WORLD)]
        dist.all_gather(every, mine)

        # each rank renders its step-0 block; the frames are summed (test only: the bench
        # itself exchanges no image data)
        sc = scenes.cornell_box()
        cam = scenes.camera(10, 8)
        orc = oracle.OrcPhysScene(sc)
        sums = orc.render_sums(cam, SPP, 4, 4, seed=1, offset=int(mine[0]))
        t = torch.from_numpy(sums.copy())
        dist.all_reduce(t, op=dist.ReduceOp.SUM)

        # per-rank timings: the job time is the slowest rank's
        mx = bench.max_over_ranks([rank + 1.0, 10.0 - rank], dist)

        if rank == 0:
            np.savez(os.path.join(out_dir, "r0.npz"), every=torch.stack(every).numpy(), summed=t.numpy(),
                     mx=np.array(mx))
    finally:
        dist.destroy_process_group()


@pytest.fixture(scope="module")
def gloo_run(tmp_path_factory):
    out = tmp_path_factory.mktemp("gloo")
    mp.start_processes(_worker, args=(_free_port(), str(out)), nprocs=WORLD, join=True, start_method="spawn")
    return np.load(out / "r0.npz")


def test_sample_blocks_are_disjoint_and_contiguous(gloo_run):
    every = gloo_run["every"]  # (rank, step)
    starts = np.sort(every.reshape(-1))
    assert np.array_equal(starts, np.arange(WORLD * STEPS) * SPP)


def test_rank_frames_sum_to_one_render(gloo_run):
    import oracle
    from rednoise_b200 import scenes

    whole = oracle.OrcPhysScene(scenes.cornell_box()).render_sums(scenes.camera(10, 8), WORLD * SPP, 4, 4, seed=1)
    assert whole.sum() > 0
    np.testing.assert_allclose(gloo_run["summed"], whole, rtol=1e-12, atol=1e-12)


def test_timing_is_max_over_ranks(gloo_run):
    assert list(gloo_run["mx"]) == [2.0, 10.0]


def test_single_rank_max_is_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks([3.5, 1.0]) == [3.5, 1.0]
    assert bench.shard_sample_offset(0, 0, 1, 64) == 0
    assert bench.shard_sample_offset(2, 0, 1, 64) == 128


def _spawned(out_dir: str):
    import datetime

    import torch
    import torch.distributed as dist

    import bench

    rank, local_rank, world = bench.dist_env()
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        t = torch.tensor([rank, local_rank, world, dist.get_rank(), dist.get_world_size()], dtype=torch.int64)
        every = [torch.zeros_like(t) for _ in range(world)]
        dist.all_gather(every, t)
        if rank == 0:
            np.save(os.path.join(out_dir, "ranks.npy"), torch.stack(every).numpy())
    finally:
        dist.destroy_process_group()


def test_spawn_ranks_sets_the_launcher_environment(tmp_path):
    """bench.py --gpus N without torchrun starts N ranks with torchrun's environment
    (RANK, LOCAL_RANK, WORLD_SIZE, MASTER_ADDR=127.0.0.1, MASTER_PORT)."""
    sys.path.insert(0, ROOT)
    import bench

    bench.spawn_ranks(2, _spawned, str(tmp_path))
    got = np.load(tmp_path / "ranks.npy")
    assert got.tolist() == [[0, 0, 2, 0, 2], [1, 1, 2, 1, 2]]
