"""Ensemble sharding over ranks (aether_fluid.sharding) on the CPU: the
cell-balanced partition, and the host-side gather over a gloo process group of
two ranks with a stand-in runner (the device part is the batched ensemble,
covered by the GPU tests)."""
import os
import socket
from collections import namedtuple

import numpy as np
import pytest

from aether_fluid.sharding import run_sharded, shard_instances

Spec = namedtuple("Spec", "nx ny nz seed")
Spec.cells = property(lambda s: s.nx * s.ny * s.nz)

PLUME48_CELLS = [32 ** 3] * 16 + [48 ** 3] * 16 + [64 * 128 * 64] * 16


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_partition_covers_every_instance_once(world):
    shards = shard_instances(PLUME48_CELLS, world)
    assert len(shards) == world
    flat = sorted(i for s in shards for i in s)
    assert flat == list(range(len(PLUME48_CELLS)))
    assert all(s == sorted(s) for s in shards)


@pytest.mark.parametrize("world", [2, 4, 8])
def test_partition_is_balanced(world):
    shards = shard_instances(PLUME48_CELLS, world)
    loads = [sum(PLUME48_CELLS[i] for i in s) for s in shards]
    # largest-first greedy: the spread is at most one instance
    assert max(loads) - min(loads) <= max(PLUME48_CELLS)
    # the 48-plume ensemble splits evenly over 2, 4 and 8 ranks
    assert max(loads) == min(loads)


def test_partition_random_sizes_bound():
    rng = np.random.default_rng(5)
    for _ in range(50):
        cells = [int(c) for c in rng.integers(1, 10_000, size=int(rng.integers(1, 40)))]
        world = int(rng.integers(1, 9))
        shards = shard_instances(cells, world)
        assert sorted(i for s in shards for i in s) == list(range(len(cells)))
        loads = [sum(cells[i] for i in s) for s in shards]
        assert max(loads) - min(loads) <= max(cells)
        assert shard_instances(cells, world) == shards  # deterministic


def test_partition_more_ranks_than_instances():
    shards = shard_instances([10, 20], 4)
    assert sorted(len(s) for s in shards) == [0, 0, 1, 1]


def test_partition_rejects_bad_input():
    with pytest.raises(ValueError):
        shard_instances([1, 2], 0)
    with pytest.raises(ValueError):
        shard_instances([1, 0], 2)


def fake_runner(local_specs, steps):
    """Telemetry that names its instance, so the gather's order can be checked."""
    k = len(local_specs)
    tel = np.zeros((steps, k, 8))
    for t in range(steps):
        for j, s in enumerate(local_specs):
            tel[t, j] = [t, s.seed, s.cells, os.getpid(), 0, 0, 0, 0]
    infos = [[("info", t, s.seed) for s in local_specs] for t in range(steps)]
    return tel, infos, {"pid": os.getpid()}


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, specs, steps, out_path):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        res = run_sharded(specs, steps, dist=dist, runner=fake_runner)
        if rank == 0:
            tel, infos, parts = res
            np.savez(out_path, tel=tel, seeds=np.array([[i[2] for i in row] for row in infos]),
                     ranks=np.array([p["rank"] for p in parts]),
                     pids=np.array([p["pid"] if "pid" in p else -1 for p in parts]))
        else:
            assert res is None
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,count", [(2, 7), (2, 1)])
def test_gather_over_two_gloo_ranks(tmp_path, world, count):
    import torch.multiprocessing as mp
    specs = [Spec(8 + 4 * (m % 3), 8, 8, 100 + m) for m in range(count)]
    steps = 3
    out = str(tmp_path / "gathered.npz")
    mp.start_processes(_rank_main, args=(world, _free_port(), specs, steps, out),
                       nprocs=world, start_method="spawn", join=True)
    got = np.load(out)
    tel, seeds = got["tel"], got["seeds"]
    assert tel.shape == (steps, count, 8)
    for m, s in enumerate(specs):
        assert np.all(tel[:, m, 1] == s.seed)
        assert np.all(tel[:, m, 2] == s.cells)
        assert np.all(seeds[:, m] == s.seed)
    assert np.array_equal(tel[:, 0, 0], np.arange(steps))
    assert sorted(got["ranks"].tolist()) == list(range(world))
    # with more than one instance, both ranks did work in their own process
    if count > 1:
        assert len(set(got["pids"].tolist())) == world


def test_single_process_path():
    specs = [Spec(8, 8, 8, 1), Spec(16, 8, 8, 2)]
    tel, infos, parts = run_sharded(specs, 2, dist=None, runner=fake_runner)
    assert tel.shape == (2, 2, 8) and parts[0]["indices"] == [0, 1]
    assert [i[2] for i in infos[1]] == [1, 2]
