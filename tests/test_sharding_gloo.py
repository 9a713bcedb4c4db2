"""Box sharding across ranks: the LPT partition and the per-box statistics
reduction, run as two gloo processes on the CPU (the same code the
benchmark's multi-GPU batched leg runs over NCCL)."""
import importlib.util
import os
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _sharding():
    path = os.path.join(ROOT, "fluid-simulation-app_b200", "sharding.py")
    spec = importlib.util.spec_from_file_location("sharding", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_lpt_partitions_every_box_once_and_balances():
    sh = _sharding()
    rng = np.random.default_rng(3)
    counts = np.exp(rng.uniform(np.log(4096), np.log(65536), 256)).astype(int)
    for world in (1, 2, 3, 4, 8):
        shards = sh.lpt_shards(counts, world)
        flat = sorted(b for s in shards for b in s)
        assert flat == list(range(256))
        loads = sh.shard_loads(counts, shards)
        ideal = counts.sum() / world
        assert max(loads) <= max(ideal * 4 / 3, counts.max()) + 1
        assert max(loads) - min(loads) <= counts.max()
    assert sh.lpt_shards([5, 5, 5], 2) == [[0, 2], [1]]


def _worker(rank, world, port, counts, values, out_path):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sh = _sharding()
    shards = sh.lpt_shards(counts, world)
    mine = shards[rank]
    full = sh.gather_box_values(mine, values[mine], len(counts))
    if rank == 0:
        np.save(out_path, full)
    dist.barrier()
    dist.destroy_process_group()


def test_per_box_statistics_reduce_across_two_gloo_ranks(tmp_path):
    rng = np.random.default_rng(5)
    counts = rng.integers(4096, 65536, 37)
    values = rng.normal(size=(37, 4))
    out = str(tmp_path / "full.npy")
    port = 29500 + os.getpid() % 1000
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, 2, port, counts, values, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    full = np.load(out)
    assert np.array_equal(full, values)
