"""Batched boxes sharded across two ranks, stepped for real.

Two processes with a gloo group share cuda:0 as two ranks would share a
node. Each takes its LPT share (sharding.lpt_shards) of eight boxes of the
batched workload's construction, steps them as one batch for three frames
of four substeps (tolerance solve, each box its own tilt and XSPH
coefficient), and the ranks assemble every box's statistics with
sharding.gather_box_values, the reduction the benchmark's multi-GPU leg
runs over NCCL. The boxes are independent: every box's resting set and
iteration counts must be bit-identical to the same box in one unsharded
batch of all eight, and the gathered rows to the unsharded batch's
statistics. The ranks' kernels never wait on one another; the only
exchange is the host-side gloo all-reduce after both have synchronised.
"""
import importlib.util
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

from test_gpu_step import assert_same_bits

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "fluid-simulation-app_b200")
NBOXES, FRAMES, WORLD = 8, 3, 2
KEYS = ("pos", "vel", "prev_vel", "prev_p", "temp", "id")


def _mod(name):
    spec = importlib.util.spec_from_file_location(name, os.path.join(PKG, name + ".py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _boxes(fcu, wl):
    return wl.batched_boxes(fcu, nboxes=NBOXES, seed=7, lo=800, hi=6000)


def _rows(stats_after):
    return [[s.total_den_iters, s.total_div_iters, s.compression_avg, s.compression_max,
             s.den_residual] for s in stats_after]


def _rank(rank, port, out_dir):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD)
    torch.cuda.set_device(0)
    fcu, wl, sh = _mod("fluidcu"), _mod("workloads"), _mod("sharding")
    cfgs = _boxes(fcu, wl)
    counts = [c.block[0] * c.block[1] * c.block[2] for c in cfgs]
    mine = sh.lpt_shards(counts, WORLD)[rank]
    batch = fcu.Batch([cfgs[b] for b in mine])
    steps_all = wl.batched_frame_steps(fcu, NBOXES, FRAMES, substeps=4, seed=7)
    batch.run([[row[b] for b in mine] for row in steps_all])
    batch.sync()
    batch.reduce_stats()
    rows = sh.gather_box_values(mine, _rows(batch.stats()), NBOXES)
    states = {f"{b}_{k}": v for i, b in enumerate(mine) for k, v in batch.state(i).items()}
    np.savez(os.path.join(out_dir, f"rank{rank}.npz"), mine=np.asarray(mine), rows=rows, **states)
    batch.close()
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_step_their_shards_as_one_batch_would(fcu, wl, tmp_path):
    sh = _mod("sharding")
    cfgs = _boxes(fcu, wl)
    counts = [c.block[0] * c.block[1] * c.block[2] for c in cfgs]
    shards = sh.lpt_shards(counts, WORLD)
    assert all(len(s) >= 2 for s in shards)
    port = 29600 + os.getpid() % 1000
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank, args=(r, port, str(tmp_path))) for r in range(WORLD)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(600)
        assert p.exitcode == 0
    # the same eight boxes in one batch on this process
    batch = fcu.Batch(cfgs)
    batch.run(wl.batched_frame_steps(fcu, NBOXES, FRAMES, substeps=4, seed=7))
    batch.sync()
    batch.reduce_stats()
    want_rows = np.asarray(_rows(batch.stats()), np.float64)
    seen = set()
    for r in range(WORLD):
        got = np.load(tmp_path / f"rank{r}.npz")
        assert got["mine"].tolist() == shards[r]
        assert np.array_equal(got["rows"], want_rows), r
        for b in shards[r]:
            want = batch.state(b)
            for k in KEYS:
                assert_same_bits(got[f"{b}_{k}"], want[k], f"rank {r} box {b} {k}")
            seen.add(b)
    assert seen == set(range(NBOXES))
    assert want_rows[:, 0].min() > 0  # every box iterated
    batch.close()
