"""The batched workload's construction and the batch handle's argument
checks (host only: every refusal here happens before any device call)."""
import ctypes as C

import numpy as np


def test_the_batched_workload_has_its_shape(fcu, wl):
    cfgs = wl.batched_boxes(fcu)
    assert len(cfgs) == 256
    counts = np.array([c.block[0] * c.block[1] * c.block[2] for c in cfgs])
    assert counts.min() >= 3000 and counts.max() <= 70000
    assert 4.5e6 < counts.sum() < 6.5e6
    for c in cfgs:
        m = c.block[1]
        assert (c.block[0], c.block[2]) == (2 * m, 2 * m)
        assert abs(c.box_hi[1] - 2 * m * 0.005) < 1e-6
        assert 0.005 <= c.xsph_blend <= 0.05
    assert len({c.seed for c in cfgs}) == 256
    assert len({round(c.xsph_blend, 7) for c in cfgs}) > 200


def test_batched_steps_follow_each_box_tilt(fcu, wl):
    steps = wl.batched_frame_steps(fcu, 3, frames=2, substeps=4, seed=3)
    assert len(steps) == 8 and all(len(r) == 3 for r in steps)
    f = [tuple(steps[0][b].force) for b in range(3)]
    assert len(set(f)) == 3
    assert all(abs(np.linalg.norm(x) - 9.81) < 1e-4 for x in f)
    assert tuple(steps[0][1].force) == tuple(steps[3][1].force)
    assert tuple(steps[0][1].force) != tuple(steps[4][1].force)


def _create(fcu, cfgs):
    arr = (fcu.FluidSimConfig * len(cfgs))(*cfgs)
    h = fcu.lib().fluid_batch_create(arr, len(cfgs))
    return h, fcu.lib().fluid_last_error().decode()


def test_batch_refuses_mismatched_solves_tracers_and_empty(fcu, wl):
    cfgs = wl.batched_boxes(fcu, nboxes=3, lo=500, hi=1000)
    cfgs[2].den_tol = 0.002
    h, msg = _create(fcu, cfgs)
    assert not h and "box 2" in msg
    cfgs = wl.batched_boxes(fcu, nboxes=2, lo=500, hi=1000)
    cfgs[1].tracers = 16
    h, msg = _create(fcu, cfgs)
    assert not h and "tracers" in msg
    h = fcu.lib().fluid_batch_create(None, 0)
    assert not h
    assert fcu.lib().fluid_batch_boxes(None) == 0
    assert fcu.lib().fluid_batch_run(None, None, 0) == -1
