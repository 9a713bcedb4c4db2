"""Batched boxes against the oracle, box by box.

A batch steps boxes of uneven sizes, each with its own XSPH coefficient,
jitter stream and tilt sequence, with every kernel launch covering all of
them. Each box must follow, bit for bit, the oracle run of that box alone:
the resting set after every checkpoint, and in the tolerance mode each
box's own iteration counts and FP64 residuals every substep (boxes stop
their loops independently).
"""
import numpy as np
import pytest

from test_gpu_step import assert_same_bits

pytestmark = pytest.mark.gpu


def oracle_twin(orc, batch, box):
    p = orc.OrParams()
    src = batch.params(box)
    for name, _ in orc.OrParams._fields_:
        v = getattr(src, name)
        if hasattr(v, "__len__"):
            getattr(p, name)[:] = list(v)
        else:
            setattr(p, name, v)
    o = orc.Sim(p, 0)
    st = batch.state(box)
    o.set_state(st["pos"], st["vel"], st["prev_vel"], st["prev_p"], st["temp"], st["id"])
    return o


def same_box(batch, o, box, what):
    a, b = batch.state(box), o.state()
    for k in ("pos", "vel", "prev_vel", "prev_p", "temp", "id"):
        assert_same_bits(a[k], b[k], f"{what} box {box} {k}")


def small_boxes(fcu, wl, nboxes, **kw):
    # counts 500..7000 keep the oracle fast; the construction is the batched
    # workload's (log-uniform counts, per-box XSPH, seeds and tilts)
    return wl.batched_boxes(fcu, nboxes=nboxes, seed=5, lo=500, hi=7000, **kw)


def to_oracle_step(orc, st):
    return orc.make_step(force=tuple(st.force), dt=st.dt, v_clamp=st.v_clamp, seed=st.seed)


def test_batched_tolerance_boxes_match_the_oracle_box_by_box(fcu, orc, wl):
    nb = 5
    cfgs = small_boxes(fcu, wl, nb)
    batch = fcu.Batch(cfgs)
    assert len(set(batch.counts)) >= 4  # 4000, 4000, 2048, 864, 500
    twins = [oracle_twin(orc, batch, b) for b in range(nb)]
    steps = wl.batched_frame_steps(fcu, nb, frames=6, substeps=4, seed=5)
    per_box_iters = [set() for _ in range(nb)]
    for k, row in enumerate(steps):
        batch.step(row)
        stats = batch.stats()
        for b in range(nb):
            iters, res = twins[b].substep_tol(to_oracle_step(orc, row[b]), 0.01, 0.001, 100)
            assert (stats[b].div_iters, stats[b].den_iters) == (int(iters[0]), int(iters[1])), (k, b)
            assert stats[b].div_residual == res[0] and stats[b].den_residual == res[1], (k, b)
            per_box_iters[b].add(int(iters[1]))
    for b in range(nb):
        same_box(batch, twins[b], b, "tolerance")
    # the boxes did not all take the same iterations
    assert len(set(frozenset(s) for s in per_box_iters)) > 1


def test_batched_fixed_schedule_matches_the_oracle_and_stats(fcu, orc, wl):
    nb = 4
    cfgs = small_boxes(fcu, wl, nb, solve=fcu.SOLVE_FIXED, div_iters=2, den_iters=3)
    batch = fcu.Batch(cfgs)
    twins = [oracle_twin(orc, batch, b) for b in range(nb)]
    steps = wl.batched_frame_steps(fcu, nb, frames=5, substeps=4, seed=6)
    batch.run(steps)
    for row in steps:
        for b in range(nb):
            twins[b].substep(to_oracle_step(orc, row[b]), 2, 3)
    for b in range(nb):
        same_box(batch, twins[b], b, "fixed")
    batch.reduce_stats()
    stats = batch.stats()
    for b in range(nb):
        o = twins[b].stats()
        assert stats[b].substeps == len(steps)
        assert stats[b].compression_avg == np.float32(o[0]), b
        assert stats[b].compression_max == np.float32(o[1]), b
        assert stats[b].density_min == np.float32(o[2]) and stats[b].density_max == np.float32(o[3]), b


def test_block_sizes_and_the_autotuner_change_no_bit(fcu, wl):
    # The sweeps' block size only regroups threads: every box stays
    # bit-identical at 64, 128 and 256 threads, and the autotuner's timed
    # substeps leave the batch where it was.
    nb = 4
    cfgs = small_boxes(fcu, wl, nb)
    steps = wl.batched_frame_steps(fcu, nb, frames=3, substeps=4, seed=9)
    ref = fcu.Batch(cfgs)
    ref.run(steps)
    for tpb in (64, 256):
        other = fcu.Batch(cfgs)
        other.set_blocks([tpb] * 7)
        assert list(other.blocks()) == [tpb] * 7
        other.run(steps)
        for b in range(nb):
            a, c = ref.state(b), other.state(b)
            for k in ("pos", "vel", "prev_vel", "prev_p", "temp", "id"):
                assert_same_bits(a[k], c[k], f"{tpb} threads box {b} {k}")
    tuned = fcu.Batch(cfgs)
    tuned.run(steps[:4])
    before = [tuned.state(b) for b in range(nb)]
    chosen, ms = tuned.autotune(steps[4])
    assert set(chosen.values()) <= {64, 128, 256} and np.all(ms > 0)
    for b in range(nb):
        after = tuned.state(b)
        for k in ("pos", "vel", "prev_vel", "prev_p", "temp", "id"):
            assert_same_bits(before[b][k], after[k], f"autotune restores box {b} {k}")
    assert tuned.stats()[0].substeps == 4
    tuned.run(steps[4:])
    for b in range(nb):
        a, c = ref.state(b), tuned.state(b)
        for k in ("pos", "vel", "prev_vel", "prev_p", "temp", "id"):
            assert_same_bits(a[k], c[k], f"tuned box {b} {k}")


def test_a_batch_of_one_is_the_one_box_simulation(fcu, wl):
    cfg = small_boxes(fcu, wl, 1)[0]
    batch = fcu.Batch([cfg])
    sim = fcu.Sim(cfg)
    steps = wl.batched_frame_steps(fcu, 1, frames=4, substeps=4, seed=7)
    batch.run(steps)
    sim.run([row[0] for row in steps])
    a, b = batch.state(0), sim.state()
    for k in ("pos", "vel", "prev_vel", "prev_p", "temp", "id"):
        assert_same_bits(a[k], b[k], k)
    sb, ss = batch.stats()[0], sim.stats()
    assert (sb.total_div_iters, sb.total_den_iters) == (ss.total_div_iters, ss.total_den_iters)
