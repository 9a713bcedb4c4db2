"""The benchmarked workloads themselves against the oracle, bit for bit.

tilt_1m is built exactly as the benchmark builds it (box geometry, h = 1.2
spacing, tolerance solve with FP64 residuals, a seeded tilt per frame, 4,096
tracers, 1,048,576 particles) and advanced through fluid_sim_frame, the call
the benchmark times: after the benchmark's warm-up frames the GPU state and
tracers are copied into the oracle, and both take the next frames: the
substeps the reference's policy picks from the one-frame-stale v_max, each
a tolerance solve, then reduce_stats and a tracer pass. The substep counts,
the particle state, the tracers, the statistics block, the iteration counts
and the FP64 residuals must be identical. A frame at a fixed four substeps
is compared the same way.

dam_break_16k (16,384 particles, two substeps per 1/120 s frame, tolerance
solve) is run for ten frames from its initial lattice the same way and
compared after every frame.

Both are float32 paths with the same operation order on both sides, so the
tolerance is zero.
"""
import numpy as np
import pytest

from test_gpu_step import assert_same_bits

pytestmark = pytest.mark.gpu
F32 = np.float32


def oracle_of(orc, sim):
    p = orc.OrParams()
    for name, _ in orc.OrParams._fields_:
        v = getattr(sim.params, name)
        if hasattr(v, "__len__"):
            getattr(p, name)[:] = list(v)
        else:
            setattr(p, name, v)
    o = orc.Sim(p, sim.ntr)
    st = sim.state()
    o.set_state(st["pos"], st["vel"], st["prev_vel"], st["prev_p"], st["temp"], st["id"])
    if sim.ntr:
        o.set_tracers(sim.tracers())
    return o


def oracle_frame(orc, o, cfg, force, frame_dt, substeps, seed, tracers):
    """What fluid_sim_frame runs (csrc/sim.cu run_frame): `substeps` equal
    substeps of dt / substeps with the CFL clamp 0.4 spacing / dt_sub
    (render.rs:3171) and seed 0, then reduce_stats, then one tracer pass at
    the frame's dt with the frame's seed."""
    dt_sub = float(F32(frame_dt) / F32(substeps))
    vc = float(F32(0.4) * F32(cfg.spacing) / F32(dt_sub))
    st = orc.make_step(force=force, dt=dt_sub, v_clamp=vc)
    its = [o.substep_tol(st, cfg.div_tol, cfg.den_tol, cfg.max_iters) for _ in range(substeps)]
    stats = o.stats()
    if tracers:
        o.tracer_pass(orc.make_step(force=force, dt=float(F32(frame_dt)), seed=seed))
    return its, stats


class Before:
    """Cumulative counters before a frame, on both sides."""

    def __init__(self, sim, o):
        st = sim.stats()
        cnt = o.field("counters")
        self.clamp_count = st.clamp_count
        self.neighbour_overflow = st.neighbour_overflow
        self.total_div_iters = st.total_div_iters
        self.total_den_iters = st.total_den_iters
        self.o_clamps = int(cnt[0])
        self.o_over = int(cnt[1])


def compare_frame(sim, o, its, ostats, before, what):
    a, b = sim.state(), o.state()
    for k in ("pos", "vel", "prev_vel", "prev_p", "temp", "id"):
        assert_same_bits(a[k], b[k], f"{what} {k}")
    if sim.ntr:
        assert np.array_equal(sim.tracers(), o.tracers()), f"{what} tracers"
    after = sim.stats()
    block = after.as_reference_block()
    # slots 9 and 10 are cumulative counters; the oracle's start at the copy
    keep = [k for k in range(14) if k not in (9, 10)]
    assert_same_bits(block[keep], ostats[keep], f"{what} stats")
    assert after.clamp_count - before.clamp_count == int(ostats[9]) - before.o_clamps, what
    assert after.neighbour_overflow - before.neighbour_overflow == int(ostats[10]) - before.o_over
    n_div = sum(int(i[0]) for i, _ in its)
    n_den = sum(int(i[1]) for i, _ in its)
    assert after.total_div_iters - before.total_div_iters == n_div, what
    assert after.total_den_iters - before.total_den_iters == n_den, what
    assert (after.div_iters, after.den_iters) == (int(its[-1][0][0]), int(its[-1][0][1])), what
    assert after.div_residual == its[-1][1][0] and after.den_residual == its[-1][1][1], what
    return n_div, n_den


WARMUP_FRAMES = 5
CHECKED_FRAMES = 2


# The benchmark's frames: substeps_for on the one-frame-stale v_max
# (render.rs:3090-3094), a sync after every frame so the stale value is the
# previous frame's. The oracle side picks its count with its own restatement
# of the policy from its own statistics.
def test_tilt_1m_frames_match_the_oracle(fcu, orc, wl):
    cfg = wl.make_config(fcu, "tilt_1m")
    sim = fcu.Sim(cfg)
    assert sim.n == 1 << 20 and sim.ntr == 4096
    frames = WARMUP_FRAMES + CHECKED_FRAMES
    forces = wl.tilt_schedule(1, frames, 1.0 / 120.0)
    dt = float(F32(1.0 / 120.0))
    for k in range(WARMUP_FRAMES):
        sim.frame(tuple(float(x) for x in forces[k]), dt, substeps=0, cap=16, seed=k)
        sim.sync()
    o = oracle_of(orc, sim)
    v_max = sim.stats().v_max
    counts = []
    for k in range(WARMUP_FRAMES, frames):
        force = tuple(float(x) for x in forces[k])
        before = Before(sim, o)
        m = orc.substeps_for(dt, v_max, cfg.spacing, 16)
        sim.frame(force, dt, substeps=0, cap=16, seed=k)
        sim.sync()
        assert sim.stats().substeps_last_frame == m, (k, m)
        its, ostats = oracle_frame(orc, o, cfg, force, dt, m, k, True)
        compare_frame(sim, o, its, ostats, before, f"tilt_1m frame {k}")
        v_max = float(ostats[6])
        counts.append(m)
    # the tilt moves the fluid past the 4-substep floor's CFL speed
    assert max(counts) > 4, counts
    sim.close()


def test_tilt_1m_fixed_four_substep_frames_match_the_oracle(fcu, orc, wl):
    cfg = wl.make_config(fcu, "tilt_1m")
    sim = fcu.Sim(cfg)
    frames = WARMUP_FRAMES + 1
    forces = wl.tilt_schedule(1, frames, 1.0 / 120.0)
    dt = float(F32(1.0 / 120.0))
    for k in range(WARMUP_FRAMES):
        sim.frame(tuple(float(x) for x in forces[k]), dt, substeps=4, cap=16, seed=k)
    sim.sync()
    o = oracle_of(orc, sim)
    force = tuple(float(x) for x in forces[WARMUP_FRAMES])
    before = Before(sim, o)
    sim.frame(force, dt, substeps=4, cap=16, seed=WARMUP_FRAMES)
    its, ostats = oracle_frame(orc, o, cfg, force, dt, 4, WARMUP_FRAMES, True)
    d, e = compare_frame(sim, o, its, ostats, before, "tilt_1m fixed four")
    assert d >= 4 and e >= 8, (d, e)  # the solve really iterated
    sim.close()


def test_dam_break_16k_ten_frames_match_the_oracle(fcu, orc, wl):
    cfg = wl.make_config(fcu, "dam_break_16k")
    sim = fcu.Sim(cfg)
    assert sim.n == 16384
    o = oracle_of(orc, sim)
    dt = float(F32(1.0 / 120.0))
    force = (0.0, -9.81, 0.0)
    for k in range(10):
        before = Before(sim, o)
        sim.frame(force, dt, substeps=2, cap=16, seed=k)
        its, ostats = oracle_frame(orc, o, cfg, force, dt, 2, k, False)
        compare_frame(sim, o, its, ostats, before, f"dam_break_16k frame {k}")
    sim.close()


# bench.py --impl reference seeds the oracle itself (it runs no product
# code); it must start from the state fluid_sim_create makes.
def test_the_reference_arm_seeds_tilt_1m_as_the_product_does(fcu, orc, wl):
    w = wl.WORKLOADS["tilt_1m"]
    sim = fcu.Sim(wl.make_config(fcu, "tilt_1m"))
    lattice, spacing = list(w["lattice"]), w["spacing"]
    pos = orc.seed_block([0, 0, 0], spacing, lattice, 0.005, 1)
    p = orc.params_box([0, 0, 0], list(w["box_hi"]), spacing, 1.2, 1000.0, len(pos))
    p.xsph_blend = 0.01
    for name, _ in orc.OrParams._fields_:
        a, b = getattr(sim.params, name), getattr(p, name)
        assert (list(a) == list(b)) if hasattr(a, "__len__") else a == b, name
    assert_same_bits(sim.state()["pos"], pos, "seed_block")
    size = [float(F32(x) * F32(spacing)) for x in lattice]
    assert np.array_equal(sim.tracers(), orc.seed_tracers_box(w["tracers"], [0, 0, 0], size, p))
    sim.close()
