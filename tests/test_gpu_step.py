"""The CUDA substep against the CPU oracle, on the same seeded inputs.

The CUDA kernels and the oracle take the same operations in the same order
(IEEE binary32, no FMA contraction, neighbours in stencil order), so the
comparisons here are bit-for-bit: every field of the resting set after one
substep and after hundreds, the density sweep's outputs, the statistics and
the tracers. The reference's own GPU tests (render.rs:5031-5275,
:5595-5792) are ported alongside, on the CUDA path.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_kats.json")))
TB = KATS["test_box"]
F32 = np.float32


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def assert_same_bits(a, b, what):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, what
    ba, bb = bits(a), bits(b)
    bad = np.nonzero(ba != bb)
    if len(bad[0]):
        i = tuple(x[0] for x in bad)
        raise AssertionError(f"{what}: {len(bad[0])} words differ, first at {i}: "
                             f"{a[i]!r} vs {b[i]!r}")


def pair(fcu, orc, tracers=0, **kw):
    """A CUDA sim and an oracle sim on the CUDA sim's initial state."""
    sim = fcu.Sim(fcu.default_config(tracers=tracers, **kw))
    p = orc.OrParams()
    for name, _ in orc.OrParams._fields_:
        v = getattr(sim.params, name)
        if hasattr(v, "__len__"):
            getattr(p, name)[:] = list(v)
        else:
            setattr(p, name, v)
    o = orc.Sim(p, tracers)
    st = sim.state()
    o.set_state(st["pos"], st["vel"], st["prev_vel"], st["prev_p"], st["temp"], st["id"])
    if tracers:
        o.set_tracers(sim.tracers())
    return sim, o


def same_state(sim, o, what=""):
    a, b = sim.state(), o.state()
    for k in ("pos", "vel", "prev_vel", "prev_p", "temp", "id"):
        assert_same_bits(a[k], b[k], f"{what} {k}")


def step_pair(fcu, orc, **kw):
    return fcu.make_step(**kw), orc.make_step(**kw)


def frame_dt(substeps):
    return float(F32(1.0 / 120.0) / F32(substeps))


def v_clamp(spacing, dt):
    return float(F32(0.4) * F32(spacing) / F32(dt))


def test_params_match_the_oracle_derivation(fcu, orc):
    sim = fcu.Sim(fcu.default_config())
    p = orc.params_slab(TB["extent"], TB["spacing"], 1.2, sim.n)
    for name, _ in orc.OrParams._fields_:
        a, b = getattr(sim.params, name), getattr(p, name)
        if hasattr(a, "__len__"):
            assert list(a) == list(b), name
        elif name != "xsph_blend":
            assert a == b, name
    assert sim.n == TB["particles"] and sim.cells == TB["cells"]
    seed = orc.seed_slab(TB["spacing"], TB["extent"], 0.5)
    assert_same_bits(sim.state()["pos"], seed, "seed_slab")


def test_density_sweep_matches_the_oracle(fcu, orc):
    sim, o = pair(fcu, orc)
    s_g, s_o = step_pair(fcu, orc, dt=0.0, v_clamp=float(np.finfo(np.float32).max))
    sim.step(s_g)
    o.substep(s_o)
    for f in ("starts", "perm", "density", "alpha", "kd", "nbr_n", "wall_grad", "work_pos"):
        assert_same_bits(sim.field(f), o.field(f), f)
    sim.reduce_stats()
    assert_same_bits(sim.stats().as_reference_block(), o.stats(), "stats")


def test_one_substep_matches_the_oracle(fcu, orc):
    sim, o = pair(fcu, orc)
    dt = frame_dt(7)
    s_g, s_o = step_pair(fcu, orc, force=(0, -9.81, 0), dt=dt, v_clamp=v_clamp(TB["spacing"], dt))
    sim.step(s_g)
    o.substep(s_o)
    for f in ("density", "alpha", "kd", "pressure", "accel", "xsph", "work_vel"):
        assert_same_bits(sim.field(f), o.field(f), f)
    same_state(sim, o, "one substep")


# render.rs:5031-5135 on the CUDA path, then the same 60 frames on the
# oracle: the trajectories agree bit for bit.
def test_sixty_frames_match_the_oracle_and_records_travel_through_the_rebuild(fcu, orc):
    sim, o = pair(fcu, orc)
    dt = frame_dt(7)
    s_g, s_o = step_pair(fcu, orc, force=(0, -9.81, -0.5), dt=dt, v_clamp=v_clamp(TB["spacing"], dt))
    sim.run([s_g] * (60 * 7))
    for _ in range(60 * 7):
        o.substep(s_o)
    same_state(sim, o, "60 frames")
    rest = sim.state()
    xyz = {tuple(bits(p[:3])): i for i, p in enumerate(rest["pos"])}
    assert len(xyz) == sim.n, "two particles share a position"
    sim.step(fcu.make_step(dt=0.0))
    starts = sim.field("starts")
    work = sim.field("work_pos")
    assert starts[-1] == sim.n
    work_vel = sim.field("work_vel")
    for k, p in enumerate(work):
        i = xyz[tuple(bits(p[:3]))]
        assert bits(rest["vel"][i]).tolist() == bits(work_vel[k]).tolist()
    means = set(bits(rest["vel"][:, 3]).tolist())
    assert len(means) > sim.n // 2


def test_rotation_and_fingers_match_the_oracle(fcu, orc):
    sim, o = pair(fcu, orc)
    dt = frame_dt(3)
    kw = dict(force=(1.0, -9.81, 0.3), dt=dt, v_clamp=v_clamp(TB["spacing"], dt), omega=(0.1, 0.2, 0.5),
              domega=(0.0, 0.0, 1.0), touch_r=0.05, touches=[(0.0, -0.2, 0.1, 0.0), (0.05, -0.25, -0.1, 0.2)])
    s_g, s_o = step_pair(fcu, orc, **kw)
    sim.run([s_g] * 30)
    for _ in range(30):
        o.substep(s_o)
    same_state(sim, o, "rotation + fingers")


def test_stats_and_tracers_match_the_oracle(fcu, orc):
    sim, o = pair(fcu, orc, tracers=4096)
    dt = frame_dt(7)
    s_g, s_o = step_pair(fcu, orc, force=(-6.0, -9.81, 0), dt=dt, v_clamp=v_clamp(TB["spacing"], dt))
    for f in range(20):
        sim.run([s_g] * 7)
        for _ in range(7):
            o.substep(s_o)
        t_g, t_o = step_pair(fcu, orc, force=(-6.0, -9.81, 0), dt=float(F32(1.0 / 120.0)), seed=f)
        sim.tracers_pass(t_g)
        o.tracer_pass(t_o)
    sim.reduce_stats()
    assert_same_bits(sim.stats().as_reference_block(), o.stats(), "stats")
    assert np.array_equal(sim.tracers(), o.tracers())


def test_the_box_geometry_with_baseline_parameters_matches_the_oracle(fcu, orc):
    cfg = dict(geometry=fcu.GEOMETRY_BOX, box_lo=(0, 0, 0), box_hi=(1, 1, 1), spacing=0.01,
               h_ratio=1.0, rest_density=1000.0, seeding=fcu.SEED_BLOCK, block=(32, 16, 32),
               jitter=0.005, seed=1, xsph_blend=0.01)
    sim, o = pair(fcu, orc, **cfg)
    assert sim.params.xsph_blend == F32(0.01)
    seed = orc.seed_block([0, 0, 0], 0.01, [32, 16, 32], 0.005, 1)
    assert_same_bits(sim.state()["pos"], seed, "seed_block")
    dt = float(F32(1.0 / 120.0))
    s_g, s_o = step_pair(fcu, orc, force=(0, -9.81, 0), dt=dt, v_clamp=v_clamp(0.01, dt))
    sim.run([s_g] * 40)
    for _ in range(40):
        o.substep(s_o)
    same_state(sim, o, "box 40 steps")


# render.rs:5251-5275
def test_one_frame_of_the_solve_stays_physical(fcu):
    sim = fcu.Sim(fcu.default_config())
    dt = frame_dt(7)
    sim.run([fcu.make_step(force=(0, -9.81, 0), dt=dt, v_clamp=v_clamp(TB["spacing"], dt))] * 7)
    sim.reduce_stats()
    f = sim.stats().as_reference_block()
    vc = v_clamp(TB["spacing"], dt)
    assert 0 < f[6] <= vc * 1.001
    assert f[4] >= 0 and f[5] < 1e6
    assert abs(f[7] - 293.15) < 1e-3 and abs(f[8] - 293.15) < 1e-3
    assert f[3] < 2 * 998.2


# render.rs:5595-5651, :5716-5743
@pytest.mark.parametrize("name,gravity,frames", [("flat", (0, 0, -9.81), 120),
                                                  ("upright", (0, -9.81, 0), 1800),
                                                  ("corner", (-6.94, -6.94, 0), 1800)])
def test_long_runs_stay_bounded(fcu, name, gravity, frames):
    sim = fcu.Sim(fcu.default_config())
    dt = frame_dt(7)
    sim.run([fcu.make_step(force=gravity, dt=dt, v_clamp=v_clamp(TB["spacing"], dt))] * (7 * frames))
    sim.reduce_stats()
    f = sim.stats().as_reference_block()
    assert f[3] < 1.2 * 998.2, (name, f[3])
    assert f[6] < 1.0, (name, f[6])
    assert f[4] >= 0 and f[5] < 1e4, (name, f[4], f[5])
    if name == "flat":
        assert abs(f[7] - 293.15) < 1 and abs(f[8] - 293.15) < 1


def test_the_step_is_bit_reproducible(fcu):
    outs = []
    for _ in range(2):
        sim = fcu.Sim(fcu.default_config())
        dt = frame_dt(7)
        sim.run([fcu.make_step(force=(0, -9.81, -0.5), dt=dt, v_clamp=v_clamp(TB["spacing"], dt))] * 140)
        outs.append(sim.state())
    for k in outs[0]:
        assert_same_bits(outs[0][k], outs[1][k], k)


# The tolerance schedule: device-side loops stop on the exact FP64 residual,
# so iteration counts, residuals and states all match the oracle's loop.
@pytest.mark.parametrize("tols", [(0.01, 0.001), (0.002, 0.0002)])
def test_the_tolerance_schedule_matches_the_oracle(fcu, orc, tols):
    div_tol, den_tol = tols
    cfg = dict(geometry=fcu.GEOMETRY_BOX, box_lo=(0, 0, 0), box_hi=(0.4, 0.4, 0.4), spacing=0.01,
               h_ratio=1.0, rest_density=1000.0, seeding=fcu.SEED_BLOCK, block=(16, 12, 16),
               jitter=0.005, seed=3, xsph_blend=0.01, solve=fcu.SOLVE_TOLERANCE, div_tol=div_tol,
               den_tol=den_tol, max_iters=100)
    sim, o = pair(fcu, orc, **cfg)
    dt = float(F32(1.0 / 120.0))
    s_g, s_o = step_pair(fcu, orc, force=(0.5, -9.81, 0.2), dt=dt, v_clamp=v_clamp(0.01, dt))
    seen = set()
    for k in range(40):
        sim.step(s_g)
        iters, res = o.substep_tol(s_o, div_tol, den_tol, 100)
        st = sim.stats()
        assert (st.div_iters, st.den_iters) == (int(iters[0]), int(iters[1])), k
        assert st.div_residual == res[0] and st.den_residual == res[1], k
        assert st.den_residual <= den_tol or st.den_iters == 100
        seen.add(int(iters[1]))
    same_state(sim, o, "tolerance")
    assert len(seen) > 1, "the iteration count never varied"


# A list cap below the neighbour count (sim_solve.wgsl:384-388): every
# particle keeps its first cap neighbours for the later sweeps, the density
# sums still see all of them, and the overflow is counted.
def test_neighbour_overflow_matches_the_oracle(fcu, orc):
    sim, o = pair(fcu, orc, nbr_cap=20)
    dt = frame_dt(7)
    s_g, s_o = step_pair(fcu, orc, force=(0, -9.81, 0), dt=dt, v_clamp=v_clamp(TB["spacing"], dt))
    sim.run([s_g] * 5)
    for _ in range(5):
        o.substep(s_o)
    for f in ("density", "alpha", "nbr_n", "counters"):
        assert_same_bits(sim.field(f), o.field(f), f)
    assert sim.field("counters")[1] > 0
    same_state(sim, o, "overflow")


# A neighbour cap past the staged kernel's shared memory takes the
# single-pass density kernel; the answer is the same.
def test_a_large_neighbour_cap_matches_the_oracle(fcu, orc):
    sim, o = pair(fcu, orc, nbr_cap=300)
    dt = frame_dt(7)
    s_g, s_o = step_pair(fcu, orc, force=(0.3, -9.81, 0), dt=dt, v_clamp=v_clamp(TB["spacing"], dt))
    sim.run([s_g] * 5)
    for _ in range(5):
        o.substep(s_o)
    same_state(sim, o, "cap 300")


# Collisions: thousands of particles inside one cell (a stencil row longer
# than the staged kernel's 4,096-slot code span, and more neighbours than
# the cap) still match the oracle bit for bit.
def test_a_dense_clump_matches_the_oracle(fcu, orc):
    cfg = dict(geometry=fcu.GEOMETRY_BOX, box_lo=(0, 0, 0), box_hi=(0.2, 0.2, 0.2), spacing=0.01,
               h_ratio=1.0, rest_density=1000.0, seeding=fcu.SEED_NONE, count=5000, xsph_blend=0.01)
    sim, o = pair(fcu, orc, **cfg)
    rng = np.random.default_rng(11)
    pos = np.zeros((5000, 4), np.float32)
    pos[:, :3] = 0.1 + rng.uniform(-0.004, 0.004, (5000, 3))
    pos[:10, :3] = pos[10, :3]  # exact duplicates: r = 0 pairs
    sim.set_state(pos4=pos)
    o.set_state(pos4=pos)
    dt = float(F32(1.0 / 120.0) / F32(16.0))
    s_g, s_o = step_pair(fcu, orc, force=(0, -9.81, 0), dt=dt, v_clamp=v_clamp(0.01, dt))
    sim.step(s_g)
    o.substep(s_o)
    for f in ("density", "alpha", "nbr_n", "counters", "kd"):
        assert_same_bits(sim.field(f), o.field(f), f)
    same_state(sim, o, "clump")
