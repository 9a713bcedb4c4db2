"""The oracle's substep against the reference's headless solver tests.

The reference runs these against its GPU step (render.rs:5031-5275,
:5595-5651); here they pin the CPU restatement the CUDA path is checked by.
"""
import json
import os

import numpy as np
import pytest

KATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_kats.json")))
TB = KATS["test_box"]


def make_box_sim(orc, tracers=0):
    L = orc.lib()
    pos = orc.seed_slab(TB["spacing"], TB["extent"], 0.5)
    p = orc.params_slab(TB["extent"], TB["spacing"], 1.2, len(pos))
    s = orc.Sim(p, tracers)
    s.set_state(pos4=pos)
    return s, pos, p


def cpu_wall_density(t):
    t = np.float32(t)
    if t >= 2:
        return np.float32(0)
    t3 = t * t * t
    if t < 1:
        return np.float32(0.5) + t * np.float32(-0.7) + t3 * (np.float32(1.0 / 3.0) + t * t * (
            np.float32(-0.15) + t * np.float32(0.05)))
    return np.float32(8.0 / 15.0) + t * np.float32(-0.8) + t3 * (np.float32(2.0 / 3.0) + t * (
        np.float32(-0.5) + t * (np.float32(0.15) - t / np.float32(60.0))))


def kernel_np(r, h):
    q = (r / h).astype(np.float32)
    sigma = np.float32(1.0) / (np.float32(np.pi) * h * h * h)
    t = np.float32(2.0) - q
    return np.where(q < 1, sigma * (np.float32(1) - np.float32(1.5) * q * q * (np.float32(1) - np.float32(0.5) * q)),
                    np.where(q < 2, sigma * np.float32(0.25) * t * t * t, np.float32(0))).astype(np.float32)


# render.rs:5139-5214 (one_density_sweep_reads_near_rest_density), on the oracle
def test_one_density_sweep_reads_near_rest_density(orc):
    L = orc.lib()
    s, pos, p = make_box_sim(orc)
    s.substep(orc.make_step(dt=0.0, v_clamp=np.finfo(np.float32).max))
    f = s.stats()
    rho0 = np.float32(L.or_rest_density())
    assert f[0] == 0.0 and f[1] == 0.0
    assert 0.4 * rho0 < f[2] < f[3]
    assert 0.9 * rho0 < f[3] < 1.1 * rho0
    assert (f[4], f[5], f[6]) == (0.0, 0.0, 0.0)
    assert (f[7], f[8]) == (np.float32(293.15), np.float32(293.15))
    assert f[9] == 0.0
    h = np.float32(1.2) * np.float32(TB["spacing"])
    sp = np.float32(TB["spacing"])
    mass = rho0 * sp * sp * sp
    half = np.array([TB["extent"][0], TB["extent"][1], 0.5 * L.or_slab_depth()], np.float32)
    working = s.field("work_pos")
    density = s.field("density")
    for i in range(0, len(working), 16):
        pw = working[i, :3]
        d2 = np.sum((pw[None, :] - working[:, :3]) ** 2, axis=1, dtype=np.float32)
        pairs = np.sum(kernel_np(np.sqrt(d2), h), dtype=np.float32)
        tl = (pw + half) / h
        th = (half - pw) / h
        fill = np.float32(sum(cpu_wall_density(t) for t in list(tl) + list(th)))
        for a, b in [(0, 1), (0, 2), (1, 2)]:
            for ta, tb in [(tl[a], tl[b]), (tl[a], th[b]), (th[a], tl[b]), (th[a], th[b])]:
                fill -= np.float32(L.or_wedge64(float(ta), float(tb)))
        expect = mass * pairs + rho0 * fill
        assert abs(density[i] - expect) <= 1e-3 * expect, (i, density[i], expect)


# render.rs:5031-5135: the rebuild lands every particle in cell order and
# permutes the seed and nothing else.
def test_the_rebuild_lands_every_particle_in_cell_order(orc):
    s, pos, p = make_box_sim(orc)
    s.substep(orc.make_step(dt=0.0))
    starts = s.field("starts")
    working = s.field("work_pos")
    g = orc.OrGrid()
    g.min[:] = list(p.box_min)
    g.cell = p.cell
    g.dims[:] = list(p.dims)
    C = orc.cell_count(g)
    # a simulation's grid keys are cell * K + the x slab: cell c holds the
    # slots starts[c * K] .. starts[(c + 1) * K] - 1, in slab order
    K = orc.sim_slabs()
    assert len(starts) == C * K + 1 and starts[C * K] == p.count
    cs = starts[::K]
    keys, _, _ = orc.grid_build(g, working)
    for k, c in enumerate(keys):
        assert cs[c] <= k < cs[c + 1]
    held = np.bincount(keys, minlength=C)
    assert np.array_equal(held, np.diff(cs.astype(np.int64)))
    f32 = np.float32
    cx = keys % p.dims[0]
    off = working[:, 0] - (f32(p.box_min[0]) + cx.astype(f32) * f32(p.cell))
    slab = sum((off >= f32(p.cell) * (f32(k) / f32(K))).astype(np.int64) for k in range(1, K))
    skey = keys.astype(np.int64) * K + slab
    assert np.all(np.diff(skey) >= 0)
    for k, c in enumerate(skey):
        assert starts[c] <= k < starts[c + 1]
    a = np.sort(pos[:, :3].view(np.uint32), axis=0)
    b = np.sort(working[:, :3].view(np.uint32), axis=0)
    seeded = sorted(map(tuple, pos[:, :3].view(np.uint32)))
    landed = sorted(map(tuple, working[:, :3].view(np.uint32)))
    assert seeded == landed


# render.rs:5251-5275 (one_frame_of_the_solve_stays_physical), on the oracle
def test_one_frame_of_the_solve_stays_physical(orc):
    s, pos, p = make_box_sim(orc)
    dt = np.float32(1.0 / 120.0) / np.float32(7.0)
    v_clamp = np.float32(0.4) * np.float32(TB["spacing"]) / dt
    st = orc.make_step(force=(0, -9.81, 0), dt=float(dt), v_clamp=float(v_clamp))
    for _ in range(7):
        s.substep(st)
    f = s.stats()
    rho0 = np.float32(998.2)
    assert 0 < f[6] <= v_clamp * 1.001
    assert f[4] >= 0 and f[5] < 1.0e6
    assert abs(f[7] - 293.15) < 1e-3 and abs(f[8] - 293.15) < 1e-3
    assert f[3] < 2.0 * rho0


# The fixed schedule and the tolerance schedule agree when the tolerance
# schedule is forced to the fixed counts' behaviour; the tolerance loop
# meets its tolerance.
def test_tolerance_schedule_meets_its_tolerance(orc):
    s, pos, p = make_box_sim(orc)
    dt = np.float32(1.0 / 120.0) / np.float32(2.0)
    st = orc.make_step(force=(0, -9.81, 0), dt=float(dt),
                       v_clamp=float(np.float32(0.4) * np.float32(TB["spacing"]) / dt))
    for _ in range(20):
        iters, res = s.substep_tol(st, 0.01, 0.001, 100)
        assert iters[0] >= 1
        assert res[1] <= 0.001 or iters[1] == 100
        assert res[0] <= 0.01 or iters[0] == 100


def test_the_oracle_is_deterministic_across_thread_counts(orc):
    outs = []
    for threads in (1, 4):
        orc.set_threads(threads)
        s, pos, p = make_box_sim(orc)
        dt = np.float32(1.0 / 120.0) / np.float32(3.0)
        st = orc.make_step(force=(1.0, -9.81, 0.3), dt=float(dt), v_clamp=float(np.float32(0.4) * np.float32(TB["spacing"]) / dt),
                           omega=(0.1, 0.2, 0.5), domega=(0.0, 0.0, 1.0), touch_r=0.05,
                           touches=[(0.0, -0.2, 0.1, 0.0)])
        for _ in range(3):
            s.substep(st)
        outs.append(s.state())
    orc.set_threads(0)
    for k in outs[0]:
        assert np.array_equal(outs[0][k].view(np.uint32), outs[1][k].view(np.uint32)), k
