"""The frame controller around the step, host only (no GPU).

Ports the reference's controller tests (crates/fluid-core/src/render.rs:
3583-3728) and MotionSample's body-force tests (crates/fluid-core/src/lib.rs:
43-72) against libfluidcu's controller (fluid_controller_*, fluid_substeps_for,
fluid_idle_gate_*).
"""
import ctypes as C
import json
import os

import numpy as np

KATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_kats.json")))
F32 = np.float32


class Gate:
    def __init__(self, fcu):
        self.L = fcu.lib()
        self.h = self.L.fluid_idle_gate_create()

    def __del__(self):
        self.L.fluid_idle_gate_destroy(self.h)

    def asleep(self, touched, smooth, dev, omega, v_max):
        s = (C.c_float * 3)(*smooth)
        o = (C.c_float * 3)(*omega)
        return bool(self.L.fluid_idle_gate_asleep(self.h, 1 if touched else 0, C.byref(s), dev,
                                                   C.byref(o), v_max))


# render.rs:3582-3605
def test_idle_gate_sleeps_when_still_and_wakes_on_shake_or_tilt(fcu):
    g = 9.81
    still = [0.0, 0.0, 0.0]
    upright = [0.0, -g, 0.0]
    gate = Gate(fcu)
    frames = fcu.lib().fluid_idle_gate_still_frames()
    assert frames == 180
    for _ in range(frames - 1):
        assert not gate.asleep(False, upright, 0.1, still, 0.03)
    assert gate.asleep(False, upright, 0.1, still, 0.03)
    assert gate.asleep(False, upright, 0.8, still, 0.03)
    assert not gate.asleep(False, upright, 2.0, still, 0.03)
    for _ in range(frames):
        gate.asleep(False, upright, 0.1, still, 0.03)
    assert gate.asleep(False, upright, 0.1, still, 0.03)
    assert not gate.asleep(False, [g * 0.05, -g, 0.0], 0.1, still, 0.03)


# render.rs:3610-3631
def test_idle_gate_wakes_on_pure_rotation(fcu):
    flat = [0.0, 0.0, -9.81]
    gate = Gate(fcu)
    for _ in range(180):
        gate.asleep(False, flat, 0.1, [0.0, 0.0, 0.0], 0.03)
    assert gate.asleep(False, flat, 0.1, [0.0, 0.0, 0.01], 0.03), "gyro noise"
    assert not gate.asleep(False, flat, 0.1, [0.0, 0.0, 0.5], 0.03), "a real turn"
    spun = Gate(fcu)
    for _ in range(2 * 180):
        assert not spun.asleep(False, flat, 0.1, [0.0, 0.0, 0.5], 0.03)


def test_a_touch_keeps_the_gate_awake(fcu):
    gate = Gate(fcu)
    for _ in range(400):
        assert not gate.asleep(True, [0, -9.81, 0], 0.0, [0, 0, 0], 0.0)


# render.rs:3635-3656: the drawable's top right is the box's
def test_the_fingers_map_drawable_points_into_the_box(fcu):
    ctl = fcu.Controller(0.01, [0.1, 0.2])
    ctl.touch(0, 1.0, 0.0, True)
    p = ctl.plan([0, -1, 0], now_ms=0.0)
    assert p.step.touch_n == 1
    assert (F32(p.step.touches[0][0]), F32(p.step.touches[0][1])) == (F32(0.1), F32(0.2))
    assert (p.step.touches[0][2], p.step.touches[0][3]) == (0.0, 0.0), "one sample makes no speed"
    assert p.step.touch_r > 0
    ctl.touch(0, 0.0, 0.0, False)
    p = ctl.plan([0, -1, 0], now_ms=1000.0 / 120.0)
    assert p.step.touch_n == 0, "lifted"


# render.rs:3662-3692
def test_a_lifted_finger_leaves_the_others_where_they_were(fcu):
    ctl = fcu.Controller(0.01, [0.1, 0.2])
    velocity = None
    t = 0.0
    for f in range(60):
        ctl.touch(0, 0.9, 0.9, True)
        ctl.touch(2, 0.2 + 0.01 * f, 0.5, True)
        p = ctl.plan([0, -1, 0], now_ms=t)
        t += 1000.0 / 120.0
        assert p.step.touch_n == 2
        velocity = (p.step.touches[1][2], p.step.touches[1][3])
    assert abs(velocity[0] - 0.24) < 0.005 and velocity[1] == 0.0
    ctl.touch(0, 0.0, 0.0, False)
    ctl.touch(2, 0.2 + 0.01 * 60.0, 0.5, True)
    p = ctl.plan([0, -1, 0], now_ms=t)
    assert p.step.touch_n == 1
    assert abs(p.step.touches[0][2] - 0.24) < 0.005


def v_for_cfl(count, dt, spacing):
    return (F32(count) - F32(0.5)) * F32(0.4) * F32(spacing) / F32(dt)


# render.rs:3696-3728
def test_the_substep_floor_scales_with_the_spacing(fcu):
    L = fcu.lib()
    for dt, spacing, expect in KATS["substeps_for"]["substep_floor"]:
        assert L.fluid_substep_floor(float(F32(dt)), float(F32(0.42) * F32(spacing))) == expect


def test_a_120hz_frame_jumps_six_or_seven_substeps_to_eight(fcu):
    nominal = float(F32(1.0) / F32(120.0))
    counts = [fcu.substeps_for(nominal, float(v_for_cfl(k, nominal, 0.01)), 0.01, 16) for k in range(5, 10)]
    assert counts == KATS["substeps_for"]["jump_counts_5_to_9"]


def test_a_120hz_frame_at_4x_floors_at_four_then_jumps_under_handling(fcu):
    nominal = float(F32(1.0) / F32(120.0))
    n = lambda v: fcu.substeps_for(nominal, float(v), 0.0062, 16)
    assert n(v_for_cfl(1, nominal, 0.0062)) == 4
    assert n(v_for_cfl(6, nominal, 0.0062)) == 8


def test_a_slipped_frame_keeps_its_cfl_count(fcu):
    dt = 0.010
    assert fcu.substeps_for(dt, float(v_for_cfl(7, dt, 0.01)), 0.01, 16) == 7


def test_a_flung_frame_stops_at_the_cap(fcu):
    assert fcu.substeps_for(float(F32(1.0) / F32(120.0)), 1.0e6, 0.01, 16) == 16


# lib.rs:43-72, through the controller's first frame (the filter starts at
# the raw body force)
def test_body_force_is_the_accelerometer_in_si(fcu):
    g = 9.80665
    cases = [([0, 0, -1], [0, 0, 0], [0, 0, -g]), ([0, 0, -1], [-0.5, 0, 0], None),
             ([0, 0, -1], [0, 0, 1], [0, 0, 0])]
    for grav, acc, expect in cases:
        ctl = fcu.Controller(0.01, [0.1, 0.2])
        p = ctl.plan(grav, acc, now_ms=0.0)
        f = [p.force.x, p.force.y, p.force.z]
        if expect is None:
            assert f[0] == F32(F32(-0.5) * F32(g))
        else:
            assert f == [float(F32(v)) for v in expect]


def test_the_first_frame_and_a_pause_encode_no_solve(fcu):
    ctl = fcu.Controller(0.01, [0.1, 0.2])
    p = ctl.plan([0, -1, 0], now_ms=100.0)
    assert p.dt == 0.0 and p.substeps == 0
    p = ctl.plan([0, -1, 0], now_ms=100.0 + 1000.0 / 120.0)
    assert p.dt > 0 and p.substeps >= 2
    p = ctl.plan([0, -1, 0], now_ms=100.0 + 1000.0 / 120.0 + 2000.0)
    assert abs(p.dt - 1.0 / 30.0) < 1e-7, "MAX_DT clamps a resume"
    assert abs(p.step.v_clamp - 0.4 * 0.01 / p.step.dt) < 1e-3


# The oracle's restatement of the substep policy (the benchmark's reference
# arm picks its substeps with it) agrees with the product's.
def test_the_oracle_substep_policy_agrees_with_the_product(fcu, orc):
    rng = np.random.default_rng(9)
    dts = [float(F32(1.0) / F32(120.0)), float(F32(1.0) / F32(60.0)), 0.01, 0.004]
    for dt in dts:
        for spacing in (0.005, 0.0062, 0.01):
            for v in np.concatenate([rng.uniform(0.0, 5.0, 200), [0.0, 1e6, np.inf]]):
                v = float(F32(v))
                assert orc.substeps_for(dt, v, spacing, 16) == fcu.substeps_for(dt, v, spacing, 16), \
                    (dt, spacing, v)
