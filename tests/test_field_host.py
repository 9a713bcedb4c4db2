"""The thickness field's host-side pieces and the oracle's restatement of
the body splat and field_filter, without a GPU."""
import math

import numpy as np


def test_keep_target_follows_the_reference_curve(fcu):
    # render.rs:1107-1111: FIELD_KEEP (0.8) times one minus a smoothstep
    # over v_max in [0.05, 0.25].
    L = fcu.lib()
    for v, want in [(0.0, 0.8), (0.05, 0.8), (0.15, 0.4), (0.25, 0.0), (3.0, 0.0)]:
        assert abs(L.fluid_field_keep_target(v) - want) < 1e-6, v
    t = (0.1 - 0.05) / 0.2
    assert abs(L.fluid_field_keep_target(0.1) - 0.8 * (1 - t * t * (3 - 2 * t))) < 1e-6


def test_one_splat_integrates_to_the_kernel_volume(orc):
    # A lone particle at the field's centre: the falloff (1 - |c|^2)^2 / 2
    # integrates to pi/6 over the unit quad's disc, times the disc's area in
    # texels; the texel sum is its midpoint-rule estimate.
    w, h = 256, 256
    geom = [0.0, 0.0, 1.0, 1.0, 0.1, 0.0, 1.0]  # centre, half extents, radius, lens ramp
    pos = np.array([[0.0, 0.0, 0.0, 0.0]], np.float32)
    f = orc.field_splat(pos, pos, pos, np.ones(1, np.float32), geom, w, h, 0, 0.0)
    r_tex = 0.1 * w / 2
    assert abs(f[..., 0].sum() / (math.pi / 6 * r_tex * r_tex) - 1) < 1e-3
    assert np.array_equal(f[..., 0], f[::-1, ::-1, 0])  # symmetric about the centre
    assert np.all(f[..., 1] == 0)


def test_decay_and_lens_channel(orc):
    w, h = 64, 64
    geom = [0.0, 0.0, 1.0, 1.0, 0.2, 0.0, 2.0]
    pos = np.array([[0.1, -0.2, 0.0, 0.0]], np.float32)
    vel = np.array([[1.0, 0.0, 0.0, 0.5]], np.float32)  # speed 1, accel lens 0.5
    one = orc.field_splat(pos, vel, vel, np.ones(1, np.float32), geom, w, h, 4, 0.0)
    # the speed lens at 1 on a 0..2 ramp halves the weight in g
    assert np.allclose(one[..., 1], 0.5 * one[..., 0], rtol=1e-6, atol=1e-6)
    again = orc.field_splat(pos, vel, vel, np.ones(1, np.float32), geom, w, h, 4, 0.8, one)
    # steady state of keep * f + (1 - keep) * s from f = s is s
    assert np.allclose(again, one, rtol=1e-6, atol=1e-7)


def test_filter_keeps_constants_and_reads_slopes(orc):
    w, h = 40, 24
    const = np.full((h, w, 2), 3.0, np.float32)
    out = orc.field_filter(const, 1.0, 1.0)
    assert np.allclose(out[..., 0], 3.0, atol=1e-6)
    assert np.allclose(out[..., 1:], 0.0, atol=1e-5)
    ramp = np.zeros((h, w, 2), np.float32)
    ramp[..., 0] = np.arange(w, dtype=np.float32)[None, :] * 0.5
    out = orc.field_filter(ramp, 1.0, 1.0)
    inner = out[:, 5:w - 5]
    assert np.allclose(inner[..., 0], ramp[:, 5:w - 5, 0], atol=1e-5)  # the blur keeps a line
    assert np.allclose(inner[..., 1], 1.0, atol=1e-5)                  # x difference: 2 * slope
    assert np.allclose(inner[..., 2], 0.0, atol=1e-6)
