"""The render-side thickness field on the GPU: the body splat with the decay
draw and field_filter, against the oracle bit for bit, and the reference's
own calibration of the settled field (render.rs:5409-5430): the reference
test box settled for 600 frames of 7 substeps under (0, -9.81, -0.5), one
splat into a 32 x 64 field, its plateau (the median of the texels at or
above 0.6 of the peak, render.rs:5295-5300) within 10 % of FIELD_SETTLED =
5.3 (render.rs:532)."""
import numpy as np
import pytest

from test_gpu_step import assert_same_bits

pytestmark = pytest.mark.gpu

F32 = np.float32
FIELD_SETTLED = 5.3


def settled_sim(fcu, frames, gravity=(0.0, -9.81, -0.5), substeps=7):
    sim = fcu.Sim(fcu.default_config())
    dt = float(F32(1.0 / 120.0) / F32(substeps))
    vc = float(F32(0.4) * F32(sim.cfg.spacing) / F32(dt))
    step = fcu.make_step(force=gravity, dt=dt, v_clamp=vc)
    sim.run([step] * (frames * substeps))
    return sim


def oracle_field(orc, sim, w, h, keep, lens, lo, hi, prev):
    st = sim.state()
    p = sim.params
    geom = [p.tracer_c[0], p.tracer_c[1], p.tracer_e[0], p.tracer_e[1], F32(p.h) * F32(1.5), lo, hi]
    return orc.field_splat(st["pos"], st["vel"], st["prev_vel"], sim.field("density"), geom, w, h, lens,
                           keep, prev)


def test_splat_decay_and_filter_match_the_oracle(fcu, orc):
    sim = settled_sim(fcu, 30)
    p = sim.params
    w, h = 48, 96
    # a fresh splat with the speed lens, then a decayed one with the
    # density lens, then the filter
    sim.field_splat(w, h, keep=0.0, lens=4, lo=0.0, hi=0.5)
    f1, _ = sim.field_read()
    o1 = oracle_field(orc, sim, w, h, 0.0, 4, 0.0, 0.5, None)
    assert_same_bits(f1, o1, "fresh splat")
    assert f1[..., 0].max() > 1.0 and f1[..., 1].max() > 0.0
    step = fcu.make_step(force=(0.0, -9.81, 0.0), dt=float(F32(1.0 / 120.0) / F32(7)),
                         v_clamp=float(F32(0.4) * F32(0.01) / (F32(1.0 / 120.0) / F32(7))))
    sim.run([step] * 7)
    sim.field_splat(w, h, keep=0.8, lens=3, lo=500.0, hi=1000.0)
    sim.field_filter()
    f2, filt = sim.field_read()
    o2 = oracle_field(orc, sim, w, h, 0.8, 3, 500.0, 1000.0, o1)
    assert_same_bits(f2, o2, "decayed splat")
    assert_same_bits(filt, orc.field_filter(o2, p.tracer_e[0], p.tracer_e[1]), "filter")


def test_the_settled_field_matches_the_calibration(fcu):
    sim = settled_sim(fcu, 600)
    sim.reduce_stats()
    st = sim.stats()
    assert st.v_max < 0.2, f"not settled: v_max {st.v_max}"
    sim.field_splat(32, 64, keep=0.0)
    f, _ = sim.field_read()
    vals = f[..., 0].ravel()
    peak = vals.max()
    interior = np.sort(vals[vals >= 0.6 * peak])
    plateau = interior[len(interior) // 2]
    print(f"settled field: plateau {plateau:.3f}, max {peak:.3f}")
    assert abs(plateau / FIELD_SETTLED - 1.0) < 0.1, plateau
