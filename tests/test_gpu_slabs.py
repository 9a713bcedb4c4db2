"""The x-slab cell order against the oracle at its edges.

A simulation's grid keys are cell * slabs + the x slab of the particle in
its cell, and density_div cuts each stencil row to the slabs within the
support's half-chord in x. Here the particles' x coordinates sit on and
next to the slab and cell boundaries (a few ulps either side), at the box's
faces and outside them (saturated cells), with y and z anywhere in the box.
After one substep the GPU and the oracle (which scans whole cells) must
agree bit for bit, and every particle's neighbour count must equal a
brute-force count over all pairs.
"""
import numpy as np
import pytest

from test_gpu_step import assert_same_bits, pair, same_state, step_pair, v_clamp

pytestmark = pytest.mark.gpu
F32 = np.float32


def edge_positions(p, count, seed):
    rng = np.random.default_rng(seed)
    lo = np.array(p.box_min, F32)
    cell = F32(p.cell)
    dims = np.array(p.dims)
    K = 4
    pos = np.zeros((count, 4), F32)
    hi = lo + dims.astype(F32) * cell
    for a in (1, 2):
        pos[:, a] = rng.uniform(lo[a], lo[a] + F32(0.9) * (hi[a] - lo[a]), count).astype(F32)
    cx = rng.integers(0, dims[0], count)
    k = rng.integers(0, K, count)
    base = lo[0] + cx.astype(F32) * cell
    x = base + cell * (k.astype(F32) / F32(K))
    # a few ulps below or above the boundary, or on it
    steps = rng.integers(-3, 4, count)
    for s in range(1, 4):
        x = np.where(steps >= s, np.nextafter(x, F32(np.inf)), x)
        x = np.where(steps <= -s, np.nextafter(x, F32(-np.inf)), x)
    pos[:, 0] = x
    # some just outside the box's x faces (saturated cells)
    out = rng.random(count) < 0.02
    side = rng.random(count) < 0.5
    d = rng.uniform(0.0, 0.3, count).astype(F32) * cell
    pos[out & side, 0] = (lo[0] - d)[out & side]
    pos[out & ~side, 0] = (lo[0] + dims[0] * cell + d)[out & ~side]
    return pos


def brute_counts(work_pos, support_sq, cap):
    x = work_pos[:, :3]
    out = np.zeros(len(x), np.int64)
    for c in range(0, len(x), 256):
        d = x[c:c + 256, None, :] - x[None, :, :]
        r2 = d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]
        r2 = r2 + d[..., 2] * d[..., 2]
        out[c:c + 256] = (r2 < F32(support_sq)).sum(1) - 1
    return np.minimum(out, cap)


@pytest.mark.parametrize("seed", [1, 2])
def test_slab_and_cell_boundaries_match_the_oracle(fcu, orc, seed):
    assert fcu.grid_slabs() == orc.sim_slabs() == 4
    n = 12000
    cfg = dict(geometry=fcu.GEOMETRY_BOX, box_lo=(0, 0, 0), box_hi=(0.24, 0.24, 0.24), spacing=0.01,
               h_ratio=1.2, rest_density=1000.0, seeding=fcu.SEED_NONE, count=n, xsph_blend=0.01)
    sim, o = pair(fcu, orc, **cfg)
    pos = edge_positions(sim.params, n, seed)
    sim.set_state(pos4=pos)
    o.set_state(pos4=pos)
    dt = float(F32(1.0 / 120.0) / F32(8.0))
    s_g, s_o = step_pair(fcu, orc, force=(0, -9.81, 0), dt=dt, v_clamp=v_clamp(0.01, dt))
    sim.step(s_g)
    o.substep(s_o)
    for f in ("starts", "perm", "density", "alpha", "kd", "nbr_n", "counters", "work_pos"):
        assert_same_bits(sim.field(f), o.field(f), f)
    same_state(sim, o, f"slab edges {seed}")
    got = sim.field("nbr_n").astype(np.int64)
    want = brute_counts(sim.field("work_pos"), sim.params.support_sq, sim.cfg.nbr_cap)
    assert np.array_equal(got, want)
    assert got.mean() > 20  # the sweep really found neighbours (~31)
    sim.close()
