"""Pins the CPU oracle to the reference's own known-answer tests.

Each test restates one `#[test]` of the reference (file:line given) against
the oracle's restatement of the same function. The reference ships no golden
vector files; its tests generate their fixtures (seed_slab, TEST_EXTENT) and
assert closed-form or quadrature values, which is what is ported here.
"""
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_kats.json")


def kats():
    with open(GOLDEN) as f:
        return json.load(f)


def k_f32(lib, r, h):
    return np.float32(lib.or_kernel(float(r), float(h)))


# sim.rs:358-373
def test_the_kernel_integrates_to_one(orc):
    L = orc.lib()
    h = np.float32(0.004)
    step = np.float32(h / np.float32(20.0))
    n = int(np.float32(2.0) * h / step) + 1
    ii = np.arange(-n, n + 1)
    s = (ii[:, None, None] ** 2 + ii[None, :, None] ** 2 + ii[None, None, :] ** 2).ravel()
    uniq, mult = np.unique(s, return_counts=True)
    total = 0.0
    for v, m in zip(uniq, mult):
        r = np.float32(np.sqrt(np.float32(v))) * step
        total += m * float(k_f32(L, r, h)) * float(step) ** 3
    assert abs(total - 1.0) < 0.01, total


# sim.rs:375-393
def test_a_lattice_at_spacing_d_recovers_rest_density(orc):
    L = orc.lib()
    rho0 = np.float32(L.or_rest_density())
    d = np.float32(0.002)
    h = np.float32(1.2) * d
    mass = rho0 * d * d * d
    rho = np.float32(0.0)
    for ix in range(-3, 4):
        for iy in range(-3, 4):
            for iz in range(-3, 4):
                r = np.float32(np.sqrt(np.float32(ix * ix + iy * iy + iz * iz))) * d
                rho = np.float32(rho + mass * k_f32(L, r, h))
    err = abs(rho - rho0) / rho0
    assert err < 0.02, (rho, err)


EXTENT = [0.0356, 0.077]


# sim.rs:395-405
def test_every_seeded_particle_lands_in_a_valid_cell(orc):
    L = orc.lib()
    g = orc.grid_slab(EXTENT, 0.0048)
    pts = orc.seed_slab(0.002, EXTENT, 0.5)
    assert len(pts) > 0
    e = np.float32(EXTENT)
    assert np.all(np.abs(pts[:, 0]) <= e[0]) and np.all(np.abs(pts[:, 1]) <= e[1])
    assert np.all(np.abs(pts[:, 2]) <= np.float32(L.or_slab_depth()) * np.float32(0.5))
    keys, starts, perm = orc.grid_build(g, pts)
    assert np.all(keys < orc.cell_count(g))


# sim.rs:407-416
def test_neighbouring_positions_map_to_adjacent_cells(orc):
    L = orc.lib()
    g = orc.grid_slab(EXTENT, 0.0048)
    cell = lambda p: L.or_cell_of(g, orc.f32(p))
    a = cell([0, 0, 0])
    assert cell([g.cell, 0, 0]) == a + 1
    assert cell([0, g.cell, 0]) == a + g.dims[0]


def wall_quadrature(d, gradient):
    # sim.rs:419-429, in FP64 (the reference sums in f32; FP64 is the
    # stricter check of the polynomial)
    n = 20000
    dr = (2.0 - d) / n
    r = d + (np.arange(n) + 0.5) * dr
    q = r
    w = np.where(q < 1, 1 - 1.5 * q * q * (1 - 0.5 * q), np.where(q < 2, 0.25 * (2 - q) ** 3, 0.0))
    w /= np.pi
    cap = 1.0 if gradient else (r - d)
    return float(np.sum(w * 2 * np.pi * r * cap * dr))


# sim.rs:431-446, against the shader copies (sim_solve.wgsl:213-235)
def test_wall_integrals_match_quadrature(orc):
    L = orc.lib()
    for i in range(40):
        d = float(np.float32(i) * np.float32(0.05))
        assert abs(L.or_wall_density(d) - wall_quadrature(d, False)) < 1e-4, d
        assert abs(L.or_wall_gradient(d) - wall_quadrature(d, True)) < 1e-4, d
    assert L.or_wall_density(2.0) == 0.0
    assert L.or_wall_gradient(2.0) == 0.0


def cpu_wall_density(t):
    # sim.rs:261-272, the CPU association of the same polynomial
    t = np.float32(t)
    if t >= 2:
        return np.float32(0)
    t3 = t * t * t
    if t < 1:
        return np.float32(0.5) + t * np.float32(-0.7) + t3 * (np.float32(1.0 / 3.0) + t * t * (
            np.float32(-0.15) + t * np.float32(0.05)))
    return np.float32(8.0 / 15.0) + t * np.float32(-0.8) + t3 * (np.float32(2.0 / 3.0) + t * (
        np.float32(-0.5) + t * (np.float32(0.15) - t / np.float32(60.0))))


def test_shader_and_cpu_wall_density_agree(orc):
    L = orc.lib()
    for t in np.linspace(0, 2.2, 111, dtype=np.float32):
        assert abs(L.or_wall_density(float(t)) - float(cpu_wall_density(t))) <= 2e-7


# sim.rs:453-483
def test_the_wall_term_closes_the_half_lattice_gap(orc):
    L = orc.lib()
    rho0 = np.float32(L.or_rest_density())
    d = np.float32(0.0025)
    h = np.float32(1.2) * d
    mass = rho0 * d * d * d
    for layer in range(4):
        z0 = (np.float32(layer) + np.float32(0.5)) * d
        half = np.float32(0)
        bulk = np.float32(0)
        for x in range(-3, 4):
            for y in range(-3, 4):
                for z in range(-6, 7):
                    dx, dy = np.float32(x) * d, np.float32(y) * d
                    dz = (np.float32(z) + np.float32(0.5)) * d - z0
                    w = mass * k_f32(L, np.sqrt(np.float32(dx * dx + dy * dy + dz * dz)), h)
                    bulk = np.float32(bulk + w)
                    if z >= 0:
                        half = np.float32(half + w)
        err = (half + rho0 * np.float32(L.or_wall_density(float(z0 / h))) - bulk) / bulk
        assert abs(err) < 0.03, (layer, err)


# sim.rs:485-494
def test_tracers_seed_inside_the_fluid_region(orc):
    L = orc.lib()
    extent = orc.f32([0.0357, 0.0774])
    out = np.zeros(2000, np.uint32)
    L.or_seed_tracers(1000, extent, 0.5, out)
    depth = np.float32(L.or_slab_depth())
    for raw in out.reshape(-1, 2):
        p = np.zeros(4, np.float32)
        L.or_unpack_tracer(orc.u32(raw), extent, p)
        assert abs(p[0]) < extent[0] and abs(p[2]) < 0.5 * depth
        assert -extent[1] < p[1] < 0.0 + 0.001


# sim.rs:496-546
def test_step_immediates_land_at_the_shader_offsets(orc):
    L = orc.lib()
    raw = np.zeros(144, np.uint8)
    touches = orc.f32([[13, 14, 15, 16], [18, 19, 20, 21], [0] * 4, [0] * 4, [0] * 4])
    L.or_pack_step(orc.f32([1, 2, 3]), orc.f32([7, 8, 9]), orc.f32([10, 11, 12]), 4.0, 5.0, 6, 2,
                   17.0, touches.ctypes.data, raw)
    f = raw.view(np.float32)
    u = raw.view(np.uint32)
    assert list(f[0:3]) == [1, 2, 3] and f[3] == 4 and list(f[4:7]) == [7, 8, 9] and f[7] == 5
    assert list(f[8:11]) == [10, 11, 12] and u[11] == 6 and f[12] == 17 and u[13] == 2
    assert list(f[16:20]) == [13, 14, 15, 16] and list(f[20:24]) == [18, 19, 20, 21]
    # the oracle's Step struct is the same layout
    st = orc.make_step(force=(1, 2, 3), dt=4, omega=(7, 8, 9), v_clamp=5, domega=(10, 11, 12),
                       seed=6, touch_r=17, touches=[(13, 14, 15, 16), (18, 19, 20, 21)])
    assert bytes(st) == raw.tobytes()


# sim.rs:548-567
def test_sim_params_land_at_the_shader_offsets(orc):
    L = orc.lib()
    g = orc.OrGrid()
    g.min[:] = [1.0, 2.0, 3.0]
    g.cell = 4.0
    g.dims[:] = [5, 6, 7]
    raw = np.zeros(64, np.uint8)
    L.or_pack_sim_params(g, 8, 9.0, 10.0, L.or_rest_density(), raw)
    f = raw.view(np.float32)
    u = raw.view(np.uint32)
    assert list(f[0:4]) == [1, 2, 3, 4] and list(u[4:8]) == [5, 6, 7, 8]
    assert list(f[8:11]) == [9, 10, np.float32(L.or_rest_density())]
    sigma = np.float32(1.0) / (np.float32(np.pi) * np.float32(729.0))
    assert list(f[11:15]) == [np.float32(1.0) / np.float32(9.0), sigma, sigma / np.float32(9.0), 324]
    assert u[15] == 0


def cubic_h1(q):
    q = np.asarray(q, np.float64)
    s = 1.0 / np.pi
    return np.where(q < 1, s * (1 - 1.5 * q * q * (1 - q / 2)),
                    np.where(q < 2, s * 0.25 * np.clip(2 - q, 0, None) ** 3, 0.0))


def line_table():
    # L(rho) = 2 * int_0^2 W(sqrt(rho^2 + z^2)) dz by the trapezoid rule at
    # 1000 steps (sim.rs:611-621), tabulated and linearly interpolated
    n = 1000
    dq = 2.0 / n
    z = np.arange(n + 1) * dq
    rho = np.linspace(0, 3.0, 6001)
    w = cubic_h1(np.sqrt(rho[:, None] ** 2 + z[None, :] ** 2))
    val = 2.0 * np.sum((w[:, :-1] + w[:, 1:]) / 2 * dq, axis=1)
    return rho, val


# sim.rs:594-662
def test_wedge_polynomials_match_quadrature(orc):
    L = orc.lib()
    rho_t, line_t = line_table()
    line = lambda r: np.interp(r, rho_t, line_t)
    m = 400
    du = 2.0 / m
    for i in range(7):
        for j in range(7):
            a, b = i * 0.3, j * 0.3
            if a * a + b * b >= 4.0:
                continue
            u1 = a + (np.arange(m) + 0.5) * du
            u2 = b + (np.arange(m) + 0.5) * du
            u1 = u1[u1 < 2.0]
            u2 = u2[u2 < 2.0]
            i2 = float(np.sum(line(np.sqrt(u1[:, None] ** 2 + u2[None, :] ** 2))) * du * du)
            d2 = -float(np.sum(line(np.sqrt(a * a + u2 ** 2))) * du)
            assert abs(L.or_wedge64(a, b) - i2) < 1.5e-3, (a, b, L.or_wedge64(a, b), i2)
            assert abs(L.or_wedge_d64(a, b) - d2) < 8e-3, (a, b, L.or_wedge_d64(a, b), d2)
            # the shader's f32 copies evaluate the same polynomials
            assert abs(L.or_wedge(a, b) - L.or_wedge64(a, b)) < 1e-6
            assert abs(L.or_wedge_d(a, b) - L.or_wedge_d64(a, b)) < 1e-6


# sim.rs:664-696
def test_the_wedge_term_closes_the_edge_lattice_gap(orc):
    L = orc.lib()
    rho0 = np.float32(L.or_rest_density())
    d = np.float32(0.0025)
    h = np.float32(1.2) * d
    mass = rho0 * d * d * d
    ii = np.arange(-6, 7)
    for lx, ly in [(0, 0), (0, 1), (1, 1), (0, 2), (2, 2)]:
        x0 = (np.float32(lx) + np.float32(0.5)) * d
        y0 = (np.float32(ly) + np.float32(0.5)) * d
        quarter = np.float32(0)
        bulk = np.float32(0)
        for x in ii:
            for y in ii:
                for z in ii:
                    dx = (np.float32(x) + np.float32(0.5)) * d - x0
                    dy = (np.float32(y) + np.float32(0.5)) * d - y0
                    dz = np.float32(z) * d
                    w = mass * k_f32(L, np.sqrt(np.float32(dx * dx + dy * dy + dz * dz)), h)
                    bulk = np.float32(bulk + w)
                    if x >= 0 and y >= 0:
                        quarter = np.float32(quarter + w)
        fill = (np.float32(L.or_wall_density(float(x0 / h))) + np.float32(L.or_wall_density(float(y0 / h)))
                - np.float32(L.or_wedge64(float(x0 / h), float(y0 / h))))
        err = (quarter + rho0 * fill - bulk) / bulk
        assert abs(err) < 0.06, (lx, ly, err)


# sim.rs:708-745
def test_wall_adhesion_polynomial_matches_the_kernel_quadrature(orc):
    L = orc.lib()
    h = 1.2 * 0.0025
    c = 2.0 * h
    n = 4000
    dr = c / n
    r = np.arange(n + 1) * dr
    a = np.where((2 * r < c) | (r > c), 0.0,
                 0.007 / c ** 3.25 * np.maximum(-4 * r * r / c + 6 * r - 2 * c, 0.0) ** 0.25)
    int_a = np.zeros(n + 1)
    for i in range(n - 1, -1, -1):
        int_a[i] = int_a[i + 1] + (a[i] + a[i + 1]) / 2 * dr
    int_j = np.zeros(n + 1)
    for i in range(n - 1, -1, -1):
        u0, u1 = i * dr, (i + 1) * dr
        int_j[i] = int_j[i + 1] + (u0 * int_a[i] + u1 * int_a[i + 1]) / 2 * dr
    j0 = 2 * np.pi * int_j[0]
    for step in range(41):
        d = c * step / 40.0
        idx = int(round(d / dr))
        quad = 2 * np.pi * int_j[idx]
        assert abs(L.or_wall_adhesion64(d / h) - quad) < 0.005 * j0, (d / h,)
        assert abs(L.or_wall_adhesion(d / h) - L.or_wall_adhesion64(d / h)) < 1e-7


def test_half_packing_round_trips_and_rounds_to_nearest_even(orc):
    L = orc.lib()
    rng = np.random.default_rng(0)
    vals = np.concatenate([rng.uniform(-100, 100, 2000), rng.uniform(-1e-5, 1e-5, 500),
                           [0.0, -0.0, 1.0, 65504.0, 6.1035156e-05, 5.9604645e-08]]).astype(np.float32)
    for v in vals:
        bits = L.or_half_bits(float(v))
        assert bits == int(np.float16(v).view(np.uint16)), v
        assert np.float32(L.or_half_value(bits)) == np.float32(np.float16(v)), v


# The headless-test box (render.rs:3868-3882): 1,620 particles and 1,568
# cells at the 1x spacing (m5-menu.md:52; render.rs:3842).
def test_the_test_box_seeds_1620_particles_in_1568_cells(orc):
    k = kats()["test_box"]
    L = orc.lib()
    dims = np.zeros(3, np.uint32)
    L.or_lattice_dims(k["spacing"], orc.f32(k["extent"]), 0.5, dims)
    assert int(np.prod(dims)) == k["particles"]
    g = orc.grid_slab(k["extent"], 2.0 * np.float32(1.2) * np.float32(k["spacing"]))
    assert orc.cell_count(g) == k["cells"]


# validate_bench's scan check (render.rs:2703-2715): starts equals a CPU
# counting scan in particle-index order, and the sort is stable.
def test_the_grid_build_is_the_stable_counting_sort(orc):
    rng = np.random.default_rng(7)
    g = orc.grid_box([0, 0, 0], [1, 1, 1], 0.05)
    pos = np.zeros((5000, 4), np.float32)
    pos[:, :3] = rng.uniform(-0.1, 1.1, (5000, 3))
    keys, starts, perm = orc.grid_build(g, pos)
    C = orc.cell_count(g)
    expect = np.zeros(C + 1, np.int64)
    np.add.at(expect, keys.astype(np.int64) + 1, 1)
    assert np.array_equal(starts, np.cumsum(expect).astype(np.uint32))
    assert np.array_equal(perm, np.argsort(keys, kind="stable").astype(np.uint32))
