"""The oracle's solver kernels, each against an independent restatement.

The reference holds known answers for the grid and for the density sweep
(its own brute-force density check, render.rs:5141-5214, within 1e-3), but
none for the kernels after it. This file extends that check to the rest of
the solver: forces_eval (sim_solve.wgsl:524-592), forces_den_apply with the
rotating frame and fingers (:630-663, :103-127), den_kappa (:674-698),
den_apply (:596-621, :700-703) and integrate (:709-756), each restated here
in float64 NumPy from the WGSL, with its neighbours found by a brute-force
search over every particle (no list, no grid), on every 16th particle of the
reference test box in motion. Each oracle kernel is run alone on the working
set (or_sim_kernel) and fed the inputs it saw; the wall polynomials, which
the reference pins against quadrature on their own (sim.rs:432-446,
:595-662, :709-745, ported in test_oracle_kat.py), are the only shared
pieces.

Tolerance: a float32 sum of ~56 pair terms against its float64 value, so
each component within 1e-4 of the sum of its terms' magnitudes (the
reference's density check allows 1e-3 of the value).

The tracer pass (splat, resolve, advect with respawns, sim_tracers.wgsl:
54-183) is restated the same way over three frames of 4,096 tracers: the
branch decisions (respawn draws) compared in float32 as the shader does,
positions to within one step of the unorm16 packing, depth and charge to
within the float16 packing.
"""
import json
import math
import os

import numpy as np
import pytest

KATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_kats.json")))
TB = KATS["test_box"]

# sim_solve.wgsl:84-172
K_NEAR = 3000.0
MU = 1.002e-3
HEAT_CAPACITY = 4184.0
CONDUCTIVITY = 0.598
EXPANSION = 2.07e-4
SIGMA_WATER = 0.0728
LATTICE_SIGMA = 0.8665
COS_CONTACT = -0.342
XSPH_RATE = 6.0
TOUCH_RATE = 40.0
LENS_RATE = 20.0
REL = 1e-4
EVERY = 16


class Box:
    """Parameters of the test box as plain floats."""

    def __init__(self, p):
        f = lambda v: float(np.float32(v))
        self.h, self.mass, self.rho0 = f(p.h), f(p.mass), f(p.rho0)
        self.sigma, self.sigma_h = f(p.sigma), f(p.sigma_h)
        self.support_sq = f(p.support_sq)
        self.lo = np.array(list(p.wall_lo), np.float64)
        self.hi = np.array(list(p.wall_hi), np.float64)
        self.xsph_blend = f(p.xsph_blend)


def kernel_q(b, q):
    return np.where(q < 1.0, b.sigma * (1.0 - 1.5 * q * q * (1.0 - 0.5 * q)),
                    b.sigma * 0.25 * (2.0 - q) ** 3)


def grad(b, x, r):
    q = r / b.h
    dw = np.where(q < 1.0, b.sigma_h * (-3.0 * q + 2.25 * q * q), b.sigma_h * (-0.75 * (2.0 - q) ** 2))
    out = (dw / np.where(r < 1e-9, 1.0, r))[:, None] * x
    out[r < 1e-9] = 0.0
    return out


def neighbours(b, pos, i):
    """Every j != i inside the support, found by brute force."""
    x = pos[i, :3][None, :] - pos[:, :3]
    r2 = np.sum(x * x, axis=1)
    m = r2 < b.support_sq
    m[i] = False
    j = np.nonzero(m)[0]
    return j, x[j], np.sqrt(r2[j])


def cohesion(r, c):
    c3 = c ** 3
    k = 32.0 / (math.pi * c3 ** 3)
    near = c3 * c3 / 64.0
    a = (c - r) ** 3 * r ** 3
    out = np.where(2.0 * r > c, k * a, k * (2.0 * a - near))
    return np.where((r >= c) | (r < 1e-9), 0.0, out)


def within(got, want, scale, what):
    got, want, scale = (np.asarray(a, np.float64) for a in (got, want, scale))
    err = np.abs(got - want)
    bad = err > REL * scale + 1e-30
    assert not np.any(bad), (what, got[bad][:4], want[bad][:4], scale[bad][:4])


def wall_adh_sum(orc, b, pos):
    L = orc.lib()
    a = np.zeros(3)
    for ax in range(3):
        a[ax] -= L.or_wall_adhesion64((pos[ax] - b.lo[ax]) / b.h)
        a[ax] += L.or_wall_adhesion64((b.hi[ax] - pos[ax]) / b.h)
    return a


def forces_eval_np(orc, b, i, pos, vel, rho, temp, prev_p):
    """sim_solve.wgsl:524-592 for particle i: (accel.xyz, heat, xsph.xyz, kd,
    pressure) and the magnitude scales of each sum."""
    j, x, r = neighbours(b, pos, i)
    e = grad(b, x, r)
    f = np.sum(x * e, axis=1) / (r * r + 0.01 * b.h * b.h)
    pair = b.mass / (rho[i] * rho[j]) * f
    dv = vel[i, :3][None, :] - vel[j, :3]
    wn = np.maximum(1.0 - r / b.h, 0.0)
    near_t = ((pos[i, 3] + pos[j, 3]) * wn * wn)[:, None] * (x / np.maximum(r, 1e-5)[:, None])
    visc_t = (2.0 * MU * pair)[:, None] * dv
    blend_t = -(b.mass / rho[j] * kernel_q(b, r / b.h))[:, None] * dv
    heat_t = 2.0 * CONDUCTIVITY / HEAT_CAPACITY * pair * (temp[i] - temp[j]) \
        - 0.5 * MU / HEAT_CAPACITY * pair * np.sum(dv * dv, axis=1)
    corr = 2.0 * b.rho0 / (rho[i] + rho[j])
    c = 2.0 * b.h
    tens_t = -((corr * b.mass * cohesion(r, c))[:, None] * x) / np.maximum(r, 1e-9)[:, None]
    gamma = SIGMA_WATER * 7040.0 / (21.0 * LATTICE_SIGMA * b.rho0 ** 2 * c * c)
    beta = SIGMA_WATER * (1.0 + COS_CONTACT) * 1558.4 / (LATTICE_SIGMA * b.rho0 ** 2 * c * c)
    adh = beta * b.rho0 * wall_adh_sum(orc, b, pos[i, :3])
    acc = visc_t.sum(0) + K_NEAR * near_t.sum(0) + gamma * tens_t.sum(0) + adh
    acc_scale = np.abs(visc_t).sum(0) + K_NEAR * np.abs(near_t).sum(0) + \
        gamma * np.abs(tens_t).sum(0) + np.abs(adh)
    half = 0.5 * prev_p[i]
    return dict(accel=acc, accel_s=acc_scale, heat=heat_t.sum(), heat_s=np.abs(heat_t).sum(),
                xsph=blend_t.sum(0), xsph_s=np.abs(blend_t).sum(0), kd=half / rho[i] ** 2,
                pressure=half, n=len(j))


def kappa_sum_np(b, i, pos, kd):
    """sim_solve.wgsl:596-606: sum over neighbours of (kd_i + kd_j) grad W."""
    j, x, r = neighbours(b, pos, i)
    t = (kd[i] + kd[j])[:, None] * grad(b, x, r)
    return t.sum(0), np.abs(t).sum(0)


def fingers_np(st, pos, v):
    """sim_solve.wgsl:103-127."""
    px = py = w_sum = 0.0
    for t in range(st.touch_n):
        tx, ty, tvx, tvy = (float(v_) for v_ in st.touches[t])
        q2 = ((pos[0] - tx) ** 2 + (pos[1] - ty) ** 2) / (st.touch_r * st.touch_r)
        if q2 < 1.0:
            w = (1.0 - q2) ** 2
            px += w * tvx
            py += w * tvy
            w_sum += w
    if w_sum <= 0.0:
        return v
    a = 1.0 - math.exp(-TOUCH_RATE * w_sum * st.dt)
    return np.array([v[0] * (1 - a) + px / w_sum * a, v[1] * (1 - a) + py / w_sum * a, v[2]])


@pytest.fixture(scope="module")
def moving_box(orc):
    """The test box after 40 substeps under a tilted gravity, rotation and
    two fingers (a working set with every term nonzero)."""
    pos = orc.seed_slab(TB["spacing"], TB["extent"], 0.5)
    p = orc.params_slab(TB["extent"], TB["spacing"], 1.2, len(pos))
    s = orc.Sim(p, 0)
    s.set_state(pos4=pos)
    dt = float(np.float32(1.0 / 120.0) / np.float32(3.0))
    vc = float(np.float32(0.4) * np.float32(TB["spacing"]) / np.float32(dt))
    kw = dict(force=(1.5, -9.81, 0.4), dt=dt, v_clamp=vc, omega=(0.2, -0.1, 0.6),
              domega=(0.0, 0.3, 1.0), touch_r=0.04,
              touches=[(0.0, -0.1, 0.3, -0.2), (0.03, -0.12, -0.2, 0.1)])
    st = orc.make_step(**kw)
    for _ in range(40):
        s.substep(st)
    return s, Box(p), st


def test_every_solver_kernel_matches_an_independent_restatement(orc, moving_box):
    s, b, st = moving_box
    s.kernel("density", st)
    assert s.field("counters")[1] == 0, "the list overflowed: it would differ from brute force"
    f64 = lambda a: np.asarray(a, np.float64)
    pos, vel = f64(s.field("work_pos")), f64(s.field("work_vel"))
    rho, alpha, wg = f64(s.field("density")), f64(s.field("alpha")), f64(s.field("wall_grad"))
    temp, prev_p = f64(s.field("work_temp")), f64(s.field("work_prev_p"))
    prev_vel = f64(s.field("work_prev_vel"))
    n = len(rho)
    idx = range(0, n, EVERY)
    nbr_n = s.field("nbr_n")
    kd_div = f64(s.field("kd"))

    # density_div beyond the density itself (which test_oracle_step.py
    # checks as the reference does): near density, alpha and the first
    # divergence kappa, with the wall gradient as an input
    for i in idx:
        j, x, r = neighbours(b, pos, i)
        assert len(j) == nbr_n[i], i
        e = b.mass * grad(b, x, r)
        wn = np.maximum(1.0 - r / b.h, 0.0) ** 3
        within(pos[i, 3], wn.sum(), wn.sum(), f"density_div rho_near {i}")
        gsum = e.sum(0) + wg[i, :3]
        gsq = np.sum(e * e)
        a = rho[i] / max(np.dot(gsum, gsum) + gsq, 1e-4)
        a_s = rho[i] / max(np.dot(np.abs(e).sum(0) + np.abs(wg[i, :3]), np.abs(e).sum(0) +
                                  np.abs(wg[i, :3])) + gsq, 1e-4)
        within(alpha[i], a, a + a_s, f"density_div alpha {i}")
        t = np.sum((vel[i, :3][None, :] - vel[j, :3]) * e, axis=1)
        drho = t.sum() + np.dot(vel[i, :3], wg[i, :3])
        drho_s = np.abs(t).sum() + np.abs(vel[i, :3] * wg[i, :3]).sum()
        within(kd_div[i], max(drho, 0.0) * a / max(st.dt, 1e-9) / rho[i],
               drho_s * a / st.dt / rho[i], f"density_div kd {i}")

    # forces_eval
    s.kernel("forces_eval", st)
    acc, xs = f64(s.field("accel")), f64(s.field("xsph"))
    kd0, p0 = f64(s.field("kd")), f64(s.field("pressure"))
    seen = 0
    for i in idx:
        w = forces_eval_np(orc, b, i, pos, vel, rho, temp, prev_p)
        assert w["n"] == nbr_n[i], i
        within(acc[i, :3], w["accel"], w["accel_s"], f"forces_eval accel {i}")
        within(acc[i, 3], w["heat"], w["heat_s"], f"forces_eval heat {i}")
        within(xs[i, :3], w["xsph"], w["xsph_s"], f"forces_eval xsph {i}")
        within(kd0[i], w["kd"], abs(w["kd"]), f"forces_eval kd {i}")
        within(p0[i], w["pressure"], abs(w["pressure"]), f"forces_eval pressure {i}")
        seen += np.any(np.abs(w["accel"]) > 0) and abs(w["heat"]) > 0
    assert seen > len(idx) // 2

    # forces_den_apply: body force, rotating frame, XSPH, fingers, the warm
    # start's kappa correction, the temperature source
    s.kernel("forces_apply", st)
    vel1, temp1 = f64(s.field("work_vel")), f64(s.field("work_temp"))
    force = np.array(list(st.force), np.float64)
    om, dom = np.array(list(st.omega), np.float64), np.array(list(st.domega), np.float64)
    blend = b.xsph_blend if b.xsph_blend >= 0.0 else 1.0 - math.exp(-XSPH_RATE * st.dt)
    touched = 0
    for i in idx:
        r_, v = pos[i, :3], vel[i, :3]
        fict = -np.cross(dom, r_) - np.cross(om, np.cross(om, r_)) - 2.0 * np.cross(om, v)
        pre = v + st.dt * (force + fict + acc[i, :3]) + blend * xs[i, :3]
        forced = fingers_np(st, r_, pre)
        touched += not np.array_equal(forced, pre)
        tot, tot_s = kappa_sum_np(b, i, pos, kd0)
        dv_full = b.mass * tot + kd0[i] * wg[i, :3]
        want = forced - st.dt * dv_full
        scale = np.abs(forced) + st.dt * (np.abs(force) + np.abs(fict) + np.abs(acc[i, :3])) + \
            blend * np.abs(xs[i, :3]) + st.dt * (b.mass * tot_s + np.abs(kd0[i] * wg[i, :3]))
        within(vel1[i, :3], want, scale, f"forces_apply vel {i}")
        within(temp1[i], temp[i] + st.dt * acc[i, 3], temp[i] * 1e-3, f"forces_apply temp {i}")
    assert touched > 0, "no checked particle was under a finger"

    # den_kappa
    s.kernel("den_kappa", st)
    kd1, pinc = f64(s.field("kd")), f64(s.field("pinc"))
    pushed = 0
    for i in idx:
        j, x, r = neighbours(b, pos, i)
        e = grad(b, x, r)
        t = np.sum((vel1[i, :3][None, :] - vel1[j, :3]) * e, axis=1)
        drho = b.mass * t.sum() + np.dot(vel1[i, :3], wg[i, :3])
        drho_s = b.mass * np.abs(t).sum() + np.abs(vel1[i, :3] * wg[i, :3]).sum()
        rho_star = rho[i] + st.dt * drho
        k = max(rho_star - b.rho0, 0.0) * alpha[i] / (st.dt * st.dt)
        # kd = k / rho: its error is that of rho* - rho0, whose terms are dt * drho
        k_s = st.dt * drho_s * alpha[i] / (st.dt * st.dt) + abs(k) * 1e-3
        within(kd1[i], k / rho[i], k_s / rho[i], f"den_kappa kd {i}")
        within(pinc[i], k * rho[i], k_s * rho[i], f"den_kappa k*rho {i}")
        pushed += k > 0
    assert 0 < pushed < len(idx)

    # den_apply
    s.kernel("den_apply", st)
    vel2, p2 = f64(s.field("work_vel")), f64(s.field("pressure"))
    for i in idx:
        tot, tot_s = kappa_sum_np(b, i, pos, kd1)
        want = vel1[i, :3] - st.dt * (b.mass * tot + kd1[i] * wg[i, :3])
        scale = np.abs(vel1[i, :3]) + st.dt * (b.mass * tot_s + np.abs(kd1[i] * wg[i, :3]))
        within(vel2[i, :3], want, scale, f"den_apply vel {i}")
        within(p2[i], p0[i] + pinc[i], abs(p0[i]) + abs(pinc[i]), f"den_apply pressure {i}")

    # integrate: reads the working set, writes the resting set at the same slot
    s.kernel("integrate", st)
    out = s.state()
    lo, hi = b.lo, b.hi
    chase = 1.0 - math.exp(-LENS_RATE * st.dt)
    clamped = walled = 0
    for i in idx:
        v = vel2[i, :3].copy()
        speed = np.linalg.norm(v)
        ceiling = 3.0 * st.v_clamp if rho[i] < 0.5 * b.rho0 else st.v_clamp
        if speed > ceiling:
            v = v * (ceiling / speed)
            clamped += 1
        accel = np.linalg.norm(v - prev_vel[i, :3]) / st.dt
        pp = pos[i, :3] + v * st.dt
        cl = np.clip(pp, lo, hi)
        v = np.where(cl != pp, 0.0, v)
        walled += np.any(cl != pp)
        # elementwise float32 arithmetic: within 1e-5 of each value
        sc = lambda a: np.abs(a) * 0.1 + 1e-6
        within(out["pos"][i, :3], cl, sc(cl), f"integrate pos {i}")
        within(out["vel"][i, :3], v, sc(v), f"integrate vel {i}")
        within(out["vel"][i, 3], vel2[i, 3] * (1 - chase) + accel * chase,
               sc(vel2[i, 3]) + sc(accel), f"integrate accel lens {i}")
        within(out["prev_vel"][i, 3], prev_vel[i, 3] * (1 - chase) + p2[i] * chase,
               sc(prev_vel[i, 3]) + sc(p2[i]), f"integrate pressure lens {i}")
        within(out["prev_p"][i], p2[i], sc(p2[i]), f"integrate prev_p {i}")
        dp = p2[i] - prev_p[i]
        t = temp1[i]
        want_t = t + t * EXPANSION / (rho[i] * HEAT_CAPACITY) * dp
        within(out["temp"][i], want_t, sc(want_t), f"integrate temp {i}")
    assert walled > 0


# The finger blend's exp (sim_solve.wgsl:122) is evaluated per particle by a
# fixed Cody-Waite reduction and a degree-7 Taylor polynomial on both the
# CUDA and the CPU side, so that the two agree bit for bit; this bounds its
# error against the double-precision exp over the range the blend reaches
# (-TOUCH_RATE * weight * dt, weight up to 5 fingers of 1, dt up to a frame)
# and beyond.
def test_the_deterministic_exp_is_within_two_ulp_of_exp(orc):
    L = orc.lib()
    lo = -TOUCH_RATE * 5.0 * (1.0 / 60.0)
    xs = np.concatenate([np.linspace(lo, 0.0, 200001, dtype=np.float32),
                         np.linspace(-80.0, 80.0, 100001, dtype=np.float32)])
    worst = 0.0
    for x in xs:
        got = np.float32(L.or_det_exp(float(x)))
        want = math.exp(float(x))
        ulp = float(np.spacing(np.float32(want)))
        worst = max(worst, abs(float(got) - want) / ulp)
    assert worst <= 2.0, worst
    assert L.or_det_exp(0.0) == 1.0
    assert L.or_det_exp(-100.0) == 0.0


# ---- the tracer pass (sim_tracers.wgsl:54-183), restated -------------------
FIXED = 65536.0
TAU, TAU_STRAY, T_CHARGE = 3.0, 0.25, 4.0
M32 = 0xFFFFFFFF


def pcg(x):
    h = (x * 747796405 + 2891336453) & M32
    h = (((h >> ((h >> 28) + 4)) ^ h) * 277803737) & M32
    return ((h >> 22) ^ h) & M32


def i32_trunc(v):
    """WGSL i32(f32): toward zero, saturating."""
    return int(max(min(math.trunc(v), 2 ** 31 - 1), -2 ** 31))


def tracer_pass_np(p, pos, vel, tracers, dt, seed):
    """splat -> resolve -> advect for the slab geometry (box extent
    -(box_min + cell)), in float64 except where the shader compares float32
    values to decide a branch. Returns decoded (x, y, z, charge) per tracer
    and which tracers respawned."""
    bmin = np.array(list(p.box_min), np.float64)
    cell = float(np.float32(p.cell))
    dims = np.array(list(p.dims), np.int64)
    e = -(bmin + cell)
    grid = np.zeros((dims[2], dims[1], dims[0], 4), np.int64)
    for k in range(len(pos)):
        u = np.floor(np.maximum((pos[k, :3] - bmin) / cell, 0.0)).astype(np.int64)
        c = np.minimum(u, dims - 1)
        g = grid[c[2], c[1], c[0]]
        for a in range(3):
            g[a] += i32_trunc(float(np.float32(np.float32(vel[k, a]) * np.float32(FIXED))))
        g[3] += 1
    f32 = np.float32
    thr = f32(f32(dt) / f32(TAU))
    thr_stray = f32(f32(dt) / f32(TAU_STRAY))
    out = np.zeros((len(tracers), 4))
    respawned = np.zeros(len(tracers), bool)

    def respawn(slot, r):
        r1 = pcg(r)
        r2 = pcg(r1)
        r3 = pcg(r2)
        r4 = pcg(r3)
        jit = (np.array([r2 >> 20, r3 >> 20, r4 >> 20], np.float64) / 4096.0 - 0.5) * (cell * 0.5)
        j = r1 % len(pos)
        q = np.clip(pos[j, :3] + jit, -e, e)
        out[slot] = [q[0], q[1], q[2], np.linalg.norm(vel[j, :3])]
        respawned[slot] = True

    for i in range(len(tracers)):
        r0 = pcg(i ^ pcg(seed))
        if f32(f32(r0) / f32(4294967295.0)) < thr:
            respawn(i, r0)
            continue
        t = tracers[i]
        xy = ((np.array([t[0] & 0xFFFF, t[0] >> 16]) / 65535.0) * 2.0 - 1.0) * e[:2]
        z = float(np.array([t[1] & 0xFFFF], np.uint16).view(np.float16)[0])
        s = float(np.array([t[1] >> 16], np.uint16).view(np.float16)[0])
        q = np.array([xy[0], xy[1], z])
        gp = (q - bmin) / cell - 0.5
        base = np.clip(np.floor(gp).astype(np.int64), 0, dims - 2)
        fr = np.clip(gp - base, 0.0, 1.0)
        mom = np.zeros(3)
        wc = 0.0
        for k in range(8):
            o = np.array([k & 1, (k >> 1) & 1, (k >> 2) & 1])
            w = np.where(o == 1, fr, 1.0 - fr)
            wt = w[0] * w[1] * w[2]
            c = base + o
            cellv = grid[c[2], c[1], c[0]]
            mom += wt * cellv[:3]
            wc += wt * cellv[3]
        if wc > 0.0:
            v = mom / (wc * FIXED)
        elif f32(f32(pcg(r0 ^ 0x85EBCA6B)) / f32(4294967295.0)) < thr_stray:
            respawn(i, pcg(r0 ^ 0x632BE59B))
            continue
        else:
            v = np.zeros(3)
        q = np.clip(q + v * dt, -e, e)
        out[i] = [q[0], q[1], q[2], max(np.linalg.norm(v), s * math.exp(-dt / T_CHARGE))]
    return out, respawned


def decode(orc, tracers, e):
    out = np.zeros((len(tracers), 4), np.float32)
    ext = np.ascontiguousarray(e[:2], np.float32)
    for i, t in enumerate(tracers):
        orc.lib().or_unpack_tracer(np.ascontiguousarray(t, np.uint32), ext, out[i])
    return out


def test_the_tracer_pass_matches_an_independent_restatement(orc, moving_box):
    s, b, st = moving_box
    p = s.p
    n_tr = 4096
    t0 = np.zeros((n_tr, 2), np.uint32)
    orc.lib().or_seed_tracers(n_tr, orc.f32(TB["extent"]), 0.5, t0.reshape(-1))
    tr = orc.Sim(p, n_tr)
    rest = s.state()
    tr.set_state(rest["pos"], rest["vel"], rest["prev_vel"], rest["prev_p"], rest["temp"], rest["id"])
    tr.set_tracers(t0)
    dt = float(np.float32(1.0 / 120.0))
    bmin = np.array(list(p.box_min), np.float64)
    e = -(bmin + float(np.float32(p.cell)))
    pos64, vel64 = rest["pos"].astype(np.float64), rest["vel"].astype(np.float64)
    before = t0.copy()
    for frame in range(3):
        seed = 11 + frame
        want, resp = tracer_pass_np(p, pos64, vel64, before, dt, seed)
        tr.tracer_pass(orc.make_step(dt=dt, seed=seed))
        got_raw = tr.tracers()
        got = decode(orc, got_raw, e)
        quantum = 2.0 * e[:2] / 65535.0
        assert np.all(np.abs(got[:, :2] - want[:, :2]) <= 1.01 * quantum), frame
        z_tol = np.maximum(np.abs(want[:, 2]) * 2.0 ** -10, 2.0 ** -24) * 1.01
        assert np.all(np.abs(got[:, 2] - want[:, 2]) <= z_tol), frame
        c_tol = np.maximum(np.abs(want[:, 3]) * 2.0 ** -10, 2.0 ** -24) * 1.01
        assert np.all(np.abs(got[:, 3] - want[:, 3]) <= c_tol), frame
        moved = np.linalg.norm(got[:, :3] - decode(orc, before, e)[:, :3], axis=1)
        assert resp.sum() > 0 and np.count_nonzero(moved[~resp]) > n_tr // 4, frame
        before = got_raw


# reduce_stats (sim_solve.wgsl:758-874) restated over the resting set and the
# last sweep's densities: the mean compression is a sum (float64 here, an
# exact fixed-point sum in the oracle), every other slot a min or max, which
# no summation order changes.
def test_the_stats_block_matches_an_independent_restatement(orc, moving_box):
    s, b, st = moving_box
    s.substep(st)
    got = s.stats()
    rho = np.asarray(s.field("density"), np.float64)
    rest = s.state()
    c = rho / b.rho0 - 1.0
    speed = np.linalg.norm(rest["vel"][:, :3].astype(np.float64), axis=1)
    want = np.array([np.maximum(c, 0.0).mean(), max(c.max(), 0.0), rho.min(), rho.max(),
                     rest["prev_vel"][:, 3].min(), rest["prev_vel"][:, 3].max(), speed.max(),
                     rest["temp"].min(), rest["temp"].max(), np.nan, np.nan, speed.min(),
                     rest["vel"][:, 3].min(), rest["vel"][:, 3].max()])
    for k in range(14):
        if k in (9, 10):
            continue
        tol = 1e-6 * abs(want[k]) + (1e-9 if k == 0 else 0.0)
        if k in (6, 11):  # float32 length against float64
            tol = 1e-6 * abs(want[k]) + 1e-12
        assert abs(float(got[k]) - want[k]) <= tol, (k, got[k], want[k])
    counters = s.field("counters")
    assert got[9] == np.float32(counters[0]) and got[10] == np.float32(counters[1])
    assert got[0] > 0 and got[6] > 0
