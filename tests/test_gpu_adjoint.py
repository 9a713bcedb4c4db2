"""The adjoint against central finite differences, and the gradient-check
harness around it.

The FP64 instance of the differentiable model is run forward at u + h d and
u - h d along 16 seeded unit directions d of the control space (the
per-frame body forces and the XSPH coefficient); each central difference
must match the adjoint's directional derivative g . d to 1e-3 relative. The
iteration counts are frozen from an FP32 forward and shared, so every
evaluation runs the same schedule. The gradient itself comes through a
torch.autograd.Function wrapping the C ABI's forward and backward (this
harness is its only user). The case is a scaled-down copy of the adjoint
workload: a 32x8x32 block in a box four block-widths wide and eight
block-heights tall, 4 substeps per frame, checkpoints every 1 or 3 frames
(so the backward recomputes two segments, the last one short).

The horizons are short because the discrete dynamics amplify perturbations
exponentially once the block starts to splash (the adjoint's norm grows
about 10x per 3 frames from frame 6 on, with every force term switched off
as well): central differences stop being a derivative estimate there, at
any step size. Two frames at step 1e-4 and four frames at step 1e-5 are
inside the linear range.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SPF = 4


def make_case(fcu, wl, frames):
    cfg = wl.box_config(fcu, (32, 8, 32), (0.64, 0.32, 0.64), 0.005, seed=7, xsph=0.01)
    dt = float(np.float32(1.0 / 120.0))
    dts = float(np.float32(dt) / np.float32(SPF))
    vc = wl.v_clamp(0.005, dts)
    forces = wl.tilt_schedule(4, frames, 1.0 / 120.0).astype(np.float64)
    rng = np.random.default_rng(11)
    target = rng.uniform([0.1, 0.01, 0.1], [0.3, 0.05, 0.3])
    return cfg, dt, vc, forces, target


def handles(fcu, wl, frames, ce):
    cfg, dt, vc, forces, target = make_case(fcu, wl, frames)
    a32 = fcu.Adjoint(cfg, frames, SPF, dt, vc, ce, precision=32)
    a32.forward(forces, 0.01, target)
    sched = a32.schedule()
    a64 = fcu.Adjoint(cfg, frames, SPF, dt, vc, ce, precision=64)
    a64.set_schedule(*sched)
    return a32, a64, forces, target, sched


def torch_fn():
    import torch

    class AdjointLoss(torch.autograd.Function):
        """loss(forces, xsph) through the C ABI; backward is the adjoint."""

        @staticmethod
        def forward(ctx, forces, xsph, handle, target):
            ctx.handle = handle
            loss = handle.forward(forces.detach().cpu().numpy(), float(xsph.detach()), target)
            return torch.tensor(loss, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gout):
            g, gx = ctx.handle.backward()
            return (torch.from_numpy(g) * gout, torch.tensor(gx, dtype=torch.float64) * gout,
                    None, None)

    return AdjointLoss


@pytest.mark.parametrize("frames,ce,h", [(2, 1, 1e-4), (4, 3, 1e-5)])
def test_fp64_adjoint_matches_central_differences_on_16_directions(fcu, wl, frames, ce, h):
    import torch
    a32, a64, forces, target, sched = handles(fcu, wl, frames, ce)
    assert sched[0].min() >= 1 and sched[1].max() >= 1
    fn = torch_fn()
    f = torch.tensor(forces, dtype=torch.float64, requires_grad=True)
    x = torch.tensor(0.01, dtype=torch.float64, requires_grad=True)
    loss = fn.apply(f, x, a64, target)
    loss.backward()
    g = np.concatenate([f.grad.numpy().ravel(), [x.grad.item()]])
    assert np.all(np.isfinite(g)) and np.linalg.norm(g) > 0
    u0 = np.concatenate([forces.ravel(), [0.01]])
    rng = np.random.default_rng(16)
    worst = 0.0
    for k in range(16):
        d = rng.normal(size=u0.size)
        d /= np.linalg.norm(d)
        lp = a64.forward((u0 + h * d)[:-1], (u0 + h * d)[-1], target)
        lm = a64.forward((u0 - h * d)[:-1], (u0 - h * d)[-1], target)
        fd = (lp - lm) / (2 * h)
        ad = float(g @ d)
        rel = abs(ad - fd) / max(abs(fd), 1e-12)
        worst = max(worst, rel)
        assert rel <= 1e-3, (k, ad, fd, rel)
    print(f"frames {frames}, step {h}: worst relative error over 16 directions {worst:.3g}")


def test_fp32_adjoint_follows_the_fp64_adjoint(fcu, wl):
    a32, a64, forces, target, sched = handles(fcu, wl, 4, 3)
    l32 = a32.forward(forces, 0.01, target)
    g32, x32 = a32.backward()
    l64 = a64.forward(forces, 0.01, target)
    g64, x64 = a64.backward()
    assert abs(l32 - l64) <= 1e-3 * abs(l64)
    a = np.concatenate([g32.ravel(), [x32]])
    b = np.concatenate([g64.ravel(), [x64]])
    cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
    assert cos > 0.999, cos
    assert np.linalg.norm(a - b) <= 0.05 * np.linalg.norm(b)


def test_the_forward_is_deterministic_and_checkpoints_do_not_change_it(fcu, wl):
    cfg, dt, vc, forces, target = make_case(fcu, wl, 4)
    a = fcu.Adjoint(cfg, 4, SPF, dt, vc, 3, precision=32)
    b = fcu.Adjoint(cfg, 4, SPF, dt, vc, 1, precision=32)
    la = a.forward(forces, 0.01, target)
    b.set_schedule(*a.schedule())
    lb = b.forward(forces, 0.01, target)
    # every reduction is in a fixed order (no floating-point atomics), so the
    # loss and the gradient are the same bits whatever the checkpointing
    assert la == lb
    ga, xa = a.backward()
    gb, xb = b.backward()
    assert np.array_equal(ga.view(np.uint64), gb.view(np.uint64)) and xa == xb
    # the backward recomputes every segment: a second forward + backward is
    # the same bits again
    assert a.forward(forces, 0.01, target) == la
    ga2, xa2 = a.backward()
    assert np.array_equal(ga2.view(np.uint64), ga.view(np.uint64)) and xa2 == xa


# The adjoint workload's own box: the 64x16x64 block (65,536 particles) of
# the benchmark's adjoint leg, checkpoints every 10 frames, 16 seeded
# directions, FP64 central differences. Four frames (16 substeps) is the
# longest horizon at which central differences at two step sizes agree:
# measured on this box, at 4 frames steps 1e-6 and 5e-7 agree with each other
# and with the adjoint to 1e-7, while at 6 frames the differences at steps
# 1e-4 .. 1e-6 differ from one another by 10-60 % (the loss is only piecewise
# smooth there: pairs cross the support radius and clamps switch within the
# step, and the sensitivity grows five- to tenfold a frame, |g| 8e-4 at 2
# frames, 6e-3 at 6, 1e2 at 10).
CONFIG4_FRAMES = 4


def test_fp64_adjoint_on_the_adjoint_workloads_box(fcu, wl):
    frames = CONFIG4_FRAMES
    cfg = wl.make_config(fcu, "adjoint_64k")
    dt = float(np.float32(1.0 / 120.0))
    dts = float(np.float32(dt) / np.float32(SPF))
    vc = wl.v_clamp(0.005, dts)
    forces = wl.tilt_schedule(2, frames, 1.0 / 120.0).astype(np.float64)
    target = np.array([0.64, 0.05, 0.64])
    a32 = fcu.Adjoint(cfg, frames, SPF, dt, vc, 10, precision=32)
    assert a32.n == 65536
    a32.forward(forces, 0.01, target)
    sched = a32.schedule()
    a64 = fcu.Adjoint(cfg, frames, SPF, dt, vc, 10, precision=64)
    a64.set_schedule(*sched)
    a64.forward(forces, 0.01, target)
    g, gx = a64.backward()
    gv = np.concatenate([g.ravel(), [gx]])
    # one checkpoint per frame recomputes four segments: the same bits
    a1 = fcu.Adjoint(cfg, frames, SPF, dt, vc, 1, precision=64)
    a1.set_schedule(*sched)
    a1.forward(forces, 0.01, target)
    g1, gx1 = a1.backward()
    assert np.array_equal(g1.view(np.uint64), g.view(np.uint64)) and gx1 == gx
    u0 = np.concatenate([forces.ravel(), [0.01]])
    rng = np.random.default_rng(16)
    floor = 1e-3 * np.linalg.norm(gv)
    worst = 0.0
    for k in range(16):
        d = rng.normal(size=u0.size)
        d /= np.linalg.norm(d)
        fd = {}
        for h in (1e-6, 5e-7):
            lp = a64.forward((u0 + h * d)[:-1], (u0 + h * d)[-1], target)
            lm = a64.forward((u0 - h * d)[:-1], (u0 - h * d)[-1], target)
            fd[h] = (lp - lm) / (2 * h)
        scale = max(abs(fd[1e-6]), floor)
        assert abs(fd[1e-6] - fd[5e-7]) <= 1e-3 * scale, (k, fd)  # the two steps agree
        rel = abs(float(gv @ d) - fd[1e-6]) / scale
        worst = max(worst, rel)
        assert rel <= 1e-3, (k, float(gv @ d), fd)
    print(f"adjoint_64k box, {frames} frames: worst relative error over 16 directions {worst:.3g}")
