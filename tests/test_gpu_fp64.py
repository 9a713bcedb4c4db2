"""The CUDA step against the FP64 oracle: the dam-break workload (16,384
particles, two substeps per 1/120 s frame, tolerance solve) on the GPU, and
the FP64 oracle (every substep operation in double) from the GPU's own
initial state and parameters, replaying the GPU's iteration counts substep
by substep. After two frames every particle is within 1e-4 spacings of the
FP64 path and the velocities within 1e-4 of the RMS speed (the same bounds
as tests/test_oracle_fp64.py, where the binary32 oracle, bit-identical to
this path, stands in for it)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

F32 = np.float32


def test_cuda_step_against_the_fp64_oracle(fcu, orc, wl):
    sim = fcu.Sim(wl.make_config(fcu, "dam_break_16k"))
    p = orc.OrParams()
    for name, _ in orc.OrParams._fields_:
        v = getattr(sim.params, name)
        if hasattr(v, "__len__"):
            getattr(p, name)[:] = list(v)
        else:
            setattr(p, name, v)
    o = orc.Sim(p, 0, fp64=True)
    st0 = sim.state()
    o.set_state(st0["pos"], st0["vel"], st0["prev_vel"], st0["prev_p"], st0["temp"], st0["id"])
    spacing = float(sim.cfg.spacing)
    dt = float(F32(F32(1.0 / 120.0) / F32(2)))
    vc = float(F32(0.4) * F32(spacing) / F32(dt))
    step = fcu.make_step(force=(0.0, -9.81, 0.0), dt=dt, v_clamp=vc)
    ostep = orc.make_step(force=(0.0, -9.81, 0.0), dt=dt, v_clamp=vc)
    for _ in range(4):
        a = sim.stats()
        sim.run([step])
        b = sim.stats()
        o.substep(ostep, int(b.total_div_iters - a.total_div_iters),
                  int(b.total_den_iters - a.total_den_iters))
    g = sim.state()
    gi = np.argsort(g["id"])
    oi = np.argsort(o.state()["id"])
    x64 = o.state64()
    dx = np.linalg.norm(g["pos"][gi, :3].astype(np.float64) - x64["pos"][oi, :3], axis=1)
    dv = np.linalg.norm(g["vel"][gi, :3].astype(np.float64) - x64["vel"][oi, :3], axis=1)
    vrms = np.sqrt(np.mean(np.sum(x64["vel"][oi, :3] ** 2, axis=1)))
    print(f"after 2 frames: max |dx| {dx.max() / spacing:.3e} spacings, "
          f"rms |dv| {np.sqrt(np.mean(dv ** 2)) / vrms:.3e} of the rms speed")
    assert 0.0 < dx.max() / spacing < 1e-4
    assert np.sqrt(np.mean(dv ** 2)) / vrms < 1e-4
