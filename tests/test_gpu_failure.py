"""Failure detection on the GPU without a fault: the grid's look-back scan,
and a radix digit pass of the grid build, are run with a predecessor tile
that never publishes, so their bounded waits give up. The call reports
FLUID_ERR_TIMEOUT with a reason, the kernel ends on its own within about a
second, and the device stays usable (a step still matches the oracle bit
for bit). The digit pass's give-up reaches the caller the way a
device-pointer build's does: through fluid_grid_build_status on the
workspace it ran on, and fluid_grid_build_static_status on the fixed
scratch."""
import pytest

from test_gpu_step import frame_dt, pair, same_state, step_pair, v_clamp

pytestmark = pytest.mark.gpu


def test_the_scan_wait_gives_up_and_reports_a_timeout(fcu, orc):
    rc, ms = fcu.selftest_scan_wait(0)
    assert rc == fcu.ERR_TIMEOUT, (rc, fcu.last_error())
    assert "gave up" in fcu.last_error()
    assert 0.0 < ms < 10000.0, ms
    print(f"bounded look-back wait gave up after {ms:.1f} ms")
    # the context is still usable
    sim, o = pair(fcu, orc)
    dt = frame_dt(1)
    st, ost = step_pair(fcu, orc, force=(0.0, -9.81, 0.0), dt=dt, v_clamp=v_clamp(sim.cfg.spacing, dt))
    sim.step(st)
    o.substep(ost, sim.cfg.div_iters, sim.cfg.den_iters)
    same_state(sim, o, "after the timeout")


def test_the_radix_pass_wait_gives_up_and_reports_a_timeout(fcu, orc):
    rc, ms = fcu.selftest_radix_wait(0)
    assert rc == fcu.ERR_TIMEOUT, (rc, fcu.last_error())
    assert "fluid_grid_build_status reported it" in fcu.last_error()
    assert 0.0 < ms < 10000.0, ms
    print(f"bounded digit look-back gave up after {ms:.1f} ms")
    sim, o = pair(fcu, orc)
    dt = frame_dt(1)
    st, ost = step_pair(fcu, orc, force=(0.0, -9.81, 0.0), dt=dt, v_clamp=v_clamp(sim.cfg.spacing, dt))
    sim.step(st)
    o.substep(ost, sim.cfg.div_iters, sim.cfg.den_iters)
    same_state(sim, o, "after the timeout")


def test_the_static_scratch_wait_is_reported_by_the_static_status(fcu, orc):
    rc, ms = fcu.selftest_static_radix_wait(0)
    assert rc == fcu.ERR_TIMEOUT, (rc, fcu.last_error())
    assert "fluid_grid_build_static_status reported it" in fcu.last_error()
    assert 0.0 < ms < 10000.0, ms
    # the status word stays set until the next static build clears it
    assert fcu.lib().fluid_grid_build_static_status(None) == fcu.ERR_TIMEOUT
    sim, o = pair(fcu, orc)
    dt = frame_dt(1)
    st, ost = step_pair(fcu, orc, force=(0.0, -9.81, 0.0), dt=dt, v_clamp=v_clamp(sim.cfg.spacing, dt))
    sim.step(st)
    o.substep(ost, sim.cfg.div_iters, sim.cfg.den_iters)
    same_state(sim, o, "after the timeout")
