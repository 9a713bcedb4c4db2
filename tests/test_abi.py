"""The C ABI library loads, exports what include/fluid_cu.h declares, and
its host-side logic behaves without a GPU (no compute calls here)."""
import ctypes as C

import numpy as np


def test_library_exports_every_declared_function(fcu):
    L = fcu.lib()
    names = fcu.header_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_struct_layouts_match_the_header(fcu):
    assert C.sizeof(fcu.FluidStep) == 144          # sim.rs:202 STEP_BYTES
    assert C.sizeof(fcu.FluidSimParams) == 116
    assert fcu.FluidStep.force.offset == 0 and fcu.FluidStep.dt.offset == 12
    assert fcu.FluidStep.omega.offset == 16 and fcu.FluidStep.v_clamp.offset == 28
    assert fcu.FluidStep.domega.offset == 32 and fcu.FluidStep.seed.offset == 44
    assert fcu.FluidStep.touch_r.offset == 48 and fcu.FluidStep.touch_n.offset == 52
    assert fcu.FluidStep.touches.offset == 64


def test_the_step_block_is_the_reference_layout(fcu, orc):
    st = fcu.make_step(force=(1, 2, 3), dt=4, omega=(7, 8, 9), v_clamp=5, domega=(10, 11, 12),
                       seed=6, touch_r=17, touches=[(13, 14, 15, 16), (18, 19, 20, 21)])
    raw = np.zeros(144, np.uint8)
    touches = orc.f32([[13, 14, 15, 16], [18, 19, 20, 21], [0] * 4, [0] * 4, [0] * 4])
    orc.lib().or_pack_step(orc.f32([1, 2, 3]), orc.f32([7, 8, 9]), orc.f32([10, 11, 12]), 4.0, 5.0,
                           6, 2, 17.0, touches.ctypes.data, raw)
    assert bytes(st) == raw.tobytes()


def test_default_config_is_the_reference_test_box(fcu):
    cfg = fcu.default_config()
    assert cfg.geometry == fcu.GEOMETRY_SLAB and cfg.seeding == fcu.SEED_SLAB
    assert abs(cfg.h_ratio - 1.2) < 1e-7 and cfg.nbr_cap == 96
    assert (cfg.div_iters, cfg.den_iters) == (1, 5)
    assert np.float32(cfg.extent[0]) == np.float32(4.0) * np.float32(0.0357)


def test_create_rejects_bad_configs_with_a_reason(fcu):
    L = fcu.lib()
    for kw in [dict(spacing=0.0), dict(h_ratio=-1.0), dict(nbr_cap=0), dict(geometry=7),
               dict(seeding=fcu.SEED_BLOCK), dict(div_iters=1000)]:
        cfg = fcu.default_config(**kw)
        assert not L.fluid_sim_create(C.byref(cfg))
        assert fcu.last_error() != ""


def test_grid_workspace_size_is_reported(fcu):
    g = fcu.FluidGrid()
    g.min[:] = [0, 0, 0]
    g.cell = 1.0
    g.dims[:] = [256, 256, 256]
    b = fcu.grid_workspace_bytes(1 << 24, g)
    # ping-pong keys and values, four words per position; no per-cell array
    assert 4 * (1 << 24) * 4 <= b < 4 * (1 << 24) * 5
    g.dims[:] = [0, 1, 1]
    assert fcu.grid_workspace_bytes(10, g) == 0


# A simulation's cells hold their slots in x-slab order on both sides: the
# oracle must sort by the same keys as the library for the sums to agree.
def test_the_library_and_the_oracle_cut_cells_into_the_same_slabs(fcu, orc):
    assert fcu.grid_slabs() == orc.sim_slabs() == 4
