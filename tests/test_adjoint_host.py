"""The adjoint handle's argument checks (host only: refused before any
device call)."""


def test_adjoint_refuses_bad_arguments(fcu, wl):
    cfg = wl.box_config(fcu, (8, 4, 8), (0.16, 0.08, 0.16), 0.005)
    L = fcu.lib()
    assert not L.fluid_adjoint_create(None, 4, 4, 0.01, 0.1, 2, 32)
    import ctypes as C
    assert not L.fluid_adjoint_create(C.byref(cfg), 4, 4, 0.01, 0.1, 2, 16)
    assert "precision" in L.fluid_last_error().decode()
    assert not L.fluid_adjoint_create(C.byref(cfg), 0, 4, 0.01, 0.1, 2, 32)
    assert not L.fluid_adjoint_create(C.byref(cfg), 4, 4, 0.0, 0.1, 2, 32)
    assert L.fluid_adjoint_backward(None, None, None) == -1
    assert L.fluid_adjoint_count(None) == 0
