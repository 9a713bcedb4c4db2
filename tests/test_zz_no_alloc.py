"""fluid_grid_build_static, the grid build that allocates nothing, against
fluid_grid_build on a caller's workspace.

Keys, cell starts and the permutation are integers, so the tolerance is
zero: every element must match. Each case makes two calls in a row on
different positions (the second without a keys buffer), so a call cannot
pass on what the previous one left in the fixed scratch. This file sorts
last so that it also runs after everything else the suite did on the device.
"""
import ctypes as C

import numpy as np
import pytest


def _grid(fcu, dims, cell=1.0):
    g = fcu.FluidGrid()
    g.min[:] = [0.0, 0.0, 0.0]
    g.cell = cell
    g.dims[:] = list(dims)
    return g


def _positions(n, dims, seed):
    rng = np.random.default_rng(seed)
    p = np.zeros((n, 4), np.float32)
    centres = rng.uniform(0.2, 0.8, (6, 3)) * np.array(dims, np.float32)
    k = n // 2
    p[:k, :3] = rng.uniform(0, 1, (k, 3)) * np.array(dims, np.float32)
    p[k:, :3] = centres[rng.integers(0, 6, n - k)] + rng.normal(0, 3.0, (n - k, 3))
    return p


def _static_build(fcu, d_pos, n, g, keys, starts, perm, stream):
    rc = fcu.lib().fluid_grid_build_static(C.c_void_p(d_pos), n, C.byref(g),
                                           C.c_void_p(keys) if keys else None,
                                           C.c_void_p(starts), C.c_void_p(perm),
                                           C.c_void_p(stream))
    assert rc == 0, fcu.lib().fluid_last_error()


def test_oversize_build_is_refused_before_any_device_work(fcu):
    g = _grid(fcu, (64, 64, 64))
    n = 1 << 20
    assert fcu.grid_workspace_bytes(n, g) > 16 << 20
    fake = C.c_void_p(256)  # never dereferenced: the size check comes first
    rc = fcu.lib().fluid_grid_build_static(fake, n, C.byref(g), None, fake, fake, None)
    assert rc == -1
    msg = fcu.lib().fluid_last_error().decode()
    assert "fluid_grid_build_static" in msg and str(16 << 20) in msg


@pytest.mark.gpu
@pytest.mark.parametrize("n,dims", [(1 << 19, (128, 128, 64)), (1000, (7, 5, 3)), (0, (4, 4, 4))])
def test_static_build_matches_workspace_build_twice(fcu, n, dims):
    import torch
    g = _grid(fcu, dims)
    cells = dims[0] * dims[1] * dims[2]
    assert fcu.grid_workspace_bytes(n, g) <= 16 << 20
    wsb = fcu.grid_workspace_bytes(n, g)
    ws = torch.empty(wsb + 256, dtype=torch.uint8, device="cuda")
    base = (ws.data_ptr() + 255) // 256 * 256
    stream = torch.cuda.Stream()
    m = max(n, 1)
    for call, seed in enumerate((11, 12)):
        pos = _positions(n, dims, seed)
        d_pos = torch.from_numpy(pos if n else np.zeros((1, 4), np.float32)).cuda()
        out = {}
        for name in ("workspace", "static"):
            keys = torch.full((m,), -1, dtype=torch.int32, device="cuda")
            starts = torch.full((cells + 1,), -1, dtype=torch.int32, device="cuda")
            perm = torch.full((m,), -1, dtype=torch.int32, device="cuda")
            torch.cuda.synchronize()
            with_keys = keys.data_ptr() if call == 0 else 0
            if name == "workspace":
                fcu.grid_build_device(d_pos.data_ptr(), n, g, with_keys, starts.data_ptr(),
                                      perm.data_ptr(), base, wsb, stream.cuda_stream)
            else:
                _static_build(fcu, d_pos.data_ptr(), n, g, with_keys, starts.data_ptr(),
                              perm.data_ptr(), stream.cuda_stream)
            stream.synchronize()
            if name == "workspace":
                assert fcu.grid_build_status(base, n, g, stream.cuda_stream) == 0
            else:
                assert fcu.lib().fluid_grid_build_static_status(C.c_void_p(stream.cuda_stream)) == 0
            out[name] = (keys.cpu().numpy()[:n], starts.cpu().numpy(), perm.cpu().numpy()[:n])
        for a, b in zip(out["workspace"], out["static"]):
            assert np.array_equal(a, b)
        assert out["static"][1][-1] == n
        if n:
            assert np.array_equal(np.sort(out["static"][2]), np.arange(n, dtype=np.int32))
