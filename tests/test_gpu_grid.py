"""The neighbour grid on the GPU against the oracle's stable counting sort.

The reference pins its grid by an exact scan comparison against a CPU
counting scan (render.rs:2703-2715, validate_bench) and by permutation
membership (render.rs:5031-5135). Here starts and the permutation are
compared element for element with the stable counting sort, on the three
distributions of the 16.7M-position grid workload (uniform, 90 % packed into
the lowest tenth, eight Gaussian clusters of sigma 4 cells) and edge cases.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def grid(orc, fcu, side):
    g = fcu.FluidGrid()
    g.min[:] = [0.0, 0.0, 0.0]
    g.cell = 1.0
    g.dims[:] = [side, side, side]
    og = orc.OrGrid()
    og.min[:] = [0.0, 0.0, 0.0]
    og.cell = 1.0
    og.dims[:] = [side, side, side]
    return g, og


@pytest.mark.parametrize("kind", ["uniform", "packed", "gaussian"])
def test_grid_is_the_stable_counting_sort(orc, fcu, wl, kind):
    side = 64
    g, og = grid(orc, fcu, side)
    pos = wl.grid_positions(kind, 1 << 20, side, seed={"uniform": 1, "packed": 2, "gaussian": 3}[kind])
    starts, perm = fcu.grid_build_host(pos, g)
    keys, e_starts, e_perm = orc.grid_build(og, pos)
    assert starts[-1] == len(pos)
    assert np.array_equal(starts, e_starts)
    assert np.array_equal(perm, e_perm)


@pytest.mark.parametrize("kind", ["uniform", "packed", "gaussian"])
def test_grid_at_full_size_16m_positions_in_2_24_cells(orc, fcu, wl, kind):
    side = 256
    g, og = grid(orc, fcu, side)
    pos = wl.grid_positions(kind, 1 << 24, side, seed={"uniform": 1, "packed": 2, "gaussian": 3}[kind])
    starts, perm = fcu.grid_build_host(pos, g)
    keys, e_starts, e_perm = orc.grid_build(og, pos)
    assert np.array_equal(starts, e_starts)
    assert np.array_equal(perm, e_perm)


def test_grid_edge_cases(orc, fcu, wl):
    side = 16
    g, og = grid(orc, fcu, side)
    cases = {
        "one": np.array([[3.5, 2.5, 1.5, 0]], np.float32),
        "all_in_one_cell": np.tile(np.array([[5.5, 5.5, 5.5, 0]], np.float32), (20000, 1)),
        "outside_and_nan": np.array([[-5, 1, 1, 0], [100, 100, 100, 0], [np.nan, 1, 1, 0],
                                     [1, -np.inf, np.inf, 0], [15.999, 0, 0, 0]] * 1000, np.float32),
        "ragged": wl.grid_positions("uniform", 4097, side, 9),
        "tile_edge": wl.grid_positions("gaussian", 4096 * 3, side, 10),
    }
    for name, pos in cases.items():
        starts, perm = fcu.grid_build_host(pos, g)
        _, e_starts, e_perm = orc.grid_build(og, pos)
        assert np.array_equal(starts, e_starts), name
        assert np.array_equal(perm, e_perm), name


def test_grid_with_no_positions(fcu):
    g = fcu.FluidGrid()
    g.min[:] = [0, 0, 0]
    g.cell = 1.0
    g.dims[:] = [4, 4, 4]
    starts, perm = fcu.grid_build_host(np.zeros((0, 4), np.float32), g)
    assert np.all(starts == 0) and len(perm) == 0


def test_grid_on_device_pointers_in_a_caller_stream(orc, fcu, wl):
    import torch
    side = 128
    g, og = grid(orc, fcu, side)
    pos = wl.grid_positions("gaussian", 1 << 21, side, 5)
    d_pos = torch.from_numpy(pos).cuda()
    n = pos.shape[0]
    C = side ** 3
    keys = torch.zeros(n, dtype=torch.int32, device="cuda")
    starts = torch.zeros(C + 1, dtype=torch.int32, device="cuda")
    perm = torch.zeros(n, dtype=torch.int32, device="cuda")
    wsb = fcu.grid_workspace_bytes(n, g)
    ws = torch.empty(wsb + 256, dtype=torch.uint8, device="cuda")
    base = (ws.data_ptr() + 255) // 256 * 256
    stream = torch.cuda.Stream()
    fcu.grid_build_device(d_pos.data_ptr(), n, g, keys.data_ptr(), starts.data_ptr(),
                          perm.data_ptr(), base, wsb, stream.cuda_stream)
    stream.synchronize()
    e_keys, e_starts, e_perm = orc.grid_build(og, pos)
    assert np.array_equal(keys.cpu().numpy().view(np.uint32), e_keys)
    assert np.array_equal(starts.cpu().numpy().view(np.uint32), e_starts)
    assert np.array_equal(perm.cpu().numpy().view(np.uint32), e_perm)
    # a second build into the same workspace gives the same answer
    fcu.grid_build_device(d_pos.data_ptr(), n, g, 0, starts.data_ptr(), perm.data_ptr(), base, wsb,
                          stream.cuda_stream)
    stream.synchronize()
    assert np.array_equal(perm.cpu().numpy().view(np.uint32), e_perm)


@pytest.mark.parametrize("dims,passes", [((4, 4, 4), 1), ((40, 40, 40), 2), ((256, 256, 256), 3),
                                         ((512, 256, 256), 4)])
def test_grid_every_digit_pass_count(orc, fcu, wl, dims, passes):
    """1 to 4 eight-bit digit passes (keys below 2^8, 2^16, 2^24, 2^25): the
    last pass writes the run ends, so each count is checked, with keys
    clustered enough that runs of equal keys cross tile boundaries."""
    cells = dims[0] * dims[1] * dims[2]
    assert passes == max(1, ((cells - 1).bit_length() + 7) // 8)
    g = fcu.FluidGrid()
    g.min[:] = [0.0, 0.0, 0.0]
    g.cell = 1.0
    g.dims[:] = list(dims)
    og = orc.OrGrid()
    og.min[:] = [0.0, 0.0, 0.0]
    og.cell = 1.0
    og.dims[:] = list(dims)
    rng = np.random.default_rng(passes)
    n = 300_000
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(0, 1, (n, 3)) * np.array(dims, np.float32)
    # a third of the points in a few cells: runs longer than a 4,096-key tile
    k = n // 3
    pos[:k, :3] = (rng.integers(0, 3, (k, 3)) + 0.5).astype(np.float32)
    starts, perm = fcu.grid_build_host(pos, g)
    _, e_starts, e_perm = orc.grid_build(og, pos)
    assert np.array_equal(starts, e_starts)
    assert np.array_equal(perm, e_perm)


@pytest.mark.parametrize("n", [1, 4095, 4096, 4097, 3 * 4096 + 5])
def test_grid_of_one_cell_at_tile_boundaries(orc, fcu, n):
    """Every key equal (one cell): the run of keys spans every tile, so each
    tile's end of it is a candidate run end and only the last one counts."""
    g = fcu.FluidGrid()
    g.min[:] = [0.0, 0.0, 0.0]
    g.cell = 1.0
    g.dims[:] = [1, 1, 1]
    og = orc.OrGrid()
    og.min[:] = [0.0, 0.0, 0.0]
    og.cell = 1.0
    og.dims[:] = [1, 1, 1]
    pos = np.random.default_rng(n).uniform(-2, 3, (n, 4)).astype(np.float32)
    starts, perm = fcu.grid_build_host(pos, g)
    _, e_starts, e_perm = orc.grid_build(og, pos)
    assert list(starts) == [0, n] and np.array_equal(starts, e_starts)
    assert np.array_equal(perm, e_perm) and np.array_equal(perm, np.arange(n, dtype=perm.dtype))
