"""A plain-C host drives the library through include/fluid_cu.h alone.

tests/c_host/frame_driver.c is what a native host (C, or a Rust/Go/Swift
binding generated from the header) links against in place of the reference's
fluid_renderer_* entry points (crates/fluid-ffi/src/lib.rs). The CPU test compiles
it as strict C11 and links it against libfluidcu.so, which shows the header
is valid C with every declaration resolved by the library. The GPU test runs
it and compares what it reads back with the same frames driven through the
ctypes binding, bit for bit."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "fluid-simulation-app_b200")
FRAMES = 30


def _compile(tmp_path):
    exe = str(tmp_path / "frame_driver")
    cmd = ["gcc", "-std=c11", "-Wall", "-Wextra", "-Werror", "-pedantic",
           "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "c_host",
                                                             "frame_driver.c"),
           "-L", LIBDIR, "-lfluidcu", "-Wl,-rpath," + LIBDIR, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_header_compiles_as_c11_and_links(fcu, tmp_path):
    assert os.path.exists(_compile(tmp_path))


@pytest.mark.gpu
def test_c_host_matches_the_ctypes_path(fcu, tmp_path):
    exe = _compile(tmp_path)
    out = str(tmp_path / "particles.bin")
    r = subprocess.run([exe, str(FRAMES), out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    f = r.stdout.split()
    got = dict(zip(f[0::2], f[1::2]))

    with fcu.Sim() as sim:
        for k in range(FRAMES):
            sim.frame((0.0, -9.81, 0.0), 1.0 / 120.0, substeps=0, cap=16, seed=k)
        st = sim.stats()
        pos, vel = sim.read_particles()
        n = sim.n
    bits = lambda v: "%08x" % int(np.float32(v).view(np.uint32))
    assert int(got["n"]) == n
    assert int(got["substeps"]) == st.substeps and st.substeps >= FRAMES
    assert got["compression_avg"] == bits(st.compression_avg)
    assert got["v_max"] == bits(st.v_max)
    raw = np.fromfile(out, np.float32).reshape(2, n, 4)
    assert raw[0].view(np.uint32).tobytes() == pos.view(np.uint32).tobytes()
    assert raw[1].view(np.uint32).tobytes() == vel.view(np.uint32).tobytes()
