"""FP32 error of the substep against the FP64 oracle (test infrastructure).

The dam-break workload (32x16x32 lattice, 16,384 particles, unit box,
spacing 0.01, h = 1.2 spacing, rho0 1000, XSPH 0.01, gravity (0, -9.81, 0),
two substeps per 1/120 s frame, tolerance solve 1 % / 0.1 %) runs in the
binary32 oracle, which the CUDA path matches bit for bit, and in the FP64
oracle (the same source compiled with every substep operation in double)
replaying the binary32 run's iteration counts substep by substep, so the
two differ by rounding alone. Prints, per frame, the largest and the RMS
position difference in units of the spacing, the RMS velocity difference
relative to the RMS speed, the centre-of-mass difference in spacings, and
both runs' mean compression (mean max(rho / rho0 - 1, 0)).

    python oracle/fp64_error.py [frames]
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from oracle import oracle as orc  # noqa: E402

SPACING = 0.01
LATTICE = (32, 16, 32)
SUBSTEPS = 2
F32 = np.float32


def dam_break(fp64):
    n = int(np.prod(LATTICE))
    p = orc.params_box([0, 0, 0], [1, 1, 1], SPACING, 1.2, 1000.0, n)
    p.xsph_blend = 0.01
    s = orc.Sim(p, 0, fp64=fp64)
    pos = orc.seed_block([0, 0, 0], SPACING, list(LATTICE), 0.005, 1)
    s.set_state(pos4=pos, temp=np.full(n, 293.15, np.float32))
    return s


def by_id(state, ids=None):
    """Positions and velocities (xyz, float64) in particle-id order: the
    two runs' slot orders part as soon as one particle lands in another
    cell."""
    ids = state["id"] if ids is None else ids
    order = np.argsort(ids)
    return {k: np.asarray(state[k], np.float64)[order, :3] for k in ("pos", "vel")}


def run(frames, report=None):
    a, b = dam_break(False), dam_break(True)
    dt = float(F32(F32(1.0 / 120.0) / F32(SUBSTEPS)))
    vc = float(F32(0.4) * F32(SPACING) / F32(dt))
    st = orc.make_step(force=(0.0, -9.81, 0.0), dt=dt, v_clamp=vc)
    rows = []
    for f in range(frames):
        for _ in range(SUBSTEPS):
            it, _ = a.substep_tol(st, 0.01, 0.001, 100)
            b.substep(st, int(it[0]), int(it[1]))
        x32, x64 = by_id(a.state()), by_id(b.state64(), b.state()["id"])
        dx = np.linalg.norm(x32["pos"] - x64["pos"], axis=1)
        dv = np.linalg.norm(x32["vel"] - x64["vel"], axis=1)
        vrms = np.sqrt(np.mean(np.sum(x64["vel"] ** 2, axis=1)))
        com = np.linalg.norm(x32["pos"].mean(axis=0) - x64["pos"].mean(axis=0))
        c32, c64 = a.stats()[0], b.stats()[0]
        row = (f + 1, dx.max() / SPACING, np.sqrt(np.mean(dx ** 2)) / SPACING,
               np.sqrt(np.mean(dv ** 2)) / max(vrms, 1e-30), com / SPACING, c32, c64)
        rows.append(row)
        if report:
            report(row)
    return rows


if __name__ == "__main__":
    frames = int(sys.argv[1]) if len(sys.argv) > 1 else 60
    print("frame  max|dx|/spacing  rms|dx|/spacing  rms|dv|/rms|v|  |dCOM|/spacing  compr. FP32  compr. FP64")
    run(frames, lambda r: print("%5d  %15.3e  %15.3e  %14.3e  %13.3e  %11.3e  %11.3e" % r, flush=True))
