"""ctypes view of the CPU oracle (oracle/fluid_oracle.cpp).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, as the checker. The product never imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libfluid_oracle.so")
LIB64_PATH = os.path.join(HERE, "_build", "libfluid_oracle64.so")

FIELD = dict(density=0, alpha=1, kd=2, pressure=3, nbr_n=4, starts=5, perm=6, work_pos=7,
             work_vel=8, accel=9, xsph=10, wall_grad=11, counters=12, work_prev_vel=13,
             work_prev_p=14, work_temp=15, pinc=16, nbr=17)
KERNEL = dict(density=0, div_apply=1, div_kappa=2, forces_eval=3, forces_apply=4, den_kappa=5,
              den_apply=6, integrate=7)


class OrGrid(C.Structure):
    _fields_ = [("min", C.c_float * 3), ("cell", C.c_float), ("dims", C.c_uint32 * 3)]


class OrParams(C.Structure):
    _fields_ = [("box_min", C.c_float * 3), ("cell", C.c_float), ("dims", C.c_uint32 * 3),
                ("count", C.c_uint32), ("h", C.c_float), ("mass", C.c_float),
                ("rho0", C.c_float), ("inv_h", C.c_float), ("sigma", C.c_float),
                ("sigma_h", C.c_float), ("support_sq", C.c_float), ("wall_lo", C.c_float * 3),
                ("wall_hi", C.c_float * 3), ("tracer_c", C.c_float * 3),
                ("tracer_e", C.c_float * 3), ("xsph_blend", C.c_float), ("nbr_cap", C.c_uint32)]


class OrStep(C.Structure):
    _fields_ = [("force", C.c_float * 3), ("dt", C.c_float), ("omega", C.c_float * 3),
                ("v_clamp", C.c_float), ("domega", C.c_float * 3), ("seed", C.c_uint32),
                ("touch_r", C.c_float), ("touch_n", C.c_uint32), ("pad", C.c_uint32 * 2),
                ("touches", (C.c_float * 4) * 5)]


assert C.sizeof(OrStep) == 144


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None
_lib64 = None


def lib():
    """The oracle (binary32, the CUDA path's bit-for-bit reference)."""
    global _lib
    if _lib is None:
        _lib = load_library(LIB_PATH)
    return _lib


def lib64():
    """The FP64 oracle: the same source with every substep operation in
    double (same C API, float in and out, plus or_sim_get_state64)."""
    global _lib64
    if _lib64 is None:
        _lib64 = load_library(LIB64_PATH)
    return _lib64


def load_library(path):
    if not os.path.exists(path):
        build()
    L = C.CDLL(path)
    f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
    u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
    F, U, D = C.c_float, C.c_uint32, C.c_double
    sig = {
        "or_hash": (U, [U]),
        "or_kernel": (F, [F, F]),
        "or_wall_density": (F, [F]),
        "or_wall_gradient": (F, [F]),
        "or_wedge64": (D, [D, D]),
        "or_wedge_d64": (D, [D, D]),
        "or_wall_adhesion64": (D, [D]),
        "or_wedge": (F, [F, F]),
        "or_wedge_d": (F, [F, F]),
        "or_wall_adhesion": (F, [F]),
        "or_half_bits": (C.c_uint16, [F]),
        "or_half_value": (F, [C.c_uint16]),
        "or_slab_depth": (F, []),
        "or_rest_density": (F, []),
        "or_cell_of": (U, [C.POINTER(OrGrid), f32p]),
        "or_grid_slab": (None, [f32p, F, C.POINTER(OrGrid)]),
        "or_grid_box": (None, [f32p, f32p, F, C.POINTER(OrGrid)]),
        "or_grid_build": (None, [C.POINTER(OrGrid), f32p, U, C.c_void_p, u32p, u32p]),
        "or_lattice_dims": (None, [F, f32p, F, u32p]),
        "or_seed_slab": (U, [F, f32p, F, C.c_void_p]),
        "or_seed_tracers": (None, [U, f32p, F, u32p]),
        "or_seed_block": (U, [f32p, F, u32p, F, C.c_uint64, C.c_void_p]),
        "or_seed_tracers_box": (None, [U, f32p, f32p, f32p, f32p, u32p]),
        "or_pack_tracer": (None, [f32p, F, f32p, u32p]),
        "or_unpack_tracer": (None, [u32p, f32p, f32p]),
        "or_pack_step": (None, [f32p, f32p, f32p, F, F, U, U, F, C.c_void_p,
                                np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")]),
        "or_pack_sim_params": (None, [C.POINTER(OrGrid), U, F, F, F,
                                      np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")]),
        "or_params_slab": (None, [f32p, F, F, U, C.POINTER(OrParams)]),
        "or_params_box": (None, [f32p, f32p, F, F, F, U, C.POINTER(OrParams)]),
        "or_sim_new": (C.c_void_p, [C.POINTER(OrParams), U]),
        "or_sim_free": (None, [C.c_void_p]),
        "or_sim_set_threads": (None, [C.c_int]),
        "or_sim_slabs": (U, []),
        "or_sim_set_state": (None, [C.c_void_p] + [C.c_void_p] * 6),
        "or_sim_get_state": (None, [C.c_void_p] + [C.c_void_p] * 6),
        "or_sim_set_tracers": (None, [C.c_void_p, u32p]),
        "or_sim_get_tracers": (None, [C.c_void_p, u32p]),
        "or_sim_substep": (None, [C.c_void_p, C.POINTER(OrStep), U, U]),
        "or_sim_substep_tol": (None, [C.c_void_p, C.POINTER(OrStep), F, F, U, u32p,
                                      np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")]),
        "or_sim_stats": (None, [C.c_void_p, f32p]),
        "or_sim_tracers": (None, [C.c_void_p, C.POINTER(OrStep)]),
        "or_sim_advect": (None, [C.c_void_p, C.POINTER(OrStep)]),
        "or_sim_field": (None, [C.c_void_p, C.c_int, C.c_void_p]),
        "or_field_splat": (None, [C.c_void_p] * 4 + [U, f32p, U, U, U, F, f32p]),
        "or_field_filter": (None, [f32p, U, U, F, F, f32p]),
        "or_sim_get_state64": (None, [C.c_void_p, C.c_void_p, C.c_void_p]),
        "or_sim_real_bytes": (C.c_int, []),
        "or_sim_kernel": (D, [C.c_void_p, C.c_int, C.POINTER(OrStep)]),
        "or_det_exp": (F, [F]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    return L


def f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def make_step(force=(0.0, 0.0, 0.0), dt=0.0, omega=(0.0, 0.0, 0.0), v_clamp=0.0,
              domega=(0.0, 0.0, 0.0), seed=0, touch_r=0.0, touches=()):
    st = OrStep()
    st.force[:] = [float(v) for v in force]
    st.dt = dt
    st.omega[:] = [float(v) for v in omega]
    st.v_clamp = v_clamp
    st.domega[:] = [float(v) for v in domega]
    st.seed = seed
    st.touch_r = touch_r
    st.touch_n = len(touches)
    for i, t in enumerate(touches):
        st.touches[i][:] = [float(v) for v in t]
    return st


def grid_slab(extent, support):
    g = OrGrid()
    lib().or_grid_slab(f32(extent), support, C.byref(g))
    return g


def grid_box(lo, hi, support):
    g = OrGrid()
    lib().or_grid_box(f32(lo), f32(hi), support, C.byref(g))
    return g


def cell_count(g):
    return g.dims[0] * g.dims[1] * g.dims[2]


def grid_build(g, pos4):
    """Stable counting sort: (keys, starts[C+1], perm)."""
    pos4 = f32(pos4).reshape(-1, 4)
    n = pos4.shape[0]
    keys = np.zeros(n, np.uint32)
    starts = np.zeros(cell_count(g) + 1, np.uint32)
    perm = np.zeros(n, np.uint32)
    lib().or_grid_build(C.byref(g), pos4, n, _ptr(keys), starts, perm)
    return keys, starts, perm


def seed_slab(spacing, extent, fill=0.5):
    e = f32(extent)
    n = lib().or_seed_slab(spacing, e, fill, None)
    out = np.zeros((n, 4), np.float32)
    lib().or_seed_slab(spacing, e, fill, _ptr(out))
    return out


def seed_block(lo, spacing, dims, jitter, seed):
    n = int(np.prod(dims))
    out = np.zeros((n, 4), np.float32)
    lib().or_seed_block(f32(lo), spacing, u32(dims), jitter, seed, _ptr(out))
    return out


def seed_tracers_box(count, lo, size, params):
    """Packed tracers uniform over [lo, lo + size) of a box (params_box)."""
    out = np.zeros(2 * count, np.uint32)
    e = f32([params.tracer_e[0], params.tracer_e[1]])
    lib().or_seed_tracers_box(count, f32(lo), f32(size), f32(list(params.tracer_c)), e, out)
    return out.reshape(-1, 2)


def params_slab(extent, spacing, h_ratio, count):
    p = OrParams()
    lib().or_params_slab(f32(extent), spacing, h_ratio, count, C.byref(p))
    return p


def params_box(lo, hi, spacing, h_ratio, rho0, count):
    p = OrParams()
    lib().or_params_box(f32(lo), f32(hi), spacing, h_ratio, rho0, count, C.byref(p))
    return p


class Sim:
    """The oracle's substep over a resting set, in slot order. fp64=True runs
    the FP64 oracle (state() still returns float32; state64() the doubles);
    library= a loaded oracle library of either kind."""

    def __init__(self, params, tracers=0, fp64=False, library=None):
        self.L = library if library is not None else (lib64() if fp64 else lib())
        self.p = params
        self.n = params.count
        self.cells = params.dims[0] * params.dims[1] * params.dims[2]
        self.ntr = tracers
        self.h = self.L.or_sim_new(C.byref(params), tracers)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.or_sim_free(self.h)
            self.h = None

    def set_state(self, pos4=None, vel4=None, prev_vel4=None, prev_p=None, temp=None, ids=None):
        conv = lambda a, k: None if a is None else (f32(a) if k == "f" else u32(a))
        arrs = [conv(pos4, "f"), conv(vel4, "f"), conv(prev_vel4, "f"), conv(prev_p, "f"),
                conv(temp, "f"), conv(ids, "u")]
        self.L.or_sim_set_state(self.h, *[_ptr(a) for a in arrs])

    def state(self):
        n = self.n
        out = dict(pos=np.zeros((n, 4), np.float32), vel=np.zeros((n, 4), np.float32),
                   prev_vel=np.zeros((n, 4), np.float32), prev_p=np.zeros(n, np.float32),
                   temp=np.zeros(n, np.float32), id=np.zeros(n, np.uint32))
        self.L.or_sim_get_state(self.h, *[_ptr(out[k]) for k in
                                         ("pos", "vel", "prev_vel", "prev_p", "temp", "id")])
        return out

    def state64(self):
        n = self.n
        pos, vel = np.zeros((n, 4), np.float64), np.zeros((n, 4), np.float64)
        self.L.or_sim_get_state64(self.h, _ptr(pos), _ptr(vel))
        return dict(pos=pos, vel=vel)

    def set_tracers(self, packed):
        self.L.or_sim_set_tracers(self.h, u32(packed).reshape(-1))

    def tracers(self):
        out = np.zeros(2 * self.ntr, np.uint32)
        self.L.or_sim_get_tracers(self.h, out)
        return out.reshape(-1, 2)

    def substep(self, step, div_iters=1, den_iters=5):
        self.L.or_sim_substep(self.h, C.byref(step), div_iters, den_iters)

    def substep_tol(self, step, div_tol, den_tol, max_iters=100):
        iters = np.zeros(2, np.uint32)
        res = np.zeros(2, np.float64)
        self.L.or_sim_substep_tol(self.h, C.byref(step), div_tol, den_tol, max_iters, iters, res)
        return iters, res

    def stats(self):
        out = np.zeros(14, np.float32)
        self.L.or_sim_stats(self.h, out)
        return out

    def tracer_pass(self, step):
        self.L.or_sim_tracers(self.h, C.byref(step))

    def advect(self, step):
        self.L.or_sim_advect(self.h, C.byref(step))

    def field(self, name):
        n = self.n
        shapes = dict(density=(n, np.float32), alpha=(n, np.float32), kd=(n, np.float32),
                      pressure=(n, np.float32), nbr_n=(n, np.uint32),
                      starts=(self.cells * sim_slabs() + 1, np.uint32), perm=(n, np.uint32),
                      work_pos=((n, 4), np.float32), work_vel=((n, 4), np.float32),
                      accel=((n, 4), np.float32), xsph=((n, 4), np.float32),
                      wall_grad=((n, 4), np.float32), counters=(2, np.uint32),
                      work_prev_vel=((n, 4), np.float32), work_prev_p=(n, np.float32),
                      work_temp=(n, np.float32), pinc=(n, np.float32),
                      nbr=((n, self.p.nbr_cap), np.uint32))
        shape, dt = shapes[name]
        out = np.zeros(shape, dt)
        self.L.or_sim_field(self.h, FIELD[name], _ptr(out))
        return out

    def kernel(self, name, step):
        """One kernel of the substep on the working set (or_sim_kernel)."""
        return self.L.or_sim_kernel(self.h, KERNEL[name], C.byref(step))


def set_threads(n):
    lib().or_sim_set_threads(n)


def sim_slabs():
    """Slabs per cell along x in a simulation's grid keys."""
    return int(lib().or_sim_slabs())


def field_splat(pos4, vel4, pvel4, density, geom, w, h, lens, keep, field2=None):
    """The body splat with the decay draw over the given resting state;
    returns the new field [h][w][2] (starting from `field2` or zeros)."""
    pos4, vel4, pvel4 = f32(pos4), f32(vel4), f32(pvel4)
    density = f32(density)
    out = np.zeros((h, w, 2), np.float32) if field2 is None else f32(field2).copy()
    lib().or_field_splat(_ptr(pos4), _ptr(vel4), _ptr(pvel4), _ptr(density), len(pos4),
                         f32(geom), w, h, lens, keep, out)
    return out


def field_filter(field2, ex, ey):
    h, w = field2.shape[:2]
    out = np.zeros((h, w, 4), np.float32)
    lib().or_field_filter(f32(field2), w, h, ex, ey, out)
    return out



# ---- the frame's substep policy (render.rs:57-106), restated ----------------
# The reference picks each frame's substep count on the host from the
# one-frame-stale v_max (render.rs:3090-3094). Float32 arithmetic as Rust's
# f32, `as u32` saturating.
_F = np.float32


def _sat_u32(v):
    v = float(v)
    if not v > 0.0:
        return 0
    return 0xFFFFFFFF if v >= 4294967296.0 else int(v)


def refine_passes(dt_sub):
    return 5 if _F(dt_sub) > _F(0.00105) else 2


def substep_floor(dt, dt_sub_max):
    return min(_sat_u32(np.ceil(_F(dt) / _F(dt_sub_max))), 8)


def substeps_for(dt, v_max, spacing, cap):
    dt, v_max, spacing = _F(dt), _F(v_max), _F(spacing)
    n = _sat_u32(np.ceil(dt * v_max / (_F(0.4) * spacing)))
    n = max(n, substep_floor(dt, _F(0.42) * spacing))
    cheap = _sat_u32(np.ceil(_F(1.0) / _F(120.0) / _F(0.00105)))
    jump = refine_passes(dt / _F(cheap)) == 2 and n < cheap and _F(n) > _F(0.65) * _F(cheap)
    if jump:
        n = cheap
    return min(n, cap)
