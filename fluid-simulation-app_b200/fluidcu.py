"""ctypes binding of libfluidcu.so (include/fluid_cu.h).

The host-side view of the C ABI that tests, the benchmark and any Python
caller use. It mirrors the reference's sim-facing interface (Renderer::new /
frame / stats / set_particles, crates/fluid-core/src/render.rs:2801-3576, and
the C ABI of crates/fluid-ffi) minus drawing. There is no CPU fallback: if
the CUDA library is missing this module raises on import of the library.
"""
import ctypes as C
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfluidcu.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "fluid_cu.h")

OK, ERR_ARG, ERR_CUDA, ERR_TIMEOUT, ERR_NAN, ERR_STATE, ERR_OOM = 0, -1, -2, -3, -4, -5, -6
GEOMETRY_SLAB, GEOMETRY_BOX = 0, 1
SEED_SLAB, SEED_BLOCK, SEED_NONE = 0, 1, 2
SOLVE_FIXED, SOLVE_TOLERANCE = 0, 1
FIELDS = dict(density=0, alpha=1, kd=2, pressure=3, nbr_n=4, starts=5, perm=6, work_pos=7,
              work_vel=8, accel=9, xsph=10, wall_grad=11, counters=12)


class FluidVec3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class FluidStep(C.Structure):
    _fields_ = [("force", C.c_float * 3), ("dt", C.c_float), ("omega", C.c_float * 3),
                ("v_clamp", C.c_float), ("domega", C.c_float * 3), ("seed", C.c_uint32),
                ("touch_r", C.c_float), ("touch_n", C.c_uint32), ("pad", C.c_uint32 * 2),
                ("touches", (C.c_float * 4) * 5)]


class FluidSimConfig(C.Structure):
    _fields_ = [("geometry", C.c_uint32), ("extent", C.c_float * 2), ("box_lo", C.c_float * 3),
                ("box_hi", C.c_float * 3), ("spacing", C.c_float), ("h_ratio", C.c_float),
                ("rest_density", C.c_float), ("seeding", C.c_uint32), ("fill", C.c_float),
                ("block", C.c_uint32 * 3), ("jitter", C.c_float), ("seed", C.c_uint64),
                ("count", C.c_uint32), ("tracers", C.c_uint32), ("xsph_blend", C.c_float),
                ("temperature", C.c_float), ("solve", C.c_uint32), ("div_iters", C.c_uint32),
                ("den_iters", C.c_uint32), ("div_tol", C.c_float), ("den_tol", C.c_float),
                ("max_iters", C.c_uint32), ("nbr_cap", C.c_uint32), ("device", C.c_int32)]


class FluidSimParams(C.Structure):
    _fields_ = [("box_min", C.c_float * 3), ("cell", C.c_float), ("dims", C.c_uint32 * 3),
                ("count", C.c_uint32), ("h", C.c_float), ("mass", C.c_float),
                ("rho0", C.c_float), ("inv_h", C.c_float), ("sigma", C.c_float),
                ("sigma_h", C.c_float), ("support_sq", C.c_float), ("wall_lo", C.c_float * 3),
                ("wall_hi", C.c_float * 3), ("tracer_c", C.c_float * 3),
                ("tracer_e", C.c_float * 3), ("xsph_blend", C.c_float), ("nbr_cap", C.c_uint32)]


class FluidSimStats(C.Structure):
    _fields_ = [("compression_avg", C.c_float), ("compression_max", C.c_float),
                ("density_min", C.c_float), ("density_max", C.c_float),
                ("pressure_min", C.c_float), ("pressure_max", C.c_float), ("v_max", C.c_float),
                ("temperature_min", C.c_float), ("temperature_max", C.c_float),
                ("clamp_count", C.c_uint32), ("neighbour_overflow", C.c_uint32),
                ("v_min", C.c_float), ("accel_min", C.c_float), ("accel_max", C.c_float),
                ("div_iters", C.c_uint32), ("den_iters", C.c_uint32),
                ("div_residual", C.c_double), ("den_residual", C.c_double),
                ("substeps", C.c_uint64), ("total_div_iters", C.c_uint64),
                ("total_den_iters", C.c_uint64), ("substeps_last_frame", C.c_uint32),
                ("error", C.c_int32)]

    def as_reference_block(self):
        """The 14-float stats block of sim_solve.wgsl:800-874, in its slot order."""
        return np.array([self.compression_avg, self.compression_max, self.density_min,
                         self.density_max, self.pressure_min, self.pressure_max, self.v_max,
                         self.temperature_min, self.temperature_max, float(self.clamp_count),
                         float(self.neighbour_overflow), self.v_min, self.accel_min,
                         self.accel_max], np.float32)


class FluidGrid(C.Structure):
    _fields_ = [("min", C.c_float * 3), ("cell", C.c_float), ("dims", C.c_uint32 * 3)]


class FluidFieldParams(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("keep", C.c_float),
                ("lens", C.c_uint32), ("lo", C.c_float), ("hi", C.c_float)]


class FluidMotion(C.Structure):
    _fields_ = [("gravity", FluidVec3), ("user_acceleration", FluidVec3),
                ("rotation_rate", FluidVec3)]


class FluidFramePlan(C.Structure):
    _fields_ = [("step", FluidStep), ("force", FluidVec3), ("omega", FluidVec3),
                ("domega", FluidVec3), ("dt", C.c_float), ("deviation", C.c_float),
                ("substeps", C.c_uint32), ("refine", C.c_uint32), ("seed", C.c_uint32),
                ("asleep", C.c_uint32), ("frames", C.c_uint64), ("idle_frames", C.c_uint64)]


assert C.sizeof(FluidStep) == 144


def header_functions():
    """Names of the functions include/fluid_cu.h declares."""
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fluid_[a-z0-9_]+)\s*\(", text)))


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it (make -C fluid-simulation-app_b200); "
                           "there is no CPU fallback")
    L = C.CDLL(LIB_PATH)
    P = C.c_void_p
    vp = C.c_void_p
    i32, u32, u64, f = C.c_int32, C.c_uint32, C.c_uint64, C.c_float
    sig = {
        "fluid_last_error": (C.c_char_p, []),
        "fluid_sim_default_config": (None, [C.POINTER(FluidSimConfig)]),
        "fluid_sim_create": (P, [C.POINTER(FluidSimConfig)]),
        "fluid_sim_destroy": (None, [P]),
        "fluid_sim_params": (i32, [P, C.POINTER(FluidSimParams)]),
        "fluid_sim_count": (u32, [P]),
        "fluid_sim_tracer_count": (u32, [P]),
        "fluid_sim_stream": (vp, [P]),
        "fluid_sim_step": (i32, [P, C.POINTER(FluidStep)]),
        "fluid_sim_run": (i32, [P, C.POINTER(FluidStep), u32]),
        "fluid_sim_reduce_stats": (i32, [P]),
        "fluid_sim_tracers": (i32, [P, C.POINTER(FluidStep)]),
        "fluid_sim_advect": (i32, [P, C.POINTER(FluidStep)]),
        "fluid_sim_frame": (i32, [P, FluidVec3, FluidVec3, FluidVec3, f, u32, u32, u32]),
        "fluid_sim_sync": (i32, [P]),
        "fluid_sim_stats": (i32, [P, C.POINTER(FluidSimStats)]),
        "fluid_sim_get_state": (i32, [P, vp, vp, vp, vp, vp, vp]),
        "fluid_sim_set_state": (i32, [P, vp, vp, vp, vp, vp, vp]),
        "fluid_sim_read_particles": (i32, [P, vp, vp]),
        "fluid_sim_get_tracers": (i32, [P, vp]),
        "fluid_sim_set_tracers": (i32, [P, vp]),
        "fluid_sim_read_field": (i32, [P, i32, vp, u64]),
        "fluid_sim_field_splat": (i32, [P, C.POINTER(FluidFieldParams)]),
        "fluid_sim_field_filter": (i32, [P]),
        "fluid_sim_field_read": (i32, [P, vp, vp]),
        "fluid_field_keep_target": (f, [f]),
        "fluid_sim_profile_step": (i32, [P, C.POINTER(FluidStep), C.POINTER(f),
                                         C.POINTER(C.c_char_p), u32]),
        "fluid_sim_kernels_per_substep": (u32, [P]),
        "fluid_sim_grid_slabs": (u32, []),
        "fluid_grid_workspace_bytes": (u64, [u32, C.POINTER(FluidGrid)]),
        "fluid_grid_build": (i32, [vp, u32, C.POINTER(FluidGrid), vp, vp, vp, vp, u64, vp]),
        "fluid_grid_build_host": (i32, [vp, u32, C.POINTER(FluidGrid), vp, vp]),
        "fluid_grid_build_static": (i32, [vp, u32, C.POINTER(FluidGrid), vp, vp, vp, vp]),
        "fluid_grid_build_status": (i32, [vp, u32, C.POINTER(FluidGrid), vp]),
        "fluid_grid_build_static_status": (i32, [vp]),
        "fluid_selftest_static_radix_wait": (i32, [i32, C.POINTER(C.c_float)]),
        "fluid_selftest_scan_wait": (i32, [i32, C.POINTER(C.c_float)]),
        "fluid_selftest_radix_wait": (i32, [i32, C.POINTER(C.c_float)]),
        "fluid_batch_create": (P, [C.POINTER(FluidSimConfig), u32]),
        "fluid_batch_destroy": (None, [P]),
        "fluid_batch_boxes": (u32, [P]),
        "fluid_batch_count": (u32, [P, u32]),
        "fluid_batch_total": (u32, [P]),
        "fluid_batch_stream": (P, [P]),
        "fluid_batch_params": (i32, [P, u32, C.POINTER(FluidSimParams)]),
        "fluid_batch_step": (i32, [P, C.POINTER(FluidStep)]),
        "fluid_batch_run": (i32, [P, C.POINTER(FluidStep), u32]),
        "fluid_batch_reduce_stats": (i32, [P]),
        "fluid_batch_stats": (i32, [P, C.POINTER(FluidSimStats)]),
        "fluid_batch_sync": (i32, [P]),
        "fluid_batch_get_state": (i32, [P, u32, vp, vp, vp, vp, vp, vp]),
        "fluid_batch_autotune": (i32, [P, C.POINTER(FluidStep), vp, vp]),
        "fluid_batch_set_blocks": (i32, [P, vp]),
        "fluid_batch_get_blocks": (i32, [P, vp]),
        "fluid_adjoint_create": (P, [C.POINTER(FluidSimConfig), u32, u32, f, f, u32, u32]),
        "fluid_adjoint_destroy": (None, [P]),
        "fluid_adjoint_count": (u32, [P]),
        "fluid_adjoint_forward": (i32, [P, vp, C.c_double, vp, vp]),
        "fluid_adjoint_backward": (i32, [P, vp, vp]),
        "fluid_adjoint_get_schedule": (i32, [P, vp, vp]),
        "fluid_adjoint_set_schedule": (i32, [P, vp, vp]),
        "fluid_adjoint_final_state": (i32, [P, vp, vp]),
        "fluid_adjoint_timing": (i32, [P, vp, vp]),
        "fluid_substep_floor": (u32, [f, f]),
        "fluid_refine_passes": (u32, [f]),
        "fluid_substeps_for": (u32, [f, f, f, u32]),
        "fluid_controller_create": (P, [f, C.POINTER(C.c_float * 2), u32]),
        "fluid_controller_destroy": (None, [P]),
        "fluid_controller_touch": (i32, [P, u32, f, f, u32]),
        "fluid_controller_plan": (i32, [P, C.POINTER(FluidMotion), C.c_double, f,
                                        C.POINTER(FluidFramePlan)]),
        "fluid_sim_frame_plan": (i32, [P, C.POINTER(FluidFramePlan)]),
        "fluid_idle_gate_create": (P, []),
        "fluid_idle_gate_destroy": (None, [P]),
        "fluid_idle_gate_still_frames": (u32, []),
        "fluid_idle_gate_asleep": (u32, [P, u32, C.POINTER(C.c_float * 3), f,
                                         C.POINTER(C.c_float * 3), f]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


class FluidError(RuntimeError):
    def __init__(self, code, what):
        super().__init__(f"{what}: status {code}: {last_error()}")
        self.code = code


def last_error():
    return lib().fluid_last_error().decode()


def check(rc, what):
    if rc != OK:
        raise FluidError(rc, what)
    return rc


def selftest_scan_wait(device=0):
    """Runs the grid scan's bounded wait out (fluid_selftest_scan_wait):
    returns (status, kernel ms); ERR_TIMEOUT is the expected status."""
    ms = C.c_float(0.0)
    rc = lib().fluid_selftest_scan_wait(device, C.byref(ms))
    return rc, ms.value


def selftest_radix_wait(device=0):
    """Runs a radix digit pass's bounded look-back out
    (fluid_selftest_radix_wait): returns (status, kernel ms); ERR_TIMEOUT is
    the expected status."""
    ms = C.c_float(0.0)
    rc = lib().fluid_selftest_radix_wait(device, C.byref(ms))
    return rc, ms.value


def selftest_static_radix_wait(device=0):
    """The same stalled digit pass on fluid_grid_build_static's fixed
    scratch, read back through fluid_grid_build_static_status."""
    ms = C.c_float(0.0)
    rc = lib().fluid_selftest_static_radix_wait(device, C.byref(ms))
    return rc, ms.value


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def default_config(**kw):
    cfg = FluidSimConfig()
    lib().fluid_sim_default_config(C.byref(cfg))
    for k, v in kw.items():
        fld = getattr(cfg, k)
        if isinstance(fld, C.Array):
            fld[:] = list(v)
        else:
            setattr(cfg, k, v)
    return cfg


def make_step(force=(0.0, 0.0, 0.0), dt=0.0, omega=(0.0, 0.0, 0.0), v_clamp=0.0,
              domega=(0.0, 0.0, 0.0), seed=0, touch_r=0.0, touches=()):
    """pack_step (sim.rs:215-252) as a struct."""
    st = FluidStep()
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


class Adjoint:
    """The differentiable model and its adjoint: the handle of fluid_adjoint_create."""

    def __init__(self, cfg, frames, substeps_per_frame, frame_dt, v_clamp, checkpoint_every=10,
                 precision=32):
        h = lib().fluid_adjoint_create(C.byref(cfg), frames, substeps_per_frame, frame_dt, v_clamp,
                                       checkpoint_every, precision)
        if not h:
            raise FluidError(ERR_ARG, "fluid_adjoint_create: " + lib().fluid_last_error().decode())
        self.h = h
        self.frames = frames
        self.substeps = frames * substeps_per_frame
        self.n = lib().fluid_adjoint_count(h)

    def close(self):
        if getattr(self, "h", None):
            lib().fluid_adjoint_destroy(self.h)
            self.h = None

    def __del__(self):
        # at interpreter exit the module's globals may already be gone; the
        # process's CUDA context goes with it
        try:
            self.close()
        except (TypeError, AttributeError):
            pass

    def forward(self, forces, xsph, target):
        f = np.ascontiguousarray(forces, np.float64).reshape(self.frames, 3)
        t = np.ascontiguousarray(target, np.float64).reshape(3)
        loss = C.c_double(0.0)
        check(lib().fluid_adjoint_forward(self.h, _p(f), float(xsph), _p(t), C.byref(loss)),
              "adjoint_forward")
        return loss.value

    def backward(self):
        g = np.zeros((self.frames, 3), np.float64)
        gx = C.c_double(0.0)
        check(lib().fluid_adjoint_backward(self.h, _p(g), C.byref(gx)), "adjoint_backward")
        return g, gx.value

    def schedule(self):
        d = np.zeros(self.substeps, np.uint32)
        e = np.zeros(self.substeps, np.uint32)
        check(lib().fluid_adjoint_get_schedule(self.h, _p(d), _p(e)), "adjoint_get_schedule")
        return d, e

    def set_schedule(self, div_iters, den_iters):
        d = np.ascontiguousarray(div_iters, np.uint32)
        e = np.ascontiguousarray(den_iters, np.uint32)
        check(lib().fluid_adjoint_set_schedule(self.h, _p(d), _p(e)), "adjoint_set_schedule")

    def final_state(self):
        p = np.zeros((self.n, 3), np.float64)
        v = np.zeros((self.n, 3), np.float64)
        check(lib().fluid_adjoint_final_state(self.h, _p(p), _p(v)), "adjoint_final_state")
        return p, v

    def timing(self):
        a, b = C.c_float(0.0), C.c_float(0.0)
        check(lib().fluid_adjoint_timing(self.h, C.byref(a), C.byref(b)), "adjoint_timing")
        return a.value, b.value


class Batch:
    """Many independent boxes stepped together: the handle of fluid_batch_create."""

    def __init__(self, cfgs):
        arr = (FluidSimConfig * len(cfgs))(*cfgs)
        h = lib().fluid_batch_create(arr, len(cfgs))
        if not h:
            raise FluidError(ERR_ARG, "fluid_batch_create: " + lib().fluid_last_error().decode())
        self.h = h
        self.nboxes = lib().fluid_batch_boxes(h)
        self.counts = [lib().fluid_batch_count(h, b) for b in range(self.nboxes)]
        self.n = lib().fluid_batch_total(h)

    def close(self):
        if getattr(self, "h", None):
            lib().fluid_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        # at interpreter exit the module's globals may already be gone; the
        # process's CUDA context goes with it
        try:
            self.close()
        except (TypeError, AttributeError):
            pass

    def params(self, box):
        p = FluidSimParams()
        check(lib().fluid_batch_params(self.h, box, C.byref(p)), "batch_params")
        return p

    def run(self, steps):
        """steps: a list of substeps, each a list of nboxes FluidStep."""
        flat = [s for sub in steps for s in sub]
        assert len(flat) == len(steps) * self.nboxes
        arr = (FluidStep * len(flat))(*flat)
        return check(lib().fluid_batch_run(self.h, arr, len(steps)), "batch_run")

    def step(self, steps):
        return self.run([steps])

    def reduce_stats(self):
        return check(lib().fluid_batch_reduce_stats(self.h), "batch_reduce_stats")

    def sync(self):
        return check(lib().fluid_batch_sync(self.h), "batch_sync")

    def stream(self):
        return lib().fluid_batch_stream(self.h)

    TUNED = ("density_div", "div_kappa", "apply", "forces_eval", "forces_apply", "den_kappa",
             "integrate")

    def autotune(self, steps):
        """Block size per tuned sweep from one timed substep per candidate
        (64/128/256) of `steps` (nboxes FluidStep); the state is restored."""
        arr = (FluidStep * self.nboxes)(*steps)
        chosen = np.zeros(7, np.uint32)
        ms = np.zeros((3, 7), np.float32)
        check(lib().fluid_batch_autotune(self.h, arr, _p(chosen), _p(ms)), "batch_autotune")
        return dict(zip(self.TUNED, chosen.tolist())), ms

    def set_blocks(self, tpb):
        a = np.ascontiguousarray(tpb, np.uint32)
        check(lib().fluid_batch_set_blocks(self.h, _p(a)), "batch_set_blocks")

    def blocks(self):
        a = np.zeros(7, np.uint32)
        check(lib().fluid_batch_get_blocks(self.h, _p(a)), "batch_get_blocks")
        return a

    def stats(self, allow_error=False):
        arr = (FluidSimStats * self.nboxes)()
        rc = lib().fluid_batch_stats(self.h, arr)
        if not allow_error:
            check(rc, "batch_stats")
        return list(arr)

    def state(self, box):
        n = self.counts[box]
        out = dict(pos=np.zeros((n, 4), np.float32), vel=np.zeros((n, 4), np.float32),
                   prev_vel=np.zeros((n, 4), np.float32), prev_p=np.zeros(n, np.float32),
                   temp=np.zeros(n, np.float32), id=np.zeros(n, np.uint32))
        check(lib().fluid_batch_get_state(self.h, box, *[_p(out[k]) for k in
                                                         ("pos", "vel", "prev_vel", "prev_p",
                                                          "temp", "id")]), "batch_get_state")
        return out


class Sim:
    """One box of fluid on one GPU: the handle of fluid_sim_create."""

    def __init__(self, cfg=None, **kw):
        if cfg is None:
            cfg = default_config(**kw)
        self.cfg = cfg
        h = lib().fluid_sim_create(C.byref(cfg))
        if not h:
            raise FluidError(ERR_ARG, "fluid_sim_create")
        self.h = h
        self.n = lib().fluid_sim_count(h)
        self.ntr = lib().fluid_sim_tracer_count(h)
        self.params = FluidSimParams()
        check(lib().fluid_sim_params(h, C.byref(self.params)), "params")
        d = self.params.dims
        self.cells = d[0] * d[1] * d[2]
        # grid keys: cell * slabs + the x slab (fluid_sim_grid_slabs)
        self.keyspace = self.cells * grid_slabs()

    def close(self):
        if getattr(self, "h", None):
            lib().fluid_sim_destroy(self.h)
            self.h = None

    def __del__(self):
        # at interpreter exit the module's globals may already be gone; the
        # process's CUDA context goes with it
        try:
            self.close()
        except (TypeError, AttributeError):
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def step(self, st):
        return check(lib().fluid_sim_step(self.h, C.byref(st)), "step")

    def run(self, steps):
        arr = (FluidStep * len(steps))(*steps)
        return check(lib().fluid_sim_run(self.h, arr, len(steps)), "run")

    def reduce_stats(self):
        return check(lib().fluid_sim_reduce_stats(self.h), "reduce_stats")

    def tracers_pass(self, st):
        return check(lib().fluid_sim_tracers(self.h, C.byref(st)), "tracers")

    def advect(self, st):
        return check(lib().fluid_sim_advect(self.h, C.byref(st)), "advect")

    def frame(self, force, dt, omega=(0, 0, 0), domega=(0, 0, 0), substeps=0, cap=16, seed=0):
        v = lambda t: FluidVec3(*[float(x) for x in t])
        return check(lib().fluid_sim_frame(self.h, v(force), v(omega), v(domega), dt, substeps,
                                           cap, seed), "frame")

    def frame_plan(self, plan):
        return check(lib().fluid_sim_frame_plan(self.h, C.byref(plan)), "frame_plan")

    def sync(self):
        return check(lib().fluid_sim_sync(self.h), "sync")

    def stats(self, allow_error=False):
        st = FluidSimStats()
        rc = lib().fluid_sim_stats(self.h, C.byref(st))
        if not allow_error:
            check(rc, "stats")
        return st

    def state(self):
        n = self.n
        out = dict(pos=np.zeros((n, 4), np.float32), vel=np.zeros((n, 4), np.float32),
                   prev_vel=np.zeros((n, 4), np.float32), prev_p=np.zeros(n, np.float32),
                   temp=np.zeros(n, np.float32), id=np.zeros(n, np.uint32))
        check(lib().fluid_sim_get_state(self.h, *[_p(out[k]) for k in
                                                  ("pos", "vel", "prev_vel", "prev_p", "temp",
                                                   "id")]), "get_state")
        return out

    def set_state(self, pos4=None, vel4=None, prev_vel4=None, prev_p=None, temp=None, ids=None):
        c = lambda a, dt: None if a is None else np.ascontiguousarray(a, dt)
        arrs = [c(pos4, np.float32), c(vel4, np.float32), c(prev_vel4, np.float32),
                c(prev_p, np.float32), c(temp, np.float32), c(ids, np.uint32)]
        return check(lib().fluid_sim_set_state(self.h, *[_p(a) for a in arrs]), "set_state")

    def read_particles(self):
        pos = np.zeros((self.n, 4), np.float32)
        vel = np.zeros((self.n, 4), np.float32)
        check(lib().fluid_sim_read_particles(self.h, _p(pos), _p(vel)), "read_particles")
        return pos, vel

    def tracers(self):
        out = np.zeros((max(self.ntr, 0), 2), np.uint32)
        check(lib().fluid_sim_get_tracers(self.h, _p(out)), "get_tracers")
        return out

    def set_tracers(self, packed):
        packed = np.ascontiguousarray(packed, np.uint32)
        check(lib().fluid_sim_set_tracers(self.h, _p(packed)), "set_tracers")

    def field_splat(self, width, height, keep=0.0, lens=0, lo=0.0, hi=1.0):
        p = FluidFieldParams(width, height, keep, lens, lo, hi)
        self._field_shape = (height, width)
        return check(lib().fluid_sim_field_splat(self.h, C.byref(p)), "field_splat")

    def field_filter(self):
        return check(lib().fluid_sim_field_filter(self.h), "field_filter")

    def field_read(self):
        h, w = self._field_shape
        f2 = np.zeros((h, w, 2), np.float32)
        f4 = np.zeros((h, w, 4), np.float32)
        check(lib().fluid_sim_field_read(self.h, _p(f2), _p(f4)), "field_read")
        return f2, f4

    def field(self, name):
        n = self.n
        shapes = dict(density=(n, np.float32), alpha=(n, np.float32), kd=(n, np.float32),
                      pressure=(n, np.float32), nbr_n=(n, np.uint32),
                      starts=(self.keyspace + 1, np.uint32), perm=(n, np.uint32),
                      work_pos=((n, 4), np.float32), work_vel=((n, 4), np.float32),
                      accel=((n, 4), np.float32), xsph=((n, 4), np.float32),
                      wall_grad=((n, 4), np.float32), counters=(2, np.uint32))
        shape, dt = shapes[name]
        out = np.zeros(shape, dt)
        check(lib().fluid_sim_read_field(self.h, FIELDS[name], _p(out), out.nbytes), name)
        return out

    def profile_step(self, st, cap=128):
        ms = (C.c_float * cap)()
        names = (C.c_char_p * cap)()
        k = lib().fluid_sim_profile_step(self.h, C.byref(st), ms, names, cap)
        if k < 0:
            raise FluidError(k, "profile_step")
        return [(names[i].decode(), ms[i]) for i in range(k)]

    def kernels_per_substep(self):
        return lib().fluid_sim_kernels_per_substep(self.h)

    def stream(self):
        return lib().fluid_sim_stream(self.h)


class Controller:
    """The frame controller of Renderer::frame (render.rs:3021-3098), host only."""

    def __init__(self, spacing, extent, cap=16):
        ext = (C.c_float * 2)(*[float(v) for v in extent])
        self.h = lib().fluid_controller_create(spacing, C.byref(ext), cap)
        if not self.h:
            raise FluidError(ERR_ARG, "fluid_controller_create")

    def close(self):
        if getattr(self, "h", None):
            lib().fluid_controller_destroy(self.h)
            self.h = None

    def __del__(self):
        # at interpreter exit the module's globals may already be gone; the
        # process's CUDA context goes with it
        try:
            self.close()
        except (TypeError, AttributeError):
            pass

    def touch(self, slot, x, y, down):
        check(lib().fluid_controller_touch(self.h, slot, x, y, 1 if down else 0), "touch")

    def plan(self, gravity, user_acceleration=(0, 0, 0), rotation_rate=(0, 0, 0), now_ms=0.0,
             v_max=0.0):
        v = lambda t: FluidVec3(*[float(x) for x in t])
        m = FluidMotion(v(gravity), v(user_acceleration), v(rotation_rate))
        out = FluidFramePlan()
        check(lib().fluid_controller_plan(self.h, C.byref(m), now_ms, v_max, C.byref(out)), "plan")
        return out


def grid_slabs():
    """Slabs per cell along x in a simulation's grid keys (fluid_sim_grid_slabs)."""
    return int(lib().fluid_sim_grid_slabs())


def substeps_for(dt, v_max, spacing, cap):
    return lib().fluid_substeps_for(dt, v_max, spacing, cap)


def grid_of(params):
    g = FluidGrid()
    g.min[:] = list(params.box_min) if hasattr(params, "box_min") else list(params.min)
    g.cell = params.cell
    g.dims[:] = list(params.dims)
    return g


def grid_build_host(pos4, grid):
    """fluid_grid_build_host: (starts[C+1], perm[n]) for host positions."""
    pos4 = np.ascontiguousarray(pos4, np.float32).reshape(-1, 4)
    n = pos4.shape[0]
    C_ = grid.dims[0] * grid.dims[1] * grid.dims[2]
    starts = np.zeros(C_ + 1, np.uint32)
    perm = np.zeros(n, np.uint32)
    check(lib().fluid_grid_build_host(_p(pos4), n, C.byref(grid), _p(starts), _p(perm)),
          "grid_build_host")
    return starts, perm


def grid_build_device(pos4_ptr, n, grid, keys_ptr, starts_ptr, perm_ptr, ws_ptr, ws_bytes,
                      stream=None):
    """fluid_grid_build on device pointers (ints, e.g. torch data_ptr())."""
    return check(lib().fluid_grid_build(C.c_void_p(pos4_ptr), n, C.byref(grid),
                                        C.c_void_p(keys_ptr) if keys_ptr else None,
                                        C.c_void_p(starts_ptr), C.c_void_p(perm_ptr),
                                        C.c_void_p(ws_ptr), ws_bytes,
                                        C.c_void_p(stream) if stream else None), "grid_build")


def grid_build_status(ws_ptr, n, grid, stream=None):
    """fluid_grid_build_status: the status code of the last build on the
    workspace (OK, or ERR_TIMEOUT when its starts and permutation are
    invalid). Not raised, returned."""
    return lib().fluid_grid_build_status(C.c_void_p(ws_ptr), n, C.byref(grid),
                                         C.c_void_p(stream) if stream else None)


def grid_workspace_bytes(n, grid):
    return lib().fluid_grid_workspace_bytes(n, C.byref(grid))
