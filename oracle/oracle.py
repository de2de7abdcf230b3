"""TEST INFRASTRUCTURE: ctypes driver of the CPU oracle (smokesim_oracle.c).

Only tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, and only as the checker / baseline.  Parity unpinned: the reference
(GLSL compute under OpenGL) cannot run here and ships no golden vectors; the
oracle is a line-by-line C restatement of its shaders.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
import threading

import numpy as np

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(ORACLE_DIR))
from smokesim_b200 import abi  # noqa: E402  (POD types only)

_libs = {}
_lock = threading.Lock()


def build(force=False):
    """Compile liboracle_f32.so / liboracle_f64.so with the committed Makefile."""
    targets = [os.path.join(ORACLE_DIR, f) for f in ("liboracle_f32.so", "liboracle_f64.so")]
    sources = [os.path.join(ORACLE_DIR, "smokesim_oracle.c"), os.path.join(ORACLE_DIR, "..", "include", "smokesim.h")]
    newest = max(os.path.getmtime(f) for f in sources if os.path.exists(f))
    if not force and all(os.path.exists(t) and os.path.getmtime(t) >= newest for t in targets):
        return
    env = dict(os.environ)
    env.pop("CC", None)
    subprocess.run(["make", "-C", ORACLE_DIR] + (["-B"] if force else []), check=True, env=env,
                   stdout=subprocess.PIPE, stderr=subprocess.STDOUT)


def load(precision="f32"):
    with _lock:
        if precision in _libs:
            return _libs[precision]
        path = os.path.join(ORACLE_DIR, f"liboracle_{precision}.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        vp, i, sz = C.c_void_p, C.c_int, C.c_size_t
        L.og_create.argtypes = [C.POINTER(abi.Desc)]
        L.og_create.restype = vp
        L.og_destroy.argtypes = [vp]
        L.og_levels.argtypes = [vp, C.POINTER(C.c_int * 3)]
        L.og_set_fp16_storage.argtypes = [vp, i, i]
        L.og_set_scene.argtypes = [vp, C.POINTER(abi.Emitter), i, C.POINTER(abi.Obstacle), i, C.POINTER(abi.Box), i]
        L.og_get_scene.argtypes = [vp, C.POINTER(abi.Emitter), i, C.POINTER(abi.Obstacle), i]
        L.og_set_field.argtypes = [vp, i, C.POINTER(C.c_float), sz]
        L.og_get_field.argtypes = [vp, i, C.POINTER(C.c_float), sz]
        L.og_get_field_f64.argtypes = [vp, i, C.POINTER(C.c_double), sz]
        L.og_set_field_f64.argtypes = [vp, i, C.POINTER(C.c_double), sz]
        L.og_set_emitter_force.argtypes = [vp, C.POINTER(C.c_float * 3)]
        L.og_set_emitter_force_f64.argtypes = [vp, C.POINTER(C.c_double * 3)]
        L.og_set_coarse_matrix.argtypes = [vp, i]
        L.og_set_coarse_matrix.restype = None
        L.og_set_force_field.argtypes = [vp, i, C.POINTER(C.c_float)]
        L.og_set_force_field.restype = None
        L.og_set_force_field_f64.argtypes = [vp, i, C.POINTER(C.c_double)]
        L.og_set_force_field_f64.restype = None
        L.og_render.argtypes = [vp, C.POINTER(abi.RenderDesc), C.c_void_p]
        L.og_render.restype = None
        L.og_set_velocity_other.argtypes = [vp, i, C.POINTER(C.c_float), sz]
        L.og_get_level.argtypes = [vp, i, i, C.POINTER(C.c_float), sz]
        L.og_set_level.argtypes = [vp, i, i, C.POINTER(C.c_float), sz]
        L.og_run_physics_step.argtypes = [vp, C.POINTER(abi.Params)]
        L.og_get_stats.argtypes = [vp, C.POINTER(abi.Stats)]
        for n in ["og_stage_advect_velocities", "og_stage_apply_buoyancy", "og_stage_apply_vorticity",
                  "og_stage_update_velocities", "og_stage_advect_smoke", "og_stage_handle_emitters",
                  "og_stage_multigrid", "og_stage_obstacles"]:
            getattr(L, n).argtypes = [vp, C.POINTER(abi.Params)]
        real = C.c_float if precision == "f32" else C.c_double
        L.og_smooth_mode.argtypes = [vp, i, i, real, real, i]
        L.og_compute_residual_mode.argtypes = [vp, i, real, real, i]
        L.og_compute_restrict.argtypes = [vp, i]
        L.og_prolong_and_add.argtypes = [vp, i]
        L.og_v_cycle.argtypes = [vp, i, C.POINTER(abi.MGSchedule), real, real]
        L.og_restrict_solid_all.argtypes = [vp]
        L.og_divergence_norm.argtypes = [vp]
        L.og_divergence_norm.restype = C.c_double
        L.og_projected_residual_norm.argtypes = [vp, real, real]
        L.og_projected_residual_norm.restype = C.c_double
        L.og_update_emitters_status.argtypes = [vp, C.c_float]
        L.og_update_emitters_status.restype = None
        L.og_init_solid_map.argtypes = [vp]
        L.og_update_solid_map.argtypes = [vp]
        L.og_num_threads.restype = i
        L.og_set_num_threads.argtypes = [i]
        _libs[precision] = L
        return L


def _fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class OracleSim:
    """One oracle grid (CPU).  Mirrors the method names of smokesim_b200.Sim."""

    def __init__(self, desc: abi.Desc, precision="f32"):
        self.L = load(precision)
        self.precision = precision
        self.desc = desc
        self.dim = desc.dim
        self.n = (desc.n[0], desc.n[1], 1 if desc.dim == 2 else desc.n[2])
        self.nch = 3 if desc.density_channels == 3 else 1
        self.h = self.L.og_create(C.byref(desc))
        if not self.h:
            raise ValueError("oracle: bad grid description")
        sizes = (C.c_int * 3 * abi.SS_MAX_LEVELS)()
        self.levels = self.L.og_levels(self.h, sizes)
        self.level_sizes = [tuple(sizes[l]) for l in range(self.levels)]

    def close(self):
        if self.h:
            self.L.og_destroy(self.h)
            self.h = None

    __del__ = close

    def shape(self, field):
        return abi.field_shape(self.dim, self.n, field, self.nch)

    def set_scene(self, emitters=(), obstacles=(), boxes=()):
        em = (abi.Emitter * max(1, len(emitters)))(*emitters)
        ob = (abi.Obstacle * max(1, len(obstacles)))(*obstacles)
        bx = (abi.Box * max(1, len(boxes)))(*boxes)
        self.L.og_set_scene(self.h, em, len(emitters), ob, len(obstacles), bx, len(boxes))

    def get_scene(self, n_emitters, n_obstacles):
        em = (abi.Emitter * max(1, n_emitters))()
        ob = (abi.Obstacle * max(1, n_obstacles))()
        self.L.og_get_scene(self.h, em, n_emitters, ob, n_obstacles)
        return list(em)[:n_emitters], list(ob)[:n_obstacles]

    def set_field(self, field, arr):
        a = np.ascontiguousarray(arr, dtype=np.float32).reshape(-1)
        rc = self.L.og_set_field(self.h, field, _fptr(a), a.size)
        if rc:
            raise ValueError(f"oracle set_field({field}) size {a.size}")

    def set_field_f64(self, field, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64).ravel()
        rc = self.L.og_set_field_f64(self.h, field, a.ctypes.data_as(C.POINTER(C.c_double)), a.size)
        if rc:
            raise ValueError(f"oracle set_field_f64({field}) rc={rc}")

    def render(self, desc):
        out = np.empty((desc.height, desc.width, 4), np.uint8)
        self.L.og_render(self.h, C.byref(desc), out.ctypes.data)
        return out

    def set_force_field(self, field):
        """Coarse control force field: an array of shape (3, n, n, n) (or
        None to remove it); float64 input is kept at FP64 precision."""
        if field is None:
            self.L.og_set_force_field(self.h, 0, None)
            return
        a = np.asarray(field)
        n = a.shape[-1]
        assert a.shape == (3, n, n, n), a.shape
        if a.dtype == np.float64:
            a = np.ascontiguousarray(a)
            self.L.og_set_force_field_f64(self.h, n, a.ctypes.data_as(C.POINTER(C.c_double)))
        else:
            a = np.ascontiguousarray(a, dtype=np.float32)
            self.L.og_set_force_field(self.h, n, a.ctypes.data_as(C.POINTER(C.c_float)))

    def set_coarse_matrix(self, on):
        """Mixed solve: coarsest level by its response matrix (default, as
        the CUDA path) or swept (the CUDA path's SMOKESIM_COARSE_SWEEPS=1)."""
        self.L.og_set_coarse_matrix(self.h, int(bool(on)))

    def set_emitter_force(self, force):
        f = (C.c_double * 3)(*[float(x) for x in force])
        self.L.og_set_emitter_force_f64(self.h, C.byref(f))

    def get_field(self, field, f64=False):
        shp = self.shape(field)
        n = int(np.prod(shp))
        if f64:
            a = np.empty(n, np.float64)
            rc = self.L.og_get_field_f64(self.h, field, a.ctypes.data_as(C.POINTER(C.c_double)), n)
        else:
            a = np.empty(n, np.float32)
            rc = self.L.og_get_field(self.h, field, _fptr(a), n)
        if rc:
            raise ValueError(f"oracle get_field({field})")
        return a.reshape(shp)

    def set_velocity_other(self, comp, arr):
        a = np.ascontiguousarray(arr, dtype=np.float32).reshape(-1)
        if self.L.og_set_velocity_other(self.h, comp, _fptr(a), a.size):
            raise ValueError("oracle set_velocity_other")

    def get_level(self, level, what):
        nx, ny, nz = self.level_sizes[level]
        a = np.empty(nx * ny * nz, np.float32)
        if self.L.og_get_level(self.h, level, what, _fptr(a), a.size):
            raise ValueError("oracle get_level")
        return a.reshape(nz, ny, nx)

    def set_level(self, level, what, arr):
        a = np.ascontiguousarray(arr, dtype=np.float32).reshape(-1)
        if self.L.og_set_level(self.h, level, what, _fptr(a), a.size):
            raise ValueError("oracle set_level")

    def step(self, params, nsteps=1):
        for _ in range(nsteps):
            self.L.og_run_physics_step(self.h, C.byref(params))

    def stats(self):
        s = abi.Stats()
        self.L.og_get_stats(self.h, C.byref(s))
        return s

    # single stages
    def stage(self, name, params):
        getattr(self.L, "og_stage_" + name)(self.h, C.byref(params))

    def update_emitters_status(self, params):
        self.L.og_update_emitters_status(self.h, params.current_time)

    def smooth(self, level, iterations, params):
        self.L.og_smooth_mode(self.h, level, iterations, params.time_step, params.density, params.mg.ref_quirks)

    def compute_residual(self, level, params):
        self.L.og_compute_residual_mode(self.h, level, params.time_step, params.density, params.mg.ref_quirks)

    def compute_restrict(self, level):
        self.L.og_compute_restrict(self.h, level)

    def prolong_and_add(self, level):
        self.L.og_prolong_and_add(self.h, level)

    def v_cycle(self, level, params):
        self.L.og_v_cycle(self.h, level, C.byref(params.mg), params.time_step, params.density)

    def restrict_solid_all(self):
        self.L.og_restrict_solid_all(self.h)

    def divergence_norm(self):
        return self.L.og_divergence_norm(self.h)

    def projected_residual_norm(self, params):
        return self.L.og_projected_residual_norm(self.h, params.time_step, params.density)


def num_threads(precision="f32"):
    return load(precision).og_num_threads()


def set_num_threads(n, precision="f32"):
    load(precision).og_set_num_threads(n)
